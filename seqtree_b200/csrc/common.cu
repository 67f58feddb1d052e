// Per-device context, workspace, pinned host cache and sequence-set upload/encoding.
#include <unistd.h>

#include "common.cuh"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <set>
#include <tuple>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace stb {

// ----------------------------------------------------------------------------- launches -----
namespace {
thread_local int t_launches = 0;
thread_local const char* t_kernel = "";
std::atomic<int64_t> g_launches{0};
}  // namespace

void note_launch(const char* kernel_name, int count) {
    t_launches += count;
    g_launches.fetch_add(count, std::memory_order_relaxed);
    if (kernel_name && *kernel_name) t_kernel = kernel_name;
}
void reset_launches() {
    t_launches = 0;
    t_kernel = "";
}
int last_launches() { return t_launches; }
int64_t total_launches() { return g_launches.load(std::memory_order_relaxed); }
const char* last_kernel() { return t_kernel; }

// ----------------------------------------------------------------------------- tuning -------
namespace {
std::mutex g_tune_mu;
std::map<std::string, int> g_tune;        // "device|key" -> choice
std::map<std::string, std::string> g_tune_log;  // "device|key" -> measured times

bool tune_on() {
    static const bool on = [] {
        const char* v = std::getenv("SEQTREE_B200_TUNE");
        return !(v && *v == '0');
    }();
    return on;
}
std::string dev_key(const std::string& key) {
    int dev = 0;
    cudaGetDevice(&dev);
    return std::to_string(dev) + "|" + key;
}
}  // namespace

bool tuning_enabled() { return tune_on(); }

void ensure_smem_limit(const void* kernel, size_t bytes) {
    // The attribute is a limit: it only ever grows here, so a launch that needs less than an
    // earlier one still fits (setting it to each call's own size would shrink it under a later,
    // larger launch that the cache believed already allowed).
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    STB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = limit[std::make_pair(dev, kernel)];
    if (bytes <= cur) return;
    STB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    cur = bytes;
}

int tuned_lookup(const std::string& key) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(dev_key(key));
    return it == g_tune.end() ? -1 : it->second;
}

int tuned_run(const std::string& key, int n, int fallback, const std::function<void(int)>& run,
              cudaStream_t stream) {
    const std::string k = dev_key(key);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(k);
        if (it != g_tune.end()) {
            run(it->second);
            return it->second;
        }
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    STB_CUDA(cudaStreamIsCapturing(stream, &cs));
    if (!tune_on() || n < 2 || cs != cudaStreamCaptureStatusNone) {
        run(fallback);
        return fallback;
    }
    cudaEvent_t e0, e1;
    STB_CUDA(cudaEventCreate(&e0));
    STB_CUDA(cudaEventCreate(&e1));
    float best = 0.f;
    int pick = fallback;
    std::string log;
    std::vector<float> ms(size_t(n), 0.f);
    try {
        for (int c = 0; c < n; ++c) {
            run(c);  // untimed: first-use effects (plans, module loading, workspace growth)
            // the median of several timed runs (one run's time varies by several percent,
            // enough to reorder variants that are close): three, or up to nine while the runs
            // so far took under 2 ms in all, so that short kernels get a steadier median
            std::vector<float> t;
            float spent = 0.f;
            while (t.size() < 3 || (t.size() < 9 && spent < 2.0f)) {
                float ti = 0.f;
                STB_CUDA(cudaEventRecord(e0, stream));
                run(c);
                STB_CUDA(cudaEventRecord(e1, stream));
                STB_CUDA(cudaEventSynchronize(e1));
                STB_CUDA(cudaEventElapsedTime(&ti, e0, e1));
                t.push_back(ti);
                spent += ti;
            }
            std::nth_element(t.begin(), t.begin() + t.size() / 2, t.end());
            ms[size_t(c)] = t[t.size() / 2];
            if (c == 0 || ms[size_t(c)] < best) {
                best = ms[size_t(c)];
                pick = c;
            }
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    char buf[64];
    for (int c = 0; c < n; ++c) {
        std::snprintf(buf, sizeof buf, "%s%d:%.3fms", c ? " " : "", c, double(ms[size_t(c)]));
        log += buf;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[k] = pick;
    g_tune_log[k] = log;
    return pick;
}

// One line per tuned key: "device|key -> choice (variant:time ...)".
std::string tuning_table() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::string out;
    for (auto& [k, v] : g_tune) out += k + " -> " + std::to_string(v) + " (" + g_tune_log[k] + ")\n";
    return out;
}

// ----------------------------------------------------------------------------- tracing ------
namespace {
bool trace_on() {
    static const bool on = [] {
        const char* v = std::getenv("SEQTREE_B200_TRACE");
        return v && *v && *v != '0';
    }();
    return on;
}
double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}
thread_local std::string t_trace;
}  // namespace

Phase::Phase(const char* n) : name(n), t0(0) {
    nvtxRangePushA(n);
    if (trace_on()) t0 = now_ms();
}

Phase::~Phase() {
    nvtxRangePop();
    if (trace_on()) {
        char buf[96];
        std::snprintf(buf, sizeof buf, " %s=%.3fms", name, now_ms() - t0);
        t_trace += buf;
    }
}

void trace_report(const char* call) {
    if (trace_on() && !t_trace.empty()) std::fprintf(stderr, "[seqtree_b200] %s:%s\n", call, t_trace.c_str());
    t_trace.clear();
}

// ----------------------------------------------------------------------------- buffers ------
void* DevBuf::get(size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (bytes > cap) {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes + bytes / 8, 4096);
        want = (want + 255) & ~size_t(255);
        STB_CUDA(cudaMalloc(&ptr, want));
        cap = want;
    }
    return ptr;
}

void* DevBuf::grow_keep(size_t bytes, size_t keep, cudaStream_t stream) {
    if (bytes <= cap) return ptr;
    size_t want = std::max<size_t>(bytes + bytes / 2, 4096);
    want = (want + 255) & ~size_t(255);
    void* fresh = nullptr;
    STB_CUDA(cudaMalloc(&fresh, want));
    if (ptr && keep) {
        const cudaError_t e = cudaMemcpyAsync(fresh, ptr, std::min(keep, cap),
                                              cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) {
            cudaFree(fresh);
            STB_CUDA(e);
        }
        STB_CUDA(cudaStreamSynchronize(stream));
    }
    if (ptr) cudaFree(ptr);
    ptr = fresh;
    cap = want;
    return ptr;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
}

DevBuf::~DevBuf() {
    // Contexts live until process exit; the driver reclaims device memory then.
}

void h2d(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    if (bytes == 0) return;
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    STB_CUDA(cudaStreamIsCapturing(stream, &st));
    if (st != cudaStreamCaptureStatusNone)
        fail(ST_EINVAL, "seqtree_b200: this call has tables or plans to upload; make the same call "
                        "once before capturing it into a CUDA graph");
    STB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
}

bool same_as_last(std::vector<uint8_t>& slot, const void* data, size_t bytes) {
    if (slot.size() == bytes && (bytes == 0 || std::memcmp(slot.data(), data, bytes) == 0))
        return true;
    slot.assign(static_cast<const uint8_t*>(data), static_cast<const uint8_t*>(data) + bytes);
    return false;
}

// ----------------------------------------------------------------------------- context ------
namespace {
std::mutex g_ctx_mu;
std::map<int, std::unique_ptr<Context>> g_ctx;
}  // namespace

Context& context() {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    int n = 0;
    if (e == cudaSuccess) e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= 0 || dev < 0) {
        cudaGetLastError();
        fail(ST_ENODEV, std::string("seqtree_b200: no usable CUDA device (") +
                            cudaGetErrorString(e == cudaSuccess ? cudaErrorNoDevice : e) + ")");
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_ctx.find(dev);
    if (it != g_ctx.end()) return *it->second;
    auto c = std::make_unique<Context>();
    c->device = dev;
    STB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    STB_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev));
    STB_CUDA(cudaDeviceGetAttribute(&c->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                    dev));
    STB_CUDA(cudaMalloc(&c->flags_d, 64 * sizeof(int64_t)));
    STB_CUDA(cudaHostAlloc(&c->flags_h, 64 * sizeof(int64_t), cudaHostAllocDefault));
    Context& ref = *c;
    g_ctx.emplace(dev, std::move(c));
    return ref;
}

int32_t alphabet_size(int32_t alphabet) {
    switch (alphabet) {
        case ST_ALPHABET_AA: return 24;   // "ARNDCQEGHILKMFPSTWYVBZX*"  (src/codec.cpp:9)
        case ST_ALPHABET_NT: return 4;    // "ACGT"                      (src/codec.cpp:10)
        case ST_ALPHABET_IUPAC: return 15;// "ACGTRYSWKMBDHVN"           (src/codec.cpp:11)
        default: return 0;
    }
}

// ----------------------------------------------------------------------------- encoding -----
namespace {

const char* symbols(int32_t alphabet) {
    switch (alphabet) {
        case ST_ALPHABET_AA: return "ARNDCQEGHILKMFPSTWYVBZX*";
        case ST_ALPHABET_NT: return "ACGT";
        default: return "ACGTRYSWKMBDHVN";
    }
}

struct Lut {
    uint8_t v[256];
};

// Case-insensitive symbol -> code table; 0xFF marks symbols outside the alphabet
// (the reference Codec, src/codec.cpp:23-35).
Lut make_lut(int32_t alphabet) {
    Lut l;
    std::memset(l.v, 0xFF, sizeof l.v);
    const char* s = symbols(alphabet);
    for (int i = 0; s[i]; ++i) {
        unsigned char up = static_cast<unsigned char>(s[i]);
        unsigned char lo = (up >= 'A' && up <= 'Z') ? static_cast<unsigned char>(up - 'A' + 'a') : up;
        l.v[up] = static_cast<uint8_t>(i);
        l.v[lo] = static_cast<uint8_t>(i);
    }
    return l;
}

// One pass over the bytes: code = lut[byte]; the smallest index of an invalid byte is
// recorded with atomicMin so the error names the same symbol the reference's sequential
// encoder stops at.
__global__ void encode_kernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out,
                              int64_t n, Lut lut, unsigned long long* first_bad, uint8_t bad_code) {
    __shared__ uint8_t s_lut[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s_lut[i] = lut.v[i];
    __syncthreads();
    const int64_t stride = int64_t(gridDim.x) * blockDim.x * 4;
    for (int64_t base = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) * 4; base < n;
         base += stride) {
        if (base + 4 <= n) {
            uint32_t w = *reinterpret_cast<const uint32_t*>(in + base);  // buffers are padded
            uint32_t o = 0;
            bool bad = false;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                uint8_t c = s_lut[(w >> (8 * b)) & 0xFF];
                if (c == 0xFF) {
                    if (!bad) atomicMin(first_bad, (unsigned long long)(base + b));
                    bad = true;
                    c = bad_code;
                }
                o |= uint32_t(c) << (8 * b);
            }
            *reinterpret_cast<uint32_t*>(out + base) = o;
        } else {
            for (int64_t i = base; i < n; ++i) {
                uint8_t c = s_lut[in[i]];
                if (c == 0xFF) {
                    atomicMin(first_bad, (unsigned long long)i);
                    c = bad_code;
                }
                out[i] = c;
            }
        }
    }
}

__global__ void lengths_kernel(const int64_t* __restrict__ off, int32_t* __restrict__ len,
                               int64_t count) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) len[i] = int32_t(off[i + 1] - off[i]);
}

}  // namespace

namespace {
std::atomic<uint64_t> g_next_uid{1};
}  // namespace

std::unique_ptr<st_seqset_s> row_view(const st_seqset_s& s, int64_t rows) {
    auto v = std::make_unique<st_seqset_s>();
    rows = std::max<int64_t>(0, std::min(rows, s.count));
    v->device = s.device;
    v->alphabet = s.alphabet;
    v->count = rows;
    v->h_off.assign(s.h_off.begin(), s.h_off.begin() + (rows + 1));
    v->h_len.assign(s.h_len.begin(), s.h_len.begin() + rows);
    v->total = v->h_off.back();
    v->max_len = rows ? *std::max_element(v->h_len.begin(), v->h_len.end()) : 0;
    v->d_bytes = s.d_bytes;
    v->d_off = s.d_off;
    v->d_len = s.d_len;
    v->owns = false;
    v->uid = g_next_uid.fetch_add(1);
    return v;
}

st_seqset_s* make_seqset(const st_strings* s, int32_t alphabet, cudaStream_t stream,
                         int64_t* bad_index, char* bad_char, DevBuf* storage, int defer_word) {
    std::atomic<uint64_t>& next_uid = g_next_uid;
    if (!s || (s->count > 0 && !s->offsets)) fail(ST_EINVAL, "seqtree_b200: null sequence set");
    if (alphabet != -1 && alphabet_size(alphabet) == 0)
        fail(ST_EINVAL, "unknown alphabet code " + std::to_string(alphabet));
    Context& ctx = context();
    auto set = std::make_unique<st_seqset_s>();
    set->device = ctx.device;
    set->uid = next_uid.fetch_add(1);
    set->alphabet = alphabet;
    set->count = s->count;
    set->h_off.assign(s->offsets, s->offsets + (s->count + 1));
    if (set->h_off.empty()) set->h_off.push_back(0);
    const int64_t base = set->h_off[0];
    for (auto& o : set->h_off) o -= base;
    set->total = set->h_off.back();
    set->h_len.resize(size_t(s->count));
    int32_t mx = 0;
    for (int64_t i = 0; i < s->count; ++i) {
        int64_t l = set->h_off[i + 1] - set->h_off[i];
        if (l < 0 || l > INT32_MAX) fail(ST_EINVAL, "seqtree_b200: offsets must be non-decreasing");
        set->h_len[size_t(i)] = int32_t(l);
        mx = std::max<int32_t>(mx, int32_t(l));
    }
    set->max_len = mx;
    const size_t padded = size_t(set->total) + 64;
    if (storage) {
        set->owns = false;
        set->d_bytes = storage[0].as<uint8_t>(padded);
        set->d_off = storage[1].as<int64_t>(size_t(s->count + 1));
        set->d_len = storage[2].as<int32_t>(size_t(std::max<int64_t>(s->count, 1)));
    } else {
        STB_CUDA(cudaMalloc(&set->d_bytes, padded));
        STB_CUDA(cudaMalloc(&set->d_off, sizeof(int64_t) * size_t(s->count + 1)));
        STB_CUDA(cudaMalloc(&set->d_len, sizeof(int32_t) * size_t(std::max<int64_t>(s->count, 1))));
    }
    STB_CUDA(cudaMemsetAsync(set->d_bytes, 0, padded, stream));
    STB_CUDA(cudaMemcpyAsync(set->d_off, set->h_off.data(), sizeof(int64_t) * size_t(s->count + 1),
                             cudaMemcpyHostToDevice, stream));
    if (s->count > 0) {
        lengths_kernel<<<unsigned(ceil_div(s->count, 256)), 256, 0, stream>>>(set->d_off, set->d_len,
                                                                              s->count);
        STB_CUDA(cudaGetLastError());
        note_launch(nullptr);
    }
    if (set->total > 0) {
        const uint8_t* src = reinterpret_cast<const uint8_t*>(s->bytes) + base;
        if (alphabet < 0) {
            STB_CUDA(cudaMemcpyAsync(set->d_bytes, src, size_t(set->total), cudaMemcpyHostToDevice,
                                     stream));
        } else {
            DevBuf& raw = ctx.work_c;
            uint8_t* d_raw = raw.as<uint8_t>(padded);
            STB_CUDA(cudaMemsetAsync(d_raw + set->total, 0, 64, stream));
            STB_CUDA(cudaMemcpyAsync(d_raw, src, size_t(set->total), cudaMemcpyHostToDevice, stream));
            auto* flag = reinterpret_cast<unsigned long long*>(ctx.flags_d + (defer_word > 0 ? defer_word : 0));
            STB_CUDA(cudaMemsetAsync(flag, 0xFF, sizeof(unsigned long long), stream));
            const Lut lut = make_lut(alphabet);
            const int64_t words = ceil_div(set->total, 4);
            const unsigned grid = unsigned(std::min<int64_t>(ceil_div(words, 256), ctx.num_sms * 8));
            encode_kernel<<<grid, 256, 0, stream>>>(d_raw, set->d_bytes, set->total, lut, flag,
                                                    uint8_t(defer_word >= 0 ? 0 : 0xFF));
            STB_CUDA(cudaGetLastError());
            note_launch(nullptr);
            if (defer_word >= 0) return set.release();
            const unsigned long long none = ~0ull;
            STB_CUDA(cudaMemcpyAsync(ctx.flags_h, flag, sizeof none, cudaMemcpyDeviceToHost, stream));
            STB_CUDA(cudaStreamSynchronize(stream));
            const unsigned long long bad = static_cast<unsigned long long>(ctx.flags_h[0]);
            if (bad != none) {
                if (bad_index) {
                    *bad_index = int64_t(bad);
                    if (bad_char) *bad_char = char(src[bad]);
                } else {
                    fail(ST_EINVAL, std::string("symbol '") + char(src[bad]) +
                                        "' is not in the alphabet");
                }
            } else if (bad_index) {
                *bad_index = -1;
            }
        }
    } else if (bad_index) {
        *bad_index = -1;
    }
    return set.release();
}

}  // namespace stb

st_seqset_s::~st_seqset_s() {
    if (!owns) return;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    if (d_bytes) cudaFree(d_bytes);
    if (d_off) cudaFree(d_off);
    if (d_len) cudaFree(d_len);
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
}

// ----------------------------------------------------------------------------- pinned -------
namespace stb {
namespace {
std::mutex g_pin_mu;
std::multimap<size_t, void*> g_pin_free;  // size -> block
std::map<void*, size_t> g_pin_size;
}  // namespace

void* host_alloc(uint64_t bytes) {
    size_t want = size_t(bytes == 0 ? 1 : bytes);
    want = (want + 4095) & ~size_t(4095);
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto it = g_pin_free.lower_bound(want);
        if (it != g_pin_free.end() && it->first <= want + want / 4) {
            void* p = it->second;
            g_pin_free.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, want, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_size[p] = want;
    return p;
}

// Returned blocks stay pinned for reuse up to a limit in total; beyond that they are unpinned and
// freed.  The limit is an eighth of physical memory (at least 8 GiB), or the number of GiB in
// SEQTREE_B200_PIN_CACHE_GB: pinning and unpinning cost about a second per 10 GB, so a repeated
// large sparse search (22 GB of rows) reuses its blocks instead of paying that on every call,
// while a machine's memory is never mostly locked by a cache.
size_t pin_cache_limit() {
    static const size_t lim = [] {
        if (const char* v = std::getenv("SEQTREE_B200_PIN_CACHE_GB")) {
            const double gb = std::atof(v);
            if (gb >= 0) return size_t(gb * double(size_t(1) << 30));
        }
        const long pages = sysconf(_SC_PHYS_PAGES), psz = sysconf(_SC_PAGE_SIZE);
        const size_t phys = pages > 0 && psz > 0 ? size_t(pages) * size_t(psz) : size_t(64) << 30;
        return std::max(size_t(8) << 30, phys / 8);
    }();
    return lim;
}

void host_free(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_pin_size.find(p);
    if (it == g_pin_size.end()) return;
    size_t cached = 0;
    for (const auto& kv : g_pin_free) cached += kv.first;
    if (cached + it->second > pin_cache_limit()) {
        g_pin_size.erase(it);
        cudaFreeHost(p);
        return;
    }
    g_pin_free.emplace(it->second, p);
}
}  // namespace stb
