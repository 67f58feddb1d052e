// Levenshtein matrix for callers that cannot allocate device memory.
//
// Some callers cannot let a library call cudaMalloc.  Examples are a process whose device memory
// is owned by its own caching allocator, or one that reserved a fixed budget up front, and a
// latency-critical path where the cost or the failure of an allocation is not acceptable.  This
// file gives them one entry point, st_levenshtein_matrix_noalloc, that allocates nothing: the
// caller passes the input sequences and the output matrix in device memory it owns, and the
// kernel's scratch (one DP row per thread) lives in a fixed-size array compiled into the library.
//
// The array is kScratchBytes (32 MiB) per device; every GPU that loads the library holds it until
// the process exits.  Its device address is looked up once per device, with that device current,
// on the first call on that device (so make that first call before any stream capture).  All
// calls share the array.  The two header words that size the launch are cleared, filled and read
// back under a per-device host lock, so concurrent host threads cannot size a launch from another
// call's header.  The DP-row region after the header is not locked: calls whose kernels overlap
// on the GPU (for example, on two streams at once) race on it and may return wrong distances.
// Each kernel also checks that its row fits the capacity it was launched with and writes -1
// (never a distance) for a pair whose row would not, touching no scratch for it.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/seqtree_b200.h"

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr size_t kScratchWords = kScratchBytes / sizeof(int32_t);
constexpr size_t kHeaderWords = 64;  // words 0/1: longest a / longest b of the current call
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) int32_t g_noalloc_scratch[kScratchWords];

int32_t* g_scratch_addr[kMaxDevices];  // device address of g_noalloc_scratch, per device
std::mutex g_setup_mu;
std::mutex g_call_mu[kMaxDevices];  // serialises the header's clear / fill / read per device

int32_t set_error(st_error* err, int32_t code, const char* msg) {
    if (err) {
        err->code = code;
        std::snprintf(err->message, sizeof err->message, "%s", msg);
    }
    return code;
}

// Longest sequence of each side (offsets are non-decreasing; lengths fit int32).
__global__ void longest_kernel(const int64_t* __restrict__ a_off, int64_t N,
                               const int64_t* __restrict__ b_off, int64_t K, int32_t* hdr) {
    int32_t la = 0, lb = 0;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += stride)
        la = max(la, int32_t(a_off[i + 1] - a_off[i]));
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < K; k += stride)
        lb = max(lb, int32_t(b_off[k + 1] - b_off[k]));
    if (la) atomicMax(&hdr[0], la);
    if (lb) atomicMax(&hdr[1], lb);
}

// The single-row unit-cost DP of the reference (src/distance.cpp:78-95): the row runs over the
// shorter string and lives in the fixed scratch, laid out [column][thread].  `row_cap` is the
// number of row words each thread owns (room / threads); a pair whose row (shorter + 1 words)
// exceeds it gets -1 and no scratch access.
__global__ void __launch_bounds__(kThreads)
levenshtein_rows_kernel(const uint8_t* __restrict__ a, const int64_t* __restrict__ ao, int64_t N,
                        const uint8_t* __restrict__ b, const int64_t* __restrict__ bo, int64_t K,
                        int32_t* __restrict__ rows, int64_t row_cap, int32_t* __restrict__ out) {
    const int64_t T = int64_t(gridDim.x) * blockDim.x;
    const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t idx = tid; idx < N * K; idx += T) {
        const int64_t i = idx / K, k = idx - i * K;
        const uint8_t* s = a + ao[i];
        const uint8_t* t = b + bo[k];
        int m = int(ao[i + 1] - ao[i]), n = int(bo[k + 1] - bo[k]);
        if (n > m) {
            const uint8_t* u = s; s = t; t = u;
            int w = m; m = n; n = w;
        }
        int32_t v;
        if (n == 0) {
            v = m;
        } else if (int64_t(n) + 1 > row_cap) {
            v = -1;
        } else {
            for (int j = 0; j <= n; ++j) rows[j * T + tid] = j;
            for (int x = 1; x <= m; ++x) {
                int diag = rows[tid];
                int left = x;
                rows[tid] = x;
                const uint8_t sx = s[x - 1];
                for (int j = 1; j <= n; ++j) {
                    const int up = rows[j * T + tid];
                    const int cur = min(min(up + 1, left + 1), diag + (sx == t[j - 1] ? 0 : 1));
                    diag = up;
                    left = cur;
                    rows[j * T + tid] = cur;
                }
            }
            v = rows[n * T + tid];
        }
        out[idx] = v;
    }
}

}  // namespace

extern "C" int32_t st_levenshtein_matrix_noalloc(const char* a_bytes, const int64_t* a_offsets,
                                                 int64_t a_count, const char* b_bytes,
                                                 const int64_t* b_offsets, int64_t b_count,
                                                 int32_t* out, void* cuda_stream, st_error* err) {
    if (a_count < 0 || b_count < 0)
        return set_error(err, ST_EINVAL, "seqtree_b200: negative sequence count");
    if (a_count == 0 || b_count == 0) return set_error(err, ST_OK, "");
    if (!a_offsets || !b_offsets || !out || !a_bytes || !b_bytes)
        return set_error(err, ST_EINVAL, "seqtree_b200: null device pointer");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return set_error(err, ST_ENODEV, "seqtree_b200: no usable CUDA device");
    }
    if (dev >= kMaxDevices) return set_error(err, ST_ENODEV, "seqtree_b200: device index too large");
    int32_t* scratch = nullptr;
    {
        // Once per device, with that device current: the device address of the fixed array.
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                char msg[200];
                std::snprintf(msg, sizeof msg, "seqtree_b200: cannot address the fixed scratch: %s",
                              cudaGetErrorString(e));
                cudaGetLastError();
                return set_error(err, ST_ECUDA, msg);
            }
            g_scratch_addr[dev] = static_cast<int32_t*>(p);
        }
        scratch = g_scratch_addr[dev];
    }
    auto stream = static_cast<cudaStream_t>(cuda_stream);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 1;

    // Longest sequence on each side.  The header is cleared, filled and read back under the
    // device's lock, so another host thread's call cannot change it in between.
    std::lock_guard<std::mutex> call_lock(g_call_mu[dev]);
    int32_t longest[2] = {0, 0};
    cudaError_t e = cudaMemsetAsync(scratch, 0, 2 * sizeof(int32_t), stream);
    if (e == cudaSuccess) {
        longest_kernel<<<sms * 4, kThreads, 0, stream>>>(a_offsets, a_count, b_offsets, b_count,
                                                         scratch);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(longest, scratch, sizeof longest, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        char msg[200];
        std::snprintf(msg, sizeof msg, "CUDA error: %s", cudaGetErrorString(e));
        return set_error(err, ST_ECUDA, msg);
    }

    // One DP row of (shorter + 1) words per thread must fit the fixed scratch for at least one
    // block of threads; the grid is the smaller of what fits, about 2,048 threads per SM, and
    // the pair count rounded up to whole blocks.
    const int64_t row = int64_t(longest[0] < longest[1] ? longest[0] : longest[1]) + 1;
    const int64_t room = int64_t(kScratchWords - kHeaderWords);
    const int64_t fit = (room / row / kThreads) * kThreads;
    if (fit < kThreads) {
        char msg[220];
        std::snprintf(msg, sizeof msg,
                      "seqtree_b200: sequences too long for the fixed %zu MiB scratch (a DP row of "
                      "%lld words for %d threads does not fit)",
                      kScratchBytes >> 20, static_cast<long long>(row), kThreads);
        return set_error(err, ST_EINVAL, msg);
    }
    const int64_t pairs = a_count * b_count;
    int64_t threads = fit;
    const int64_t want = int64_t(sms) * 2048;
    if (threads > want) threads = want;
    const int64_t need = (pairs + kThreads - 1) / kThreads * kThreads;
    if (threads > need) threads = need;
    levenshtein_rows_kernel<<<unsigned(threads / kThreads), kThreads, 0, stream>>>(
        reinterpret_cast<const uint8_t*>(a_bytes), a_offsets, a_count,
        reinterpret_cast<const uint8_t*>(b_bytes), b_offsets, b_count, scratch + kHeaderWords,
        room / threads, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        char msg[200];
        std::snprintf(msg, sizeof msg, "CUDA error: %s", cudaGetErrorString(e));
        return set_error(err, ST_ECUDA, msg);
    }
    return set_error(err, ST_OK, "");
}
