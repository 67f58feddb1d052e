// Shared host/device infrastructure of libseqtree_b200: error plumbing, the per-device
// context (stream, grow-only device workspace, pinned staging), and the device-resident
// sequence set.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/seqtree_b200.h"

namespace stb {

// ----------------------------------------------------------------------------- errors -------
// Every failure inside the library is a StError carrying the C-ABI code and the exact message
// the reference raises for the same condition; the extern "C" wrappers turn it into st_error.
struct StError : std::runtime_error {
    int32_t code;
    StError(int32_t c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int32_t code, const std::string& msg) { throw StError(code, msg); }

#define STB_CUDA(expr)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (expr);                                                              \
        if (e_ != cudaSuccess)                                                                \
            ::stb::fail(e_ == cudaErrorMemoryAllocation ? ST_ENOMEM : ST_ECUDA,               \
                        std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " +       \
                            __FILE__ + ":" + std::to_string(__LINE__));                      \
    } while (0)

// Launch bookkeeping: the number of kernels the last call launched and the main variant.
void note_launch(const char* kernel_name, int count = 1);
void reset_launches();

// Host-side phase tracing.  Every Phase opens an NVTX range (visible to Nsight tools, free
// otherwise); with SEQTREE_B200_TRACE=1 in the environment the wall time of each phase is also
// recorded and trace_report() prints one line per call to stderr.
struct Phase {
    const char* name;
    double t0;
    explicit Phase(const char* n);
    ~Phase();
};
void trace_report(const char* call);

// ----------------------------------------------------------------------------- context ------
// A device buffer that only grows; reused across calls so steady-state calls allocate nothing.
struct DevBuf {
    void* ptr = nullptr;
    size_t cap = 0;
    void* get(size_t bytes);
    template <class T>
    T* as(size_t count) { return static_cast<T*>(get(count * sizeof(T))); }
    // Grows to at least `bytes`, keeping the first `keep` bytes (device-to-device on `stream`).
    void* grow_keep(size_t bytes, size_t keep, cudaStream_t stream);
    void release();  // frees the memory now (owners that do not live until exit)
    ~DevBuf();
};

struct Context {
    int device = 0;
    std::mutex mu;              // serialises calls on this device
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    int max_smem_optin = 0;
    // Small device word area for error reporting, with a pinned host mirror.  Word 0: first
    // invalid symbol of an encode; word 8: a bounded wait gave up; word 9: an int32 overflow;
    // words 16-19: byte-presence bitmap.  Words 8-15 are cleared before and read after each
    // host call.
    int64_t* flags_d = nullptr;
    int64_t* flags_h = nullptr;
    // second stream and events of the host calls that overlap the result copy with the kernels
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t block_ev[8] = {};
    // named scratch, grow-only
    DevBuf out_buf, q_codes, r_codes, table_buf, prior_buf, ftab_buf, work_a, work_b, work_c;
    // sparse output: unsorted hit keys and scores, sorted keys, radix-sort scratch
    DevBuf sp_keys, sp_vals, sp_sorted, sp_temp;
    // candidate lists of the learned-proposal kernel; the threshold form's table
    DevBuf topk_cand, prop_thr, prop_items;
    std::vector<uint8_t> prop_thr_key;
    // bf16 operands of the training GEMM, packed in the tensor-core layout
    DevBuf gemm_a, gemm_b;
    // storage of the transient sets made by the host-buffer entry points
    DevBuf tq[3], tr[3];  // bytes, offsets, lengths
    // plans reused by transient sets (rebuilt in place for every call)
    std::shared_ptr<void> tmp_query_plan, tmp_ref_plan, tmp_wave_plan[2];
    // query plan of a row block (sparse calls whose hits are taken in several blocks)
    std::shared_ptr<void> tmp_block_plan;
    // sparse result of the host-buffer sparse call (an st_hits_s)
    std::shared_ptr<void> tmp_hits;
};

// Context of the current CUDA device (created on first use).  Fails with ST_ENODEV when no
// device is usable.
Context& context();

// Raises `kernel`'s dynamic shared-memory limit to `bytes` on the current device, once per
// (device, kernel, size).  The attribute belongs to a device, so a process that uses several
// devices needs the call on each of them.
void ensure_smem_limit(const void* kernel, size_t bytes);

// Host -> device copy of per-call tables or plans.  Refuses to run while `stream` is being
// captured into a CUDA graph: the captured copy would read host memory that is gone when the
// graph is replayed.  Plans and tables are cached, so a call made once before capturing leaves
// nothing to upload inside the capture.
void h2d(void* dst, const void* src, size_t bytes, cudaStream_t stream);

// Byte-exact content cache: returns true when `bytes` equals what was uploaded last time
// under `slot`, so re-uploads of unchanged tables are skipped.
bool same_as_last(std::vector<uint8_t>& slot, const void* data, size_t bytes);

// ----------------------------------------------------------------------------- tuning -------
// Measured choice among `n` launch variants that produce identical results.  The first time `key`
// is seen on a device (and tuning is on and `stream` is not being captured), every variant runs
// once untimed and then 3-9 times timed with CUDA events on `stream` (more while the runs are
// short), and the one with the fastest median is cached; every
// call ends with the chosen variant's results in place.  Later calls with the key run the cached
// choice directly.  Tuning is off with SEQTREE_B200_TUNE=0; then, and while `stream` is being
// captured before the key was tuned, `run(fallback)` runs (`fallback` may be -1, the caller's
// static choice).
int tuned_run(const std::string& key, int n, int fallback, const std::function<void(int)>& run,
              cudaStream_t stream);
// The cached choice for `key` on the current device, or -1.
int tuned_lookup(const std::string& key);
// False when SEQTREE_B200_TUNE=0 switched measured tuning off.
bool tuning_enabled();
// log2 bucket of a size, for shape keys.
inline int size_bucket(int64_t n) {
    int b = 0;
    while (n > 1) {
        n >>= 1;
        ++b;
    }
    return b;
}

// ----------------------------------------------------------------------------- sets ---------
// A sequence set resident on one device: the concatenated (encoded or raw) bytes, offsets and
// lengths, plus host-side length metadata used to plan launches.
}  // namespace stb

struct st_seqset_s {
    int device = 0;
    int32_t alphabet = -1;      // ST_ALPHABET_* or -1 for raw bytes
    int64_t count = 0;
    int64_t total = 0;          // bytes
    int32_t max_len = 0;
    std::vector<int64_t> h_off; // count + 1
    std::vector<int32_t> h_len; // count
    uint8_t* d_bytes = nullptr; // encoded codes (alphabet >= 0) or raw bytes, +64 B padding
    int64_t* d_off = nullptr;
    int32_t* d_len = nullptr;
    bool owns = true;           // false: storage borrowed from the context (transient set)
    uint64_t uid = 0;           // unique per set; plans record the uid they were built for
    // plan caches (opaque; transient sets share the context's)
    std::shared_ptr<void> gb_query_plan, gb_ref_plan, wave_plan;
    ~st_seqset_s();
};

// A thresholded sparse result resident on one device: CSR rows over the query set.
struct st_hits_s {
    int device = 0;
    int64_t rows = 0, cols = 0, nnz = 0;
    uint64_t cap_hint = 0;       // hit-buffer size that the next call starts from
    int64_t block_rows_hint = 0; // query rows per block the last call needed (0: one block)
    stb::DevBuf indptr;          // rows + 1 int64
    stb::DevBuf ref_ids;         // nnz int32, ascending within a row
    stb::DevBuf scores;          // nnz int32
    ~st_hits_s() {
        indptr.release();
        ref_ids.release();
        scores.release();
    }
};

namespace stb {

// Uploads and encodes `s` onto the current device.  When `bad_index` is non-null the first
// invalid symbol's byte index is returned there (or -1) instead of failing, so a caller can
// order errors across two sets exactly as the reference does.
// `storage` (three buffers: bytes, offsets, lengths) makes a transient set that borrows
// context memory instead of allocating.
// `defer_word` >= 0 defers the symbol check: nothing waits for the encode, an invalid symbol is
// stored as code 0 (so every later kernel indexes its tables in range) and the first invalid
// byte index is left in device word `defer_word` of the context's flag area (all ones when
// there is none) for the caller to read after its own final synchronisation.
st_seqset_s* make_seqset(const st_strings* s, int32_t alphabet, cudaStream_t stream,
                         int64_t* bad_index, char* bad_char, DevBuf* storage = nullptr,
                         int defer_word = -1);

int32_t alphabet_size(int32_t alphabet);

// The first `rows` sequences of `s` as a set that borrows its device storage (no copy, no
// allocation; plans go to the context's transient slots).  Valid while `s` lives.
std::unique_ptr<st_seqset_s> row_view(const st_seqset_s& s, int64_t rows);

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace stb
