// Control-calibrated per-query score cutoffs (seqtree python/seqtree/evalue.py:86-143,
// thetas_from_scores / _theta), computed on CSR rows of control hit scores in device memory --
// typically the rows the sparse gap-block kernel just produced.
//
// For one row the cutoff is the largest t in [0, theta_max] with count(score <= t) <= k (the
// reference sorts the row and takes min(theta_max, s[k] - 1); the two agree), or -1 when no t
// qualifies, when k < 1, or when the chosen cutoff admits no control hit while the E-value
// target is below the rule-of-three bound (c_max < 3).  exclude_exact drops score-0 hits first.
// One warp per row: a binary search over t, each probe one coalesced pass over the row.
#include "common.cuh"

namespace stb {

namespace {

__device__ __forceinline__ int64_t warp_count_le(const int32_t* s, int64_t a, int64_t b, int32_t t,
                                                 bool exclude_exact, int lane) {
    int64_t c = 0;
    for (int64_t i = a + lane; i < b; i += 32) {
        const int32_t v = s[i];
        c += (v <= t && !(exclude_exact && v == 0)) ? 1 : 0;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    return c;
}

__global__ void thetas_kernel(const int64_t* __restrict__ indptr, const int32_t* __restrict__ scores,
                              int64_t rows, int32_t k, int rule3, int32_t theta_max,
                              int exclude_exact, int32_t* __restrict__ out) {
    const int64_t row = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= rows) return;
    const int64_t a = indptr[row], b = indptr[row + 1];
    int32_t theta = -1;
    if (k >= 1) {
        if (warp_count_le(scores, a, b, theta_max, exclude_exact, lane) <= k) {
            theta = theta_max;
        } else if (warp_count_le(scores, a, b, 0, exclude_exact, lane) <= k) {
            int32_t lo = 0, hi = theta_max;  // count(lo) <= k < count(hi)
            while (hi - lo > 1) {
                const int32_t mid = lo + (hi - lo) / 2;
                if (warp_count_le(scores, a, b, mid, exclude_exact, lane) <= k) lo = mid;
                else hi = mid;
            }
            theta = lo;
        }
        if (theta >= 0 && rule3 && warp_count_le(scores, a, b, theta, exclude_exact, lane) == 0)
            theta = -1;
    }
    if (lane == 0) out[row] = theta;
}

}  // namespace

void thetas_csr(const int64_t* indptr_d, const int32_t* scores_d, int64_t rows, int32_t k, int rule3,
                int32_t theta_max, int exclude_exact, int32_t* out_d, cudaStream_t stream) {
    if (rows < 0) fail(ST_EINVAL, "seqtree_b200: negative row count");
    if (theta_max < 0) fail(ST_EINVAL, "theta_max must be >= 0");
    if (rows == 0) return;
    if (!indptr_d || !out_d) fail(ST_EINVAL, "seqtree_b200: null CSR input or output");
    const int64_t threads = rows * 32;
    thetas_kernel<<<unsigned(ceil_div(threads, 256)), 256, 0, stream>>>(
        indptr_d, scores_d, rows, k, rule3, theta_max, exclude_exact, out_d);
    STB_CUDA(cudaGetLastError());
    note_launch("thetas_kernel");
}

}  // namespace stb
