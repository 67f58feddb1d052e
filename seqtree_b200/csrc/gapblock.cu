// Dense single-gap-block penalty matrix on sm_100a.
//
// Reference arithmetic (seqtree src/gapblock.cpp:39-62): for a pair (q, r) with L = min(m,n),
// d = |m-n|, the layout whose block opens at column i of the shorter sequence costs
//     pre[i] + suf[i] + prior[i]     (prefix on diagonal 0, suffix on diagonal d)
// and the score is the minimum over i in [0, L] plus gap_open + (d-1)*gap_extend; at d == 0
// it is the plain substitution sum.  With P0[j] = pen on diagonal 0 and Pd[j] = pen on
// diagonal d, pre[i] + suf[i] = S + C[i] where S = sum_j Pd[j] and C[i] = sum_{j<i}(P0 - Pd),
// so one forward sweep visits every block position -- that is the form computed here.  The
// result is the same integer as the reference's (integer sums, no reassociation hazard while
// the reference itself does not overflow int32).
//
// Fast path (every length <= 64, min(m,n) <= 32, L*max_pen <= 8191):
//   * Queries are sorted by length and paired; the penalties of a pair against one ref residue
//     travel as int16x2.  A query profile QP[pair][j][b] = pen(q1[j], b) | pen(q2[j], b) << 16
//     (32 words per row: one pass over the banks) is built once per call in global memory.
//   * Refs are cut into chunks of RC columns (original order); inside a chunk they are grouped
//     by length into warp tasks of <= 32 refs, so d, L and the prior row are warp-uniform.  The
//     refs' codes are laid out per task as [j][lane] bytes holding 4*code (a byte offset into a
//     profile row), also once per call.
//   * A CTA owns (chunk, 4 query pairs).  Two bulk (TMA) copies stage its 4-pair profile slab
//     and the chunk's code slab into shared memory, completing on one mbarrier.  A warp unit is
//     (task, slice of 4 pairs of one length); the 4 pairs are swept together, and every lookup
//     is LDS [lane register + compile-time immediate]: the register is the residue's byte offset
//     and the immediate ((slice*4 + pair)*LQ + j)*128.  Both penalties of two pairs arrive in
//     one LDS, the running sums are plain 32-bit adds on halves kept in [0, 2^15), and one DPX
//     __viaddmin_s16x2 updates both running minima.
//   * Results go through a shared tile so that global stores are coalesced 16-byte vectors in
//     the original column order; the per-(m,n) term (prior minimum + gap cost) is added there.
// General path: one thread per pair in int32 for any lengths and penalty magnitudes.
//
// Thresholded sparse form (for matrices too large to hold densely): the same kernels keep only
// the cells with score <= max_penalty.  Hits are appended as (query << shift | ref, score) with one
// atomic per warp, then radix-sorted by key and turned into CSR rows (indptr, ref ids, scores):
// exactly the entries of the dense matrix's rows that pass the threshold, in ref order.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <numeric>
#include <type_traits>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "sparse.cuh"

namespace stb {

namespace {

constexpr int kGP = 4;          // query pairs per CTA (tile rows = 8 queries; 8 pairs measured slower)
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRow = 32;        // words per profile row
constexpr int kPairsPerSlice = 4;
static_assert(kWarps == 2 * kGP, "the ordered sparse epilogue gives each tile row one warp");

// ---------------------------------------------------------------------------- plans ---------
// Plans depend only on the lengths (and codes) of a set, so a device-resident set builds them
// once; transient sets (host-buffer calls) rebuild them in place inside the context's plan
// objects, whose device buffers only grow.
struct QueryPlan {
    uint64_t uid = 0;                    // set the plan was built for
    int64_t r0 = 0, r1 = -1;             // its rows [r0, r1) (r1 = -1: the whole set)
    int64_t P = 0;                       // query pairs, a multiple of 4
    std::vector<int2> pairs;             // original indices (-1 marks an empty slot)
    std::vector<int32_t> plen;           // m of each pair
    DevBuf d_pairs, d_plen;
    std::vector<uint8_t> prof_key;       // (A, LQ, penalty grid) the profile was built for
    DevBuf d_prof;                       // [P][LQ][32] uint32
};

struct RefPlan {
    uint64_t uid = 0;
    int rc = 0;                          // columns per chunk
    int64_t nchunks = 0;
    int64_t ntasks = 0;
    int64_t max_slab = 0;                // largest per-chunk code slab (bytes)
    int max_tasks = 0;                   // most warp tasks in one chunk
    int64_t slab_bytes = 0;              // whole slab
    std::vector<int32_t> sorted;
    std::vector<int4> tasks;             // (n, start in sorted, count <= 32, slab byte offset)
    std::vector<int32_t> task_off;       // nchunks + 1
    DevBuf d_sorted, d_tasks, d_task_off;
    DevBuf d_slab;                       // per task: n rows of 32 bytes (4*code per lane)
};

// Queries (rows [r0, r1) of the set; r1 = -1 for all) sorted by length (stable) and paired
// within each length; an odd one out is paired with -1.  Each length's pairs are padded with
// (-1, -1) to a multiple of 4, so that every slice of 4 consecutive pairs has one length.  Empty
// slots are computed and never stored.
void build_query_plan(QueryPlan& plan, const st_seqset_s& q, cudaStream_t stream, int64_t r0 = 0,
                      int64_t r1 = -1) {
    const int64_t N = (r1 < 0 ? q.count : r1) - r0;
    std::vector<int32_t> order(static_cast<size_t>(N));
    std::iota(order.begin(), order.end(), int32_t(r0));
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return q.h_len[size_t(a)] < q.h_len[size_t(b)]; });
    plan.pairs.clear();
    plan.plen.clear();
    for (int64_t i = 0; i < N;) {
        const int32_t m = q.h_len[size_t(order[size_t(i)])];
        int64_t e = i;
        while (e < N && q.h_len[size_t(order[size_t(e)])] == m) ++e;
        const size_t first = plan.pairs.size();
        for (int64_t t = i; t < e; t += 2)
            plan.pairs.push_back(make_int2(order[size_t(t)], t + 1 < e ? order[size_t(t + 1)] : -1));
        while ((plan.pairs.size() - first) % kPairsPerSlice) plan.pairs.push_back(make_int2(-1, -1));
        plan.plen.resize(plan.pairs.size(), m);
        i = e;
    }
    plan.P = int64_t(plan.pairs.size());
    h2d(plan.d_pairs.as<int2>(size_t(plan.P)), plan.pairs.data(),
                             sizeof(int2) * size_t(plan.P), stream);
    h2d(plan.d_plen.as<int32_t>(size_t(plan.P)), plan.plen.data(),
                             sizeof(int32_t) * size_t(plan.P), stream);
    plan.prof_key.clear();
    plan.uid = q.uid;
    plan.r0 = r0;
    plan.r1 = r1;
}

// Refs in chunks of rc columns (original order); inside a chunk a counting sort by length
// yields warp tasks of <= 32 refs of one length.  Each task's code rows occupy n*32 bytes of
// the slab, so a chunk's slab is one contiguous range.
void build_ref_plan(RefPlan& plan, const st_seqset_s& r, int rc, cudaStream_t stream,
                    bool upload = true) {
    const int64_t K = r.count;
    plan.rc = rc;
    plan.nchunks = ceil_div(K, rc);
    plan.sorted.resize(size_t(K));
    plan.tasks.clear();
    plan.task_off.assign(size_t(plan.nchunks + 1), 0);
    plan.max_slab = 0;
    plan.max_tasks = 0;
    std::vector<int32_t> cnt(size_t(r.max_len) + 2);
    std::vector<int32_t> start(cnt.size());
    int64_t slab = 0;
    for (int64_t c = 0; c < plan.nchunks; ++c) {
        const int64_t k0 = c * rc, k1 = std::min<int64_t>(K, k0 + rc);
        std::fill(cnt.begin(), cnt.end(), 0);
        for (int64_t k = k0; k < k1; ++k) cnt[size_t(r.h_len[size_t(k)]) + 1]++;
        for (size_t l = 1; l < cnt.size(); ++l) cnt[l] += cnt[l - 1];
        std::copy(cnt.begin(), cnt.end(), start.begin());
        for (int64_t k = k0; k < k1; ++k)
            plan.sorted[size_t(k0 + start[size_t(r.h_len[size_t(k)])]++)] = int32_t(k);
        const int64_t slab0 = slab;
        for (int32_t l = 0; l <= r.max_len; ++l) {
            const int32_t b = cnt[size_t(l)], e = cnt[size_t(l) + 1];
            for (int32_t s = b; s < e; s += 32) {
                plan.tasks.push_back(make_int4(l, int32_t(k0) + s, std::min(32, e - s), int32_t(slab)));
                slab += int64_t(l) * 32;
            }
        }
        plan.max_slab = std::max(plan.max_slab, slab - slab0);
        plan.max_tasks = std::max(plan.max_tasks, int(plan.tasks.size()) - plan.task_off[size_t(c)]);
        plan.task_off[size_t(c + 1)] = int32_t(plan.tasks.size());
    }
    if (slab > INT32_MAX) fail(ST_EINVAL, "seqtree_b200: reference set too large for one call");
    plan.ntasks = int64_t(plan.tasks.size());
    plan.slab_bytes = slab;
    if (!upload) return;
    h2d(plan.d_sorted.as<int32_t>(size_t(K)), plan.sorted.data(),
                             sizeof(int32_t) * size_t(K), stream);
    h2d(plan.d_tasks.as<int4>(plan.tasks.size()), plan.tasks.data(),
                             sizeof(int4) * plan.tasks.size(), stream);
    h2d(plan.d_task_off.as<int32_t>(plan.task_off.size()),
                             plan.task_off.data(), sizeof(int32_t) * plan.task_off.size(), stream);
    plan.d_slab.as<uint8_t>(size_t(slab) + 16);
    plan.uid = r.uid;
}

template <class Plan>
Plan& plan_slot(std::shared_ptr<void>& own, std::shared_ptr<void>& shared, bool owns) {
    std::shared_ptr<void>& slot = owns ? own : shared;
    if (!slot) slot = std::make_shared<Plan>();
    return *static_cast<Plan*>(slot.get());
}

// QP[p][j][b] for b < 32 (zero beyond A, beyond the pair's length and for empty slots).
__global__ void profile_kernel(const uint8_t* __restrict__ codes, const int64_t* __restrict__ off,
                               const int2* __restrict__ pairs, const int32_t* __restrict__ plen,
                               const int32_t* __restrict__ pen, int A, int LQ, int64_t total,
                               uint32_t* __restrict__ prof) {
    const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int64_t p = idx / (int64_t(LQ) * kRow);
    const int j = int((idx / kRow) % LQ);
    const int b = int(idx % kRow);
    const int2 pr = pairs[p];
    uint32_t v = 0;
    if (b < A && j < plen[p] && pr.x >= 0) {
        const int c1 = codes[off[pr.x] + j];
        const int c2 = codes[off[pr.y >= 0 ? pr.y : pr.x] + j];
        v = uint32_t(pen[c1 * A + b]) | (uint32_t(pen[c2 * A + b]) << 16);
    }
    prof[idx] = v;
}

// Per task: n rows of 32 lane bytes, each 4*code (lanes past the task's count repeat lane 0).
__global__ void ref_slab_kernel(const uint8_t* __restrict__ codes, const int64_t* __restrict__ off,
                                const int32_t* __restrict__ sorted, const int4* __restrict__ tasks,
                                uint8_t* __restrict__ slab) {
    const int4 t = tasks[blockIdx.x];
    for (int idx = threadIdx.x; idx < t.x * 32; idx += blockDim.x) {
        const int j = idx >> 5, l = idx & 31;
        const int k = sorted[t.y + (l < t.z ? l : 0)];
        slab[int64_t(t.w) + idx] = uint8_t(codes[off[k] + j] * 4);
    }
}

// ---------------------------------------------------------------------------- fast kernel ---
struct FastArgs {
    const uint32_t* prof;    // [P][LQ][32]
    const uint8_t* slab;     // ref code slab
    const int32_t* rlen;
    int64_t K;
    int rc;                  // columns per chunk
    const int2* pairs;       // (q1, q2); -1 marks an empty slot
    const int32_t* plen;
    int64_t P;
    const int32_t* ref_sorted;
    const int4* tasks;
    const int32_t* task_off;
    int slab_cap;            // shared bytes reserved for a chunk's slab
    int max_tasks;           // shared task slots (the most tasks of one chunk)
    const uint32_t* prior2;  // rows (M*W1 + d) of pstride words, value i at i + 3; or null
    int pstride;
    const int32_t* ftab;     // [m*W1 + n]: per-(m,n) additive term (prior minimum + gap cost)
    int W1;
    uint32_t bias2;          // BIAS in both halves
    int32_t* out;            // dense output (unused by the sparse form)
    unsigned long long* err; // set when the bounded wait for the staging copies gives up
    SparseSink sink;         // sparse output (unused by the dense form)
    // Persistent form: a grid of about one wave of CTAs takes tiles (chunk, pair group) from a
    // global counter, longest query pairs first (the pairs are sorted by length), so the
    // expensive tiles start early and the wave drains evenly.  0: one CTA per tile.
    int persistent;
    int nchunks;
    int ntiles;
    unsigned int* queue;     // zeroed before every launch
};

// One non-blocking probe of an mbarrier phase (callers bound the number of probes).
__device__ __forceinline__ uint32_t mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

// One warp unit: the 4 pairs of one slice of the CTA against the 32 refs of one task.  The
// sweep reads each residue offset straight from the staged code slab; the slice base and the
// row offset j*128 are folded into two per-position addresses, so the 8 lookups of a position
// are LDS [address + compile-time immediate (pair * LQ * 128)].  Query-longer pairs shift the
// diagonal-d address by d rows; ref-longer pairs read the residue d positions further on.
template <int LQ, bool PRIOR>
__device__ __forceinline__ void run_unit(const FastArgs& a, const uint8_t* smem,
                                         const uint8_t* s_codes, uint32_t* s_tile,
                                         const int32_t* s_plen, const int16_t* s_col, int slice,
                                         const int4 task, int tb, int64_t k0, int lane) {
    constexpr int kRowB = kRow * 4;
    constexpr int kPairB = LQ * kRowB;
    const int n = task.x;
    const int m = s_plen[slice * kPairsPerSlice];
    const int L = min(m, n);
    const int d = abs(m - n);
    const int dq = m > n ? d : 0;   // query longer: diagonal d is d profile rows further down
    const int dr = n > m ? d : 0;   // ref longer: diagonal d reads residue j + d
    const uint8_t* rows0 = s_codes + tb + lane;
    const uint8_t* rowsd = rows0 + dr * 32;
    const uint32_t base0 = uint32_t(slice * kPairsPerSlice * kPairB);
    const uint32_t based = base0 + uint32_t(dq * kRowB);
    uint32_t res[kPairsPerSlice];
    if (d == 0) {
        uint32_t S[kPairsPerSlice] = {0u, 0u, 0u, 0u};
#pragma unroll 4
        for (int j = 0; j < L; ++j) {
            const uint32_t a0 = base0 + uint32_t(j * kRowB) + rows0[j * 32];
#pragma unroll
            for (int q = 0; q < kPairsPerSlice; ++q)
                S[q] += *reinterpret_cast<const uint32_t*>(smem + a0 + q * kPairB);
        }
#pragma unroll
        for (int q = 0; q < kPairsPerSlice; ++q) res[q] = S[q];
    } else {
        // Prior row of (max(m,n), d): value i at prow[i + 3], so values j+1..j+4 of an aligned
        // group of four positions are one 16-byte load.
        const uint32_t* prow = PRIOR ? a.prior2 + (size_t(max(m, n)) * a.W1 + d) * a.pstride : nullptr;
        uint32_t S[kPairsPerSlice], Cb[kPairsPerSlice], best[kPairsPerSlice];
        const uint32_t first = PRIOR ? a.bias2 + __ldg(prow + 3) : a.bias2;
#pragma unroll
        for (int q = 0; q < kPairsPerSlice; ++q) {
            S[q] = 0u;
            Cb[q] = a.bias2;
            best[q] = first;
        }
        // The sweep, in two versions: when the query is the longer one (dr == 0) both diagonals
        // read residue j of the ref, so one byte load serves both addresses.
        auto sweep = [&](auto same_residue) {
            constexpr bool kSame = decltype(same_residue)::value;
            auto step = [&](int j, uint32_t pr) {
                const uint32_t c0 = rows0[j * 32];
                const uint32_t a0 = base0 + uint32_t(j * kRowB) + c0;
                const uint32_t ad = based + uint32_t(j * kRowB) + (kSame ? c0 : uint32_t(rowsd[j * 32]));
#pragma unroll
                for (int q = 0; q < kPairsPerSlice; ++q) {
                    const uint32_t p0v = *reinterpret_cast<const uint32_t*>(smem + a0 + q * kPairB);
                    const uint32_t pdv = *reinterpret_cast<const uint32_t*>(smem + ad + q * kPairB);
                    S[q] += pdv;
                    Cb[q] = Cb[q] + p0v - pdv;  // per-half exact: halves stay in [0, 2^15)
                    best[q] = __viaddmin_s16x2(Cb[q], pr, best[q]);
                }
            };
            // The prior values of the next group of four positions are requested one group
            // ahead, so their load latency hides behind the current group's lookups.
            int j = 0;
            uint4 pnext = make_uint4(0u, 0u, 0u, 0u);
            if constexpr (PRIOR)
                if (L >= 4) pnext = __ldg(reinterpret_cast<const uint4*>(prow + 4));
            for (; j + 4 <= L; j += 4) {
                const uint4 pv = pnext;
                if constexpr (PRIOR)
                    if (j + 8 <= L) pnext = __ldg(reinterpret_cast<const uint4*>(prow + j + 8));
                step(j, pv.x);
                step(j + 1, pv.y);
                step(j + 2, pv.z);
                step(j + 3, pv.w);
            }
            for (; j < L; ++j) step(j, PRIOR ? __ldg(prow + j + 4) : 0u);
        };
        if (dr == 0)
            sweep(std::true_type{});
        else
            sweep(std::false_type{});
#pragma unroll
        for (int q = 0; q < kPairsPerSlice; ++q) res[q] = S[q] + best[q] - a.bias2;
    }
    if (lane < task.z) {
        const int col = s_col[int(task.y - k0) + lane];
#pragma unroll
        for (int q = 0; q < kPairsPerSlice; ++q)
            s_tile[(slice * kPairsPerSlice + q) * a.rc + col] = res[q];
    }
}

template <int LQ, bool PRIOR, bool SPARSE>
__global__ void __launch_bounds__(kThreads, 3) gapblock_fast_kernel(const FastArgs a) {
    extern __shared__ __align__(128) uint8_t smem[];
    constexpr int kProfB = kGP * LQ * kRow * 4;
    const int prof_area = kProfB > (kGP / kPairsPerSlice) * a.rc * 4 ? kProfB
                                                                    : (kGP / kPairsPerSlice) * a.rc * 4;
    uint8_t* s_codes = smem + prof_area;
    uint32_t* s_tile = reinterpret_cast<uint32_t*>(s_codes + a.slab_cap);
    int32_t* s_ftab = reinterpret_cast<int32_t*>(s_tile + kGP * a.rc);
    uint8_t* s_len = reinterpret_cast<uint8_t*>(s_ftab + ((a.W1 * a.W1 + 3) & ~3));
    int4* s_task = reinterpret_cast<int4*>(s_len + ((a.rc + 15) & ~15));
    int16_t* s_col = reinterpret_cast<int16_t*>(s_task + a.max_tasks);
    int32_t* s_plen = reinterpret_cast<int32_t*>(s_col + ((a.rc + 7) & ~7));
    uint64_t* s_bar = reinterpret_cast<uint64_t*>(s_plen + kGP);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    volatile int* s_next = reinterpret_cast<volatile int*>(s_bar + 1);  // in the barrier's 16 bytes
    const uint32_t bar = uint32_t(__cvta_generic_to_shared(s_bar));
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
    const int npg = int((a.P + kGP - 1) / kGP);
    for (int iter = 0;; ++iter) {
    int chunk, pg;
    if (a.persistent) {
        if (tid == 0) *s_next = int(atomicAdd(a.queue, 1u));
        __syncthreads();
        const int t = *s_next;
        if (t >= a.ntiles) break;
        pg = npg - 1 - t / a.nchunks;
        chunk = t - (t / a.nchunks) * a.nchunks;
    } else {
        if (iter > 0) break;
        chunk = blockIdx.x;
        pg = int(blockIdx.y + blockIdx.z * gridDim.y);  // pair groups past 65,535 use z
        if (pg >= npg) break;
    }
    const uint32_t parity = uint32_t(iter & 1);
    const int64_t k0 = int64_t(chunk) * a.rc;
    const int kcount = int(a.K - k0 < a.rc ? a.K - k0 : a.rc);
    const int p0 = pg * kGP;
    const int np = int(a.P - p0 < kGP ? a.P - p0 : kGP);
    const int t0 = a.task_off[chunk], t1 = a.task_off[chunk + 1];
    const int tw0 = a.tasks[t0].w;
    const int slab_bytes = (t1 > t0 ? a.tasks[t1 - 1].w + a.tasks[t1 - 1].x * 32 : tw0) - tw0;

    // Stage the CTA's profile slab and the chunk's code slab with two bulk (TMA) copies that
    // complete on one mbarrier, while the other threads load the (m, n) terms and lengths.
    // (In the persistent form every tile is one phase of the barrier; the previous tile's
    // generic-proxy writes to the same shared memory are ordered before these copies by the
    // barrier that ended it and the proxy fence.)
    if (tid == 0) {
        const uint32_t prof_bytes = uint32_t(np) * LQ * kRow * 4;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(prof_bytes + uint32_t(slab_bytes))
                     : "memory");
        bulk_g2s(uint32_t(__cvta_generic_to_shared(smem)),
                 a.prof + size_t(p0) * LQ * kRow, prof_bytes, bar);
        if (slab_bytes > 0)
            bulk_g2s(uint32_t(__cvta_generic_to_shared(s_codes)), a.slab + tw0,
                     uint32_t(slab_bytes), bar);
    }
    // Per-tile metadata in shared memory, so that a warp unit starts without a chain of global
    // loads: the chunk's tasks, each sorted slot's column, the pairs' query lengths.
    for (int i = tid; i < a.W1 * a.W1; i += kThreads) s_ftab[i] = a.ftab[i];
    for (int c = tid; c < kcount; c += kThreads) {
        s_len[c] = uint8_t(a.rlen[k0 + c]);
        s_col[c] = int16_t(a.ref_sorted[k0 + c] - k0);
    }
    for (int i = tid; i < t1 - t0; i += kThreads) s_task[i] = a.tasks[t0 + i];
    if (tid < np) s_plen[tid] = a.plen[p0 + tid];
    __syncthreads();
    {
        // Bounded wait on phase 0 by every thread.  If any thread runs out, the CTA records
        // the failure, waits once more (bounded) for its copies in flight, and leaves as a
        // whole -- the host then reports ST_ETIMEOUT and no tile is stored.
        uint32_t done = 0;
        for (int it = 0; it < (1 << 20) && !done; ++it) done = mbar_try_wait(bar, parity);
        if (__syncthreads_or(!done)) {
            if (tid == 0) atomicExch(a.err, 1ull);
            for (int it = 0; it < (1 << 20) && !done; ++it) done = mbar_try_wait(bar, parity);
            __syncthreads();
            return;
        }
    }

    const int nslices = np / kPairsPerSlice;
    const int units = (t1 - t0) * nslices;
    for (int u = warp; u < units; u += kWarps) {
        const int ti = u / nslices;
        const int4 task = s_task[ti];
        const int tb = task.w - tw0;
        run_unit<LQ, PRIOR>(a, smem, s_codes, s_tile, s_plen, s_col, u - ti * nslices, task, tb,
                            k0, lane);
    }
    __syncthreads();

    // Per-slice column terms fcol[slice][c] = ftab[m_slice][len(c)], written over the profile
    // (no longer read), then the coalesced write-out: each thread takes one pair and four
    // columns, reads the packed tile and the terms once and stores both queries' rows as
    // 16-byte vectors.
    int32_t* s_fcol = reinterpret_cast<int32_t*>(smem);
    for (int i = tid; i < nslices * a.rc; i += kThreads) {
        const int sl = i / a.rc, c = i - sl * a.rc;
        s_fcol[i] = c < kcount ? s_ftab[s_plen[sl * kPairsPerSlice] * a.W1 + s_len[c]] : 0;
    }
    __syncthreads();
    const int cols4 = (kcount + 3) >> 2;
    if (SPARSE && a.sink.ordered) {
        // Ordered form: warp w owns tile row (pair w / 2, half w % 2).  It counts its hits, the
        // CTA reserves one segment for all of them, and the warp writes its row's hits there in
        // ascending column order, recording the piece (row, chunk) it wrote.
        __shared__ unsigned long long s_rowcnt[kWarps + 1];  // row counts, then the base
        __shared__ int s_fits;
        const unsigned full = 0xffffffffu;
        const int pl = warp >> 1, hf = warp & 1;
        int qrow = -1;
        if (pl < np) {
            const int2 pr = a.pairs[p0 + pl];
            qrow = hf ? pr.y : pr.x;
        }
        const uint32_t* src = s_tile + pl * a.rc;
        const int32_t* fc = s_fcol + (pl / kPairsPerSlice) * a.rc;
        // Lane l takes columns 4l..4l+3 of each 128-column group (16-byte loads of the packed
        // tile and of the column terms); bit u of the result marks a hit in column 4l + u.
        auto group = [&](int g, int32_t (&v)[4]) {
            const int c = g * 128 + lane * 4;
            uint32_t hits = 0;
            if (c < kcount) {
                const uint4 t = *reinterpret_cast<const uint4*>(src + c);
                const int4 f = *reinterpret_cast<const int4*>(fc + c);
                const uint32_t tw[4] = {t.x, t.y, t.z, t.w};
                const int32_t fw[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    v[u] = int32_t((hf ? (tw[u] >> 16) : (tw[u] & 0xFFFFu)) + uint32_t(fw[u]));
                    if (c + u < kcount && v[u] <= a.sink.thresh) hits |= 1u << u;
                }
            }
            return hits;
        };
        const int groups = (kcount + 127) >> 7;
        int n = 0;
        if (qrow >= 0)
            for (int g = 0; g < groups; ++g) {
                int32_t v[4];
                n += __popc(group(g, v));
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(full, n, o);
        if (lane == 0) s_rowcnt[warp] = (unsigned long long)n;
        __syncthreads();
        if (tid == 0) {
            unsigned long long tot = 0;
            for (int w = 0; w < kWarps; ++w) tot += s_rowcnt[w];
            const unsigned long long base = tot ? atomicAdd(a.sink.count, tot) : 0ull;
            s_rowcnt[kWarps] = base;
            s_fits = base + tot <= a.sink.cap ? 1 : 0;  // else counted only; the host re-runs
        }
        __syncthreads();
        if (qrow >= 0) {
            unsigned long long off = s_rowcnt[kWarps];
            for (int w = 0; w < warp; ++w) off += s_rowcnt[w];
            const int64_t piece = (int64_t(qrow) - a.sink.row0) * a.sink.nchunks + chunk;
            if (lane == 0) {
                a.sink.piece_off[piece] = int64_t(off);
                a.sink.piece_cnt[piece] = n;
            }
            if (s_fits && n > 0) {
                for (int g = 0; g < groups; ++g) {
                    int32_t v[4];
                    uint32_t hits = group(g, v);
                    const int cnt = __popc(hits);
                    int incl = cnt;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int t = __shfl_up_sync(full, incl, o);
                        if (lane >= o) incl += t;
                    }
                    unsigned long long pos = off + (unsigned long long)(incl - cnt);
                    const int c = g * 128 + lane * 4;
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (hits & (1u << u)) a.sink.seg[pos++] = make_int2(int(k0 + c + u), v[u]);
                    off += (unsigned long long)__shfl_sync(full, incl, 31);
                }
            }
        }
    } else if constexpr (SPARSE) {
        // Every lane runs the same number of rounds (sink_append is warp-collective).
        const int total = np * cols4;
        for (int i0 = 0; i0 < total; i0 += kThreads) {
            const int i = i0 + tid;
            uint32_t hits = 0;
            int pl = 0, c = 0;
            int2 pr = make_int2(-1, -1);
            if (i < total) {
                pl = i / cols4;
                c = (i - pl * cols4) * 4;
                pr = a.pairs[p0 + pl];
            }
            const uint32_t* src = s_tile + pl * a.rc + c;
            const int32_t* fc = s_fcol + (pl / kPairsPerSlice) * a.rc + c;
            if (pr.x >= 0) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (c + u >= kcount) break;
                    const uint32_t t = src[u];
                    const uint32_t f = uint32_t(fc[u]);
                    if (int32_t((t & 0xFFFFu) + f) <= a.sink.thresh) hits |= 1u << u;
                    if (pr.y >= 0 && int32_t((t >> 16) + f) <= a.sink.thresh) hits |= 16u << u;
                }
            }
            sink_append(a.sink, hits, lane, [&](int b, unsigned long long& key, int32_t& val) {
                const int u = b & 3;
                const uint32_t t = src[u];
                val = int32_t((b < 4 ? (t & 0xFFFFu) : (t >> 16)) + uint32_t(fc[u]));
                key = sink_key(a.sink, b < 4 ? pr.x : pr.y, k0 + c + u);
            });
        }
    } else {
    const bool vec = (a.K & 3) == 0;
    for (int i = tid; i < np * cols4; i += kThreads) {
        const int pl = i / cols4;
        const int c = (i - pl * cols4) * 4;
        const int2 pr = a.pairs[p0 + pl];
        if (pr.x < 0) continue;
        const uint32_t* src = s_tile + pl * a.rc + c;
        const int32_t* fc = s_fcol + (pl / kPairsPerSlice) * a.rc + c;
        int32_t* d1 = a.out + int64_t(pr.x) * a.K + k0 + c;
        int32_t* d2 = pr.y >= 0 ? a.out + int64_t(pr.y) * a.K + k0 + c : nullptr;
        if (vec && c + 4 <= kcount) {
            const uint4 t = *reinterpret_cast<const uint4*>(src);
            const int4 f = *reinterpret_cast<const int4*>(fc);
            *reinterpret_cast<int4*>(d1) =
                make_int4(int32_t((t.x & 0xFFFFu) + uint32_t(f.x)), int32_t((t.y & 0xFFFFu) + uint32_t(f.y)),
                          int32_t((t.z & 0xFFFFu) + uint32_t(f.z)), int32_t((t.w & 0xFFFFu) + uint32_t(f.w)));
            if (d2)
                *reinterpret_cast<int4*>(d2) =
                    make_int4(int32_t((t.x >> 16) + uint32_t(f.x)), int32_t((t.y >> 16) + uint32_t(f.y)),
                              int32_t((t.z >> 16) + uint32_t(f.z)), int32_t((t.w >> 16) + uint32_t(f.w)));
        } else {
            for (int u = 0; u < 4 && c + u < kcount; ++u) {
                d1[u] = int32_t((src[u] & 0xFFFFu) + uint32_t(fc[u]));
                if (d2) d2[u] = int32_t((src[u] >> 16) + uint32_t(fc[u]));
            }
        }
    }
    }
    __syncthreads();  // this tile's shared memory is free for the next one
    }
}

// ---------------------------------------------------------------------------- general -------
struct GeneralArgs {
    const uint8_t* qcodes;
    const int64_t* qoff;
    const uint8_t* rcodes;
    const int64_t* roff;
    int64_t row0;         // first query row (row blocks of the sparse form)
    int64_t N, K;         // rows in this launch, refs
    const int32_t* pen;   // A*A
    int A;
    int32_t go, ge;
    const int32_t* prior; // (pw+1)^3 or null
    int64_t pw1;
    int32_t* out;         // dense output (unused by the sparse form)
    SparseSink sink;      // sparse output (unused by the dense form)
};

// The gap-block score of one pair in int32 arithmetic with the reference's wrap
// (src/gapblock.cpp:39-62, in the single-sweep form S + min_i(C_i + p_i)).
// Score of one pair; with `pos`, also the block position of the minimum (the smallest such
// position; 0 when the lengths are equal), counted in residues of the shorter sequence.
__device__ __forceinline__ int32_t gapblock_cell(const uint8_t* q, int m, const uint8_t* r, int n,
                                                 const int32_t* s_pen, int A, int32_t go, int32_t ge,
                                                 const int32_t* prior, int64_t pw1,
                                                 int32_t* pos = nullptr) {
    const int L = min(m, n), d = abs(m - n);
    if (pos) *pos = 0;
    if (d == 0) {
        uint32_t s = 0;
        for (int j = 0; j < L; ++j) s += uint32_t(s_pen[q[j] * A + r[j]]);
        return int32_t(s);
    }
    const bool ql = m > n;
    const int32_t* prow = prior ? prior + (int64_t(max(m, n)) * pw1 + d) * pw1 : nullptr;
    int32_t S = 0, C = 0;
    int32_t best = prow ? prow[0] : 0;
    int32_t at = 0;
    for (int j = 0; j < L; ++j) {
        const int32_t p0v = s_pen[q[j] * A + r[j]];
        const int32_t pdv = ql ? s_pen[q[j + d] * A + r[j]] : s_pen[q[j] * A + r[j + d]];
        S += pdv;
        C += p0v - pdv;
        const int32_t cand = C + (prow ? prow[j + 1] : 0);
        if (cand < best) {
            best = cand;
            at = j + 1;
        }
    }
    if (pos) *pos = at;
    return int32_t(uint32_t(S) + uint32_t(best) + uint32_t(go) + uint32_t(d - 1) * uint32_t(ge));
}

// One thread per listed pair (qi[p], ri[p]); out[p] = its score.
__global__ void __launch_bounds__(256) gapblock_pairs_kernel(
    const uint8_t* __restrict__ qcodes, const int64_t* __restrict__ qoff,
    const uint8_t* __restrict__ rcodes, const int64_t* __restrict__ roff,
    const int32_t* __restrict__ qi, const int32_t* __restrict__ ri, int64_t n,
    const int32_t* __restrict__ pen, int A, int32_t go, int32_t ge,
    const int32_t* __restrict__ prior, int64_t pw1, int32_t* __restrict__ out,
    int32_t* __restrict__ pos_out) {
    extern __shared__ int32_t s_pen[];
    for (int i = threadIdx.x; i < A * A; i += blockDim.x) s_pen[i] = pen[i];
    __syncthreads();
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = qi[p], k = ri[p];
        const int m = int(qoff[i + 1] - qoff[i]), nn = int(roff[k + 1] - roff[k]);
        int32_t at = 0;
        out[p] = gapblock_cell(qcodes + qoff[i], m, rcodes + roff[k], nn, s_pen, A, go, ge, prior,
                               pw1, pos_out ? &at : nullptr);
        if (pos_out) pos_out[p] = at;
    }
}

// One thread per (i, k) in row-major order, int32 arithmetic with the reference's wrap.  The
// loop runs the same number of rounds on every lane (the sparse append is warp-collective).
template <bool SPARSE>
__global__ void __launch_bounds__(256) gapblock_general_kernel(const GeneralArgs a) {
    extern __shared__ int32_t s_pen[];
    for (int i = threadIdx.x; i < a.A * a.A; i += blockDim.x) s_pen[i] = a.pen[i];
    __syncthreads();
    const int64_t total = a.N * a.K;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < total;
         base += int64_t(gridDim.x) * blockDim.x) {
        const int64_t idx = base + threadIdx.x;
        if (!SPARSE && idx >= total) break;
        const bool live = idx < total;
        const int64_t il = live ? idx / a.K : 0, k = live ? idx - il * a.K : 0;
        const int64_t i = a.row0 + il;
        const int m = int(a.qoff[i + 1] - a.qoff[i]);
        const int n = int(a.roff[k + 1] - a.roff[k]);
        const int32_t v = gapblock_cell(a.qcodes + a.qoff[i], m, a.rcodes + a.roff[k], n, s_pen,
                                        a.A, a.go, a.ge, a.prior, a.pw1);
        if constexpr (SPARSE) {
            sink_append(a.sink, live && v <= a.sink.thresh ? 1u : 0u, int(threadIdx.x & 31),
                        [&](int, unsigned long long& key, int32_t& val) {
                            key = sink_key(a.sink, i, k);
                            val = v;
                        });
        } else {
            a.out[idx] = v;
        }
    }
}

template <int LQ, bool PRIOR>
const char* launch_fast(const FastArgs& args, dim3 grid, size_t smem, cudaStream_t stream) {
    const bool sparse = args.sink.keys != nullptr || args.sink.ordered;  // either sparse form
    auto kern = sparse ? gapblock_fast_kernel<LQ, PRIOR, true>
                       : gapblock_fast_kernel<LQ, PRIOR, false>;
    STB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    kern<<<grid, kThreads, smem, stream>>>(args);
    STB_CUDA(cudaGetLastError());
    return sparse ? "gapblock_fast_kernel<sparse>" : "gapblock_fast_kernel";
}

// Profile height LQ >= longest query: rows per pair in shared memory.
int profile_height(int longest_query) {
    for (int h : {16, 24, 32, 48})
        if (longest_query <= h) return h;
    return 64;
}

template <int LQ>
const char* dispatch_prior(bool prior, const FastArgs& args, dim3 grid, size_t smem,
                           cudaStream_t stream) {
    return prior ? launch_fast<LQ, true>(args, grid, smem, stream)
                 : launch_fast<LQ, false>(args, grid, smem, stream);
}

const char* dispatch_fast(int lq, bool prior, const FastArgs& args, dim3 grid, size_t smem,
                          cudaStream_t stream) {
    switch (lq) {
        case 16: return dispatch_prior<16>(prior, args, grid, smem, stream);
        case 24: return dispatch_prior<24>(prior, args, grid, smem, stream);
        case 32: return dispatch_prior<32>(prior, args, grid, smem, stream);
        case 48: return dispatch_prior<48>(prior, args, grid, smem, stream);
        default: return dispatch_prior<64>(prior, args, grid, smem, stream);
    }
}

// Words per prior row: value i at i + 3, rounded up so that every row is 16-byte aligned and
// the last aligned group of four stays inside the row.
int prior_stride(int W1) { return (W1 + 3 + 4 + 3) & ~3; }

// Device-side tables of the fast path and the arguments they were built from.
struct GbTables {
    std::vector<uint8_t> key;
    DevBuf pen, ftab, prior2;
};

GbTables& gb_tables(int device) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<GbTables>> all;
    std::lock_guard<std::mutex> lk(mu);
    auto& p = all[device];
    if (!p) p = std::make_unique<GbTables>();
    return *p;
}

// Penalty grid; per-(M,d) prior rows shifted by their minimum (added back through ftab) and
// clamped at CAP = 2*BIAS + 1 -- a clamped position can never win, because the position holding
// the row's minimum scores at most BIAS while a clamped one scores above it;
// ftab[m][n] = prior minimum + gap_open + (d-1)*gap_extend (int32 wrap, as the reference's
// int32 arithmetic).
void build_tables(GbTables& tb, const std::vector<int32_t>& pen, int32_t go, int32_t ge, int W,
                  int32_t bias, const int32_t* prior, int64_t W1p, cudaStream_t stream) {
    const int W1 = W + 1;
    const int32_t cap = 2 * bias + 1;
    std::vector<int32_t> ftab(size_t(W1) * W1, 0);
    const int pstride = prior_stride(W1);
    std::vector<uint32_t> prior2;
    if (prior) prior2.assign(size_t(W1) * W1 * pstride, 0);
    for (int m = 0; m <= W; ++m)
        for (int n = 0; n <= W; ++n) {
            const int M = std::max(m, n), d = std::abs(m - n), L = std::min(m, n);
            if (d == 0) continue;
            int32_t pmin = 0;
            if (prior) {
                const int32_t* row = prior + (int64_t(M) * W1p + d) * W1p;
                pmin = row[0];
                for (int i = 1; i <= L; ++i) pmin = std::min(pmin, row[i]);
                if (m >= n) {  // fill each (M, d) row once
                    uint32_t* dst = prior2.data() + (size_t(M) * W1 + d) * pstride + 3;
                    for (int i = 0; i <= L; ++i)
                        dst[i] = uint32_t(std::min<int64_t>(int64_t(row[i]) - pmin, cap)) * 0x10001u;
                }
            }
            ftab[size_t(m) * W1 + n] = int32_t(uint32_t(pmin) + uint32_t(go) +
                                               uint32_t(d - 1) * uint32_t(ge));
        }
    h2d(tb.pen.as<int32_t>(pen.size()), pen.data(), pen.size() * 4, stream);
    h2d(tb.ftab.as<int32_t>(ftab.size()), ftab.data(), ftab.size() * 4, stream);
    if (prior)
        h2d(tb.prior2.as<uint32_t>(prior2.size()), prior2.data(),
                                 prior2.size() * 4, stream);
}

// Shared memory of one CTA for a given chunk width.
// CTAs per SM the fast kernel's registers allow (256 threads x <= 80 registers).
constexpr int kTargetBlocks = 3;

// The dense variant stands in for both forms when sizing (same registers and shared memory,
// apart from the epilogue).
const void* fast_kernel_ptr(int lq, bool prior) {
#define STB_K(LQ)                                                                             \
    if (lq == LQ)                                                                             \
        return prior ? reinterpret_cast<const void*>(gapblock_fast_kernel<LQ, true, false>)   \
                     : reinterpret_cast<const void*>(gapblock_fast_kernel<LQ, false, false>);
    STB_K(16) STB_K(24) STB_K(32) STB_K(48)
#undef STB_K
    return prior ? reinterpret_cast<const void*>(gapblock_fast_kernel<64, true, false>)
                 : reinterpret_cast<const void*>(gapblock_fast_kernel<64, false, false>);
}

// The profile area is reused for the per-slice column terms at write-out time.
size_t fast_smem(int lq, int64_t slab_cap, int rc, int W1, int max_tasks) {
    const size_t prof = std::max(size_t(kGP) * lq * kRow * 4, size_t(kGP / kPairsPerSlice) * rc * 4);
    return prof + size_t(slab_cap) + size_t(kGP) * rc * 4 + size_t((W1 * W1 + 3) & ~3) * 4 +
           size_t((rc + 15) & ~15) + size_t(max_tasks) * 16 + size_t((rc + 7) & ~7) * 2 +
           size_t(kGP) * 4 + 16;
}

}  // namespace

namespace {

// Chunk widths the fast kernel may use.  The widest that reaches the best CTA residency is the
// static choice; the autotuner (dense calls) measures all of them once per shape.
constexpr int kRcCandidates[] = {1536, 1280, 1024, 896, 768, 640, 512, 384, 256};
constexpr int kNumRc = int(sizeof(kRcCandidates) / sizeof(kRcCandidates[0]));
// Pairs a dense call's first-time tuning runs each variant on (its first query rows).
constexpr int64_t kTuneSlicePairs = int64_t(100) * 1000 * 1000;
thread_local int t_force_rc = 0;           // set while the autotuner times one chunk width
thread_local int t_force_persistent = -1;  // and the launch form (-1: the tuned or static one)

// The conditions under which gapblock_run takes the fast kernel (non-negative penalties, every
// length <= 64, halves that cannot carry), the form whose sparse output is ordered.
bool fast_form_possible(const st_seqset_s& qs, const st_seqset_s& rs, const int32_t* penalty,
                        int32_t matrix_size) {
    if (qs.alphabet < 0 || qs.alphabet != rs.alphabet) return false;
    const int A = alphabet_size(qs.alphabet);
    if (penalty && matrix_size != A) return false;
    int64_t maxpen = 0;
    for (int x = 0; x < A; ++x)
        for (int y = 0; y < A; ++y) {
            const int64_t v = penalty ? penalty[x * A + y] : int64_t(x != y);
            if (v < 0) return false;
            maxpen = std::max(maxpen, v);
        }
    const int32_t longest = std::max(qs.max_len, rs.max_len);
    return longest <= 64 && int64_t(std::min(qs.max_len, rs.max_len)) * maxpen <= 8191;
}

std::string gb_shape_key(const st_seqset_s& qs, const st_seqset_s& rs, bool has_prior) {
    return "gapblock|" + std::to_string(profile_height(qs.max_len)) + "|" +
           std::to_string(int(has_prior)) + "|" + std::to_string(std::max(qs.max_len, rs.max_len)) +
           "|" + std::to_string(size_bucket(qs.count)) + "|" + std::to_string(size_bucket(rs.count));
}

// Validated inputs -> the dense matrix in `out_d` (device, N*K int32), or, when `sink` is given,
// the cells that pass its threshold appended to it.
// `r0`, `r1` restrict the queries to rows [r0, r1) (r1 = -1: all rows): the sparse form's row
// blocks, and the dense form's first-time tuning slice (which starts at row 0).
void gapblock_run(st_seqset_s& qs, st_seqset_s& rs, const int32_t* penalty, int32_t matrix_size,
                  int32_t go, int32_t ge, const int32_t* prior, int64_t prior_len,
                  uint32_t prior_width, int32_t* out_d, SparseSink* sink,
                  cudaStream_t stream, int64_t r0 = 0, int64_t r1 = -1) {
    if (go < 0 || ge < 0) fail(ST_EINVAL, "gap_open and gap_extend must be >= 0");
    if (qs.alphabet < 0 || qs.alphabet != rs.alphabet)
        fail(ST_EINVAL, "seqtree_b200: gap-block sets must be encoded with one alphabet");
    const int A = alphabet_size(qs.alphabet);
    if (penalty && matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
    const int64_t N = qs.count, K = rs.count;
    if (N == 0 || K == 0) return;
    const int32_t longest = std::max(qs.max_len, rs.max_len);
    const int64_t W1p = int64_t(prior_width) + 1;
    const bool has_prior = prior && prior_len > 0;
    if (has_prior) {
        if (prior_len != W1p * W1p * W1p)
            fail(ST_EINVAL, "prior table must have (prior_width + 1)^3 entries");
        if (uint32_t(longest) > prior_width)
            fail(ST_EINVAL, "a sequence is longer than the prior table's width");
    }
    Context& ctx = context();

    // Penalty grid (unit cost when null): src/gapblock.cpp:25-31.
    std::vector<int32_t> pen(size_t(A) * A);
    for (int x = 0; x < A; ++x)
        for (int y = 0; y < A; ++y) pen[size_t(x) * A + y] = penalty ? penalty[x * A + y] : int32_t(x != y);
    int64_t maxpen = 0;
    bool nonneg = true;
    for (int32_t v : pen) {
        maxpen = std::max<int64_t>(maxpen, v);
        nonneg &= v >= 0;
    }
    const int32_t Lmax = std::min(qs.max_len, rs.max_len);
    const int64_t lmaxpen = int64_t(Lmax) * maxpen;
    bool fast = nonneg && longest <= 64 && lmaxpen <= 8191;

    const int W = longest, W1 = W + 1;
    const int lq = profile_height(qs.max_len);
    const int tuned_choice =
        t_force_rc ? -1
                   : tuned_lookup(sink ? "sparse|" + gb_shape_key(qs, rs, has_prior)
                                       : gb_shape_key(qs, rs, has_prior));
    RefPlan* rpp = nullptr;
    size_t smem = 0;
    if (fast) {
        RefPlan& rp = plan_slot<RefPlan>(rs.gb_ref_plan, ctx.tmp_ref_plan, rs.owns);
        const int want_rc = t_force_rc ? t_force_rc : (tuned_choice >= 0 ? kRcCandidates[tuned_choice % kNumRc] : 0);
        if (rp.uid != rs.uid || (want_rc && rp.rc != want_rc)) {
            Phase ph("ref_plan");
            // Chunk width: the autotuner's measured choice when there is one; otherwise the
            // widest (best warp fill) that still reaches the highest CTA residency the
            // kernel's registers allow, checked with the occupancy calculator.
            const void* kern = fast_kernel_ptr(lq, has_prior);
            int best_rc = 0, best_blocks = -1;
            const std::vector<int> widths =
                want_rc ? std::vector<int>{want_rc} : std::vector<int>{1024, 896, 768, 640, 512, 384, 256};
            for (int rc : widths) {
                build_ref_plan(rp, rs, rc, stream, /*upload=*/false);
                const size_t sm = fast_smem(lq, (rp.max_slab + 15) & ~int64_t(15), rc, W1,
                                            rp.max_tasks);
                if (sm > size_t(ctx.max_smem_optin)) continue;
                int blocks = 0;
                STB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              ctx.max_smem_optin));
                STB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, kThreads, sm));
                if (blocks > best_blocks) {
                    best_blocks = blocks;
                    best_rc = rc;
                }
                if (blocks >= kTargetBlocks) break;
            }
            if (best_rc) {
                build_ref_plan(rp, rs, best_rc, stream);
            } else {
                rp.uid = 0;  // no width fits shared memory: the plan is not used (general kernel)
                rp.ntasks = 0;
            }
            const unsigned blocks = unsigned(rp.ntasks);
            if (blocks) {
                ref_slab_kernel<<<blocks, 128, 0, stream>>>(
                    rs.d_bytes, rs.d_off, static_cast<int32_t*>(rp.d_sorted.ptr),
                    static_cast<int4*>(rp.d_tasks.ptr), static_cast<uint8_t*>(rp.d_slab.ptr));
                STB_CUDA(cudaGetLastError());
                note_launch(nullptr);
            }
        }
        smem = fast_smem(lq, (rp.max_slab + 15) & ~int64_t(15), rp.rc, W1, rp.max_tasks);
        fast = rp.uid == rs.uid && smem <= size_t(ctx.max_smem_optin);
        rpp = &rp;
    }

    if (!sink && !out_d) fail(ST_EINVAL, "seqtree_b200: null output buffer");
    if (!fast && sink && sink->ordered)
        fail(ST_ECUDA, "seqtree_b200: internal error: the ordered sparse form needs the fast kernel");
    if (!fast) {
        int32_t* d_pen = ctx.table_buf.as<int32_t>(pen.size());
        h2d(d_pen, pen.data(), pen.size() * 4, stream);
        int32_t* d_prior = nullptr;
        if (has_prior) {
            d_prior = ctx.prior_buf.as<int32_t>(size_t(prior_len));
            h2d(d_prior, prior, size_t(prior_len) * 4, stream);
        }
        const int64_t rows = (r1 < 0 ? N : r1) - r0;
        GeneralArgs g{qs.d_bytes, qs.d_off, rs.d_bytes, rs.d_off, r0, rows, K, d_pen, A, go, ge,
                      d_prior, W1p, out_d, sink ? *sink : SparseSink{}};
        const int64_t blocks = std::min<int64_t>(ceil_div(rows * K, 256), int64_t(ctx.num_sms) * 16);
        if (sink)
            gapblock_general_kernel<true><<<unsigned(blocks), 256, size_t(A) * A * 4, stream>>>(g);
        else
            gapblock_general_kernel<false><<<unsigned(blocks), 256, size_t(A) * A * 4, stream>>>(g);
        STB_CUDA(cudaGetLastError());
        note_launch(sink ? "gapblock_general_kernel<sparse>" : "gapblock_general_kernel");
        return;
    }
    RefPlan& rp = *rpp;

    // Tables for this (matrix, gaps, prior, lengths): rebuilt only when they change, so repeated
    // calls with the same arguments enqueue nothing but the kernel.
    GbTables& tb = gb_tables(ctx.device);
    const int32_t bias = int32_t(std::max<int64_t>(lmaxpen, 1));
    {
        std::vector<uint8_t> key;
        auto put = [&key](const void* p, size_t n) {
            const auto* b = static_cast<const uint8_t*>(p);
            key.insert(key.end(), b, b + n);
        };
        const int64_t hdr[8] = {A, go, ge, W, bias, int64_t(prior_width), has_prior, 0};
        put(hdr, sizeof hdr);
        put(pen.data(), pen.size() * 4);
        if (has_prior) put(prior, size_t(prior_len) * 4);
        Phase ph("tables");
        if (!same_as_last(tb.key, key.data(), key.size())) {
            try {
                build_tables(tb, pen, go, ge, W, bias, has_prior ? prior : nullptr, W1p, stream);
            } catch (...) {
                tb.key.clear();  // not uploaded: the next call builds them again
                throw;
            }
        }
    }

    // Query pairs and their profile (rebuilt when the set or the penalty grid changes).
    const bool row_block = r0 != 0 || (r1 >= 0 && r1 != N);
    QueryPlan& qp = row_block ? plan_slot<QueryPlan>(ctx.tmp_block_plan, ctx.tmp_block_plan, false)
                              : plan_slot<QueryPlan>(qs.gb_query_plan, ctx.tmp_query_plan, qs.owns);
    if (qp.uid != qs.uid || qp.r0 != r0 || qp.r1 != (row_block ? r1 : -1)) {
        Phase ph("query_plan");
        build_query_plan(qp, qs, stream, r0, row_block ? r1 : -1);
    }
    {
        std::vector<uint8_t> key(sizeof(int) * 2 + pen.size() * 4);
        const int hdr[2] = {A, lq};
        std::memcpy(key.data(), hdr, sizeof hdr);
        std::memcpy(key.data() + sizeof hdr, pen.data(), pen.size() * 4);
        if (!same_as_last(qp.prof_key, key.data(), key.size())) {
            qp.prof_key.clear();  // set again once the profile kernel is enqueued
            const int64_t total = qp.P * lq * kRow;
            uint32_t* prof = qp.d_prof.as<uint32_t>(size_t(total));
            profile_kernel<<<unsigned(ceil_div(total, 256)), 256, 0, stream>>>(
                qs.d_bytes, qs.d_off, static_cast<int2*>(qp.d_pairs.ptr),
                static_cast<int32_t*>(qp.d_plen.ptr), static_cast<int32_t*>(tb.pen.ptr), A, lq,
                total, prof);
            STB_CUDA(cudaGetLastError());
            note_launch(nullptr);
            qp.prof_key = key;
        }
    }

    auto* err = reinterpret_cast<unsigned long long*>(ctx.flags_d + 8);
    STB_CUDA(cudaMemsetAsync(err, 0, 8, stream));

    FastArgs fa{};
    fa.prof = static_cast<uint32_t*>(qp.d_prof.ptr);
    fa.slab = static_cast<uint8_t*>(rp.d_slab.ptr);
    fa.rlen = rs.d_len;
    fa.K = K;
    fa.rc = rp.rc;
    fa.pairs = static_cast<int2*>(qp.d_pairs.ptr);
    fa.plen = static_cast<int32_t*>(qp.d_plen.ptr);
    fa.P = qp.P;
    fa.ref_sorted = static_cast<int32_t*>(rp.d_sorted.ptr);
    fa.tasks = static_cast<int4*>(rp.d_tasks.ptr);
    fa.task_off = static_cast<int32_t*>(rp.d_task_off.ptr);
    fa.slab_cap = int((rp.max_slab + 15) & ~int64_t(15));
    fa.max_tasks = rp.max_tasks;
    fa.prior2 = has_prior ? static_cast<uint32_t*>(tb.prior2.ptr) : nullptr;
    fa.ftab = static_cast<int32_t*>(tb.ftab.ptr);
    fa.W1 = W1;
    fa.pstride = prior_stride(W1);
    fa.bias2 = uint32_t(bias) * 0x10001u;
    fa.out = out_d;
    fa.err = err;
    if (sink && sink->ordered) {
        const int64_t rows = (r1 < 0 ? N : r1) - r0;
        if (rows * int64_t(rp.nchunks) > sink->piece_cap)
            fail(ST_ECUDA, "seqtree_b200: internal error: sparse piece table too small");
        sink->nchunks = rp.nchunks;
        sink->row0 = r0;
    }
    if (sink) fa.sink = *sink;

    const int64_t npg = ceil_div(qp.P, kGP);
    const int64_t ntiles = int64_t(rp.nchunks) * npg;
    const int tuned_mode = t_force_persistent >= 0 ? t_force_persistent
                           : (tuned_choice >= 0 ? tuned_choice / kNumRc : 0);
    dim3 grid(unsigned(rp.nchunks), unsigned(npg));
    if (tuned_mode == 1 && ntiles < (int64_t(1) << 31)) {
        const void* kern = fast_kernel_ptr(lq, has_prior);
        int per_sm = 0;
        STB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        STB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
        fa.persistent = 1;
        fa.nchunks = rp.nchunks;
        fa.ntiles = int(ntiles);
        fa.queue = reinterpret_cast<unsigned int*>(ctx.flags_d + 13);
        STB_CUDA(cudaMemsetAsync(fa.queue, 0, sizeof(unsigned int), stream));
        grid = dim3(unsigned(std::min<int64_t>(ntiles, int64_t(std::max(per_sm, 1)) * ctx.num_sms)), 1);
    } else if (npg > 65535) {
        // pair groups split over y and z (the kernel skips the padding of the last z slice)
        grid.y = 65535;
        grid.z = unsigned(ceil_div(npg, 65535));
        if (grid.z > 65535) fail(ST_EINVAL, "seqtree_b200: too many query pairs for one launch");
    }
    const char* name = dispatch_fast(lq, has_prior, fa, grid, smem, stream);
    note_launch(name);
    // The timeout flag is read by the caller after its synchronisation point.
}

}  // namespace

void gapblock_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* penalty, int32_t matrix_size,
                   int32_t go, int32_t ge, const int32_t* prior, int64_t prior_len,
                   uint32_t prior_width, int32_t* out_d, cudaStream_t stream) {
    auto run = [&] {
        gapblock_run(qs, rs, penalty, matrix_size, go, ge, prior, prior_len, prior_width, out_d,
                     nullptr, stream);
    };
    // Only the fast kernel has a chunk width to choose (non-negative penalties, lengths <= 64;
    // the remaining range checks happen inside and fall back to the general kernel).
    bool nonneg = true;
    const int A = qs.alphabet >= 0 ? alphabet_size(qs.alphabet) : 0;
    if (penalty && matrix_size == A)
        for (int i = 0; i < A * A; ++i) nonneg &= penalty[i] >= 0;
    if (!nonneg || qs.count == 0 || rs.count == 0 || std::max(qs.max_len, rs.max_len) > 64 ||
        qs.alphabet < 0 || qs.alphabet != rs.alphabet || (penalty && matrix_size != A)) {
        run();
        return;
    }
    const bool has_prior = prior && prior_len > 0;
    const std::string key = gb_shape_key(qs, rs, has_prior);
    // Candidates: every chunk width, each with one CTA per tile and in the persistent form.
    auto variant = [&](int c, int64_t rows) {
        t_force_rc = c >= 0 ? kRcCandidates[c % kNumRc] : 0;  // -1: the static choice
        t_force_persistent = c >= 0 ? c / kNumRc : -1;
        try {
            if (rows < 0)
                run();
            else
                gapblock_run(qs, rs, penalty, matrix_size, go, ge, prior, prior_len, prior_width,
                             out_d, nullptr, stream, 0, rows);
        } catch (...) {
            t_force_rc = 0;
            t_force_persistent = -1;
            throw;
        }
        t_force_rc = 0;
        t_force_persistent = -1;
    };
    // A shape seen for the first time is tuned on its first query rows only (about
    // kTuneSlicePairs pairs, written into their own rows of the result), so the first call costs
    // the variants' runs on that slice rather than on the whole matrix; the chosen variant then
    // computes the whole matrix.
    const int64_t slice = std::min<int64_t>(
        qs.count, std::max<int64_t>(4 * kGP * 2, kTuneSlicePairs / std::max<int64_t>(rs.count, 1)));
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    STB_CUDA(cudaStreamIsCapturing(stream, &cs));
    if (slice < qs.count && tuning_enabled() && cs == cudaStreamCaptureStatusNone &&
        tuned_lookup(key) < 0)
        tuned_run(key, 2 * kNumRc, -1, [&](int c) { variant(c, slice); }, stream);
    tuned_run(key, 2 * kNumRc, -1, [&](int c) { variant(c, -1); }, stream);
}

// Scores of listed pairs (device index arrays) into out_d; the general int32 kernel's
// arithmetic, so any lengths and penalties.
void gapblock_pairs_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* qi_d, const int32_t* ri_d,
                         int64_t n, const int32_t* penalty, int32_t matrix_size, int32_t go,
                         int32_t ge, const int32_t* prior, int64_t prior_len, uint32_t prior_width,
                         int32_t* out_d, int32_t* pos_d, cudaStream_t stream) {
    if (go < 0 || ge < 0) fail(ST_EINVAL, "gap_open and gap_extend must be >= 0");
    if (qs.alphabet < 0 || qs.alphabet != rs.alphabet)
        fail(ST_EINVAL, "seqtree_b200: gap-block sets must be encoded with one alphabet");
    const int A = alphabet_size(qs.alphabet);
    if (penalty && matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
    if (n < 0) fail(ST_EINVAL, "seqtree_b200: negative pair count");
    if (n == 0) return;
    const int64_t W1p = int64_t(prior_width) + 1;
    const bool has_prior = prior && prior_len > 0;
    if (has_prior) {
        if (prior_len != W1p * W1p * W1p)
            fail(ST_EINVAL, "prior table must have (prior_width + 1)^3 entries");
        if (uint32_t(std::max(qs.max_len, rs.max_len)) > prior_width)
            fail(ST_EINVAL, "a sequence is longer than the prior table's width");
    }
    Context& ctx = context();
    std::vector<int32_t> pen(size_t(A) * A);
    for (int x = 0; x < A; ++x)
        for (int y = 0; y < A; ++y) pen[size_t(x) * A + y] = penalty ? penalty[x * A + y] : int32_t(x != y);
    // Tables cached per device by content, so repeated calls upload nothing (and can be
    // captured in a CUDA graph once warmed up).
    struct PairTables {
        std::vector<uint8_t> key;
        DevBuf pen, prior;
    };
    static std::mutex mu;
    static std::map<int, std::unique_ptr<PairTables>> all;
    PairTables* pt;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto& slot = all[ctx.device];
        if (!slot) slot = std::make_unique<PairTables>();
        pt = slot.get();
    }
    {
        std::vector<uint8_t> key(pen.size() * 4 + (has_prior ? size_t(prior_len) * 4 : 0) + 8);
        const int64_t hdr = has_prior ? prior_len : -1;
        std::memcpy(key.data(), &hdr, 8);
        std::memcpy(key.data() + 8, pen.data(), pen.size() * 4);
        if (has_prior) std::memcpy(key.data() + 8 + pen.size() * 4, prior, size_t(prior_len) * 4);
        if (!same_as_last(pt->key, key.data(), key.size())) {
            pt->key.clear();
            h2d(pt->pen.as<int32_t>(pen.size()), pen.data(), pen.size() * 4, stream);
            if (has_prior)
                h2d(pt->prior.as<int32_t>(size_t(prior_len)), prior, size_t(prior_len) * 4, stream);
            pt->key = key;
        }
    }
    const int32_t* d_pen = static_cast<const int32_t*>(pt->pen.ptr);
    const int32_t* d_prior = has_prior ? static_cast<const int32_t*>(pt->prior.ptr) : nullptr;
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), int64_t(ctx.num_sms) * 16);
    gapblock_pairs_kernel<<<unsigned(blocks), 256, size_t(A) * A * 4, stream>>>(
        qs.d_bytes, qs.d_off, rs.d_bytes, rs.d_off, qi_d, ri_d, n, d_pen, A, go, ge, d_prior, W1p,
        out_d, pos_d);
    STB_CUDA(cudaGetLastError());
    note_launch("gapblock_pairs_kernel");
}

// ---------------------------------------------------------------------------- sparse --------
namespace {

int bits_for(int64_t n) {  // bits to hold 0..n-1 (at least 1)
    int b = 1;
    while (b < 62 && (int64_t(1) << b) < n) ++b;
    return b;
}

}  // namespace

// Hits of one query-row block: the kernel appends (key, score) pairs, a radix sort orders them by
// key (row-major), and csr_block_kernel writes the block's rows of indptr (offset by `base`) and ref ids.
// The block's ref ids and scores land at `base` in the result arrays.
namespace {

__global__ void csr_block_kernel(const unsigned long long* __restrict__ keys, int64_t H, int shift,
                                 int64_t row0, int64_t rows, int64_t base,
                                 int64_t* __restrict__ indptr, int32_t* __restrict__ ref_ids) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const unsigned long long mask = (1ull << shift) - 1;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t <= rows || t < H;
         t += stride) {
        if (t <= rows) {
            const unsigned long long want = static_cast<unsigned long long>(row0 + t) << shift;
            int64_t lo = 0, hi = H;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (keys[mid] < want) lo = mid + 1;
                else hi = mid;
            }
            indptr[row0 + t] = base + lo;
        }
        if (t < H) ref_ids[base + t] = int32_t(keys[t] & mask);
    }
}

// Ordered form, step 1: hits of each row of the block (the sum of its pieces), one warp per row.
__global__ void piece_rows_kernel(const int32_t* __restrict__ piece_cnt, int64_t rows, int nchunks,
                                  int64_t* __restrict__ rowcnt) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < rows; r += nw) {
        const int32_t* pc = piece_cnt + r * nchunks;
        long long sum = 0;
        for (int c = lane; c < nchunks; c += 32) sum += pc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) rowcnt[r] = sum;
    }
}

// Ordered form, step 2: the block's CSR rows.  start[r] is the exclusive prefix of the rows' hits
// inside the block (start[rows] the block's total) and base the hits of earlier blocks.  A warp
// walks its row's pieces in chunk order -- ascending columns -- and copies each (ref id, score)
// run into place.
__global__ void piece_copy_kernel(const int2* __restrict__ seg, const int64_t* __restrict__ piece_off,
                                  const int32_t* __restrict__ piece_cnt,
                                  const int64_t* __restrict__ start, int64_t rows, int nchunks,
                                  int64_t row0, int64_t base, int64_t* __restrict__ indptr,
                                  int32_t* __restrict__ ref_ids, int32_t* __restrict__ scores) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < rows; r += nw) {
        long long pos = base + start[r];
        if (lane == 0) {
            indptr[row0 + r] = pos;
            if (r == rows - 1) indptr[row0 + rows] = base + start[rows];
        }
        for (int c0 = 0; c0 < nchunks; c0 += 32) {
            const int c = c0 + lane;
            const int32_t cnt = c < nchunks ? piece_cnt[r * nchunks + c] : 0;
            const long long src = cnt > 0 ? piece_off[r * nchunks + c] : 0;
            long long incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long t = __shfl_up_sync(full, incl, o);
                if (lane >= o) incl += t;
            }
            const long long dst = pos + incl - cnt;
            uint32_t m = __ballot_sync(full, cnt > 0);
            while (m) {
                const int L = __ffs(int(m)) - 1;
                m &= m - 1;
                const int32_t n = __shfl_sync(full, cnt, L);
                const long long s0 = __shfl_sync(full, src, L);
                const long long d0 = __shfl_sync(full, dst, L);
                for (int i = lane; i < n; i += 32) {
                    const int2 h = seg[s0 + i];
                    ref_ids[d0 + i] = h.x;
                    scores[d0 + i] = h.y;
                }
            }
            pos += __shfl_sync(full, incl, 31);
        }
    }
}

// Hits one sort takes at most (2^28, about 10 GB of scratch); larger outputs are produced in
// query-row blocks.  SEQTREE_B200_SPARSE_BLOCK_HITS lowers it (at least 1024), e.g. to bound the
// scratch memory.
uint64_t max_block_hits() {
    uint64_t v = uint64_t(1) << 28;
    if (const char* e = std::getenv("SEQTREE_B200_SPARSE_BLOCK_HITS")) {
        const long long x = std::atoll(e);
        if (x > 0) v = std::min<uint64_t>(v, std::max<uint64_t>(uint64_t(x), 1024));
    }
    return v;
}

// Hits one block of the ordered form holds (2^31: 16 GB of segments), or the same override as
// the sort's cap, so that the row-block path can be exercised on small inputs.
uint64_t max_segment_hits() {
    const char* e = std::getenv("SEQTREE_B200_SPARSE_BLOCK_HITS");
    return (e && std::atoll(e) > 0) ? max_block_hits() : (uint64_t(1) << 31);
}

}  // namespace

void gapblock_sparse_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* penalty,
                          int32_t matrix_size, int32_t go, int32_t ge, const int32_t* prior,
                          int64_t prior_len, uint32_t prior_width, int32_t max_penalty,
                          st_hits_s& hits, cudaStream_t stream) {
    if (max_penalty < 0) fail(ST_EINVAL, "max_penalty must be >= 0");
    Context& ctx = context();
    const int64_t N = qs.count, K = rs.count;
    hits.rows = N;
    hits.cols = K;
    hits.nnz = 0;
    int64_t* indptr = hits.indptr.as<int64_t>(size_t(N) + 1);
    if (N == 0 || K == 0) {
        // the dense call's checks still apply (they come before its empty-shape return)
        gapblock_run(qs, rs, penalty, matrix_size, go, ge, prior, prior_len, prior_width, nullptr,
                     nullptr, stream);
        STB_CUDA(cudaMemsetAsync(indptr, 0, sizeof(int64_t) * size_t(N + 1), stream));
        return;
    }
    const int shift = bits_for(K);
    if (shift + bits_for(N) > 63) fail(ST_EINVAL, "seqtree_b200: matrix too large for sparse keys");
    const int end_bit = shift + bits_for(N);
    const uint64_t kMaxBlockHits = max_block_hits();
    auto* count = reinterpret_cast<unsigned long long*>(ctx.flags_d + 10);
    const bool ordered = fast_form_possible(qs, rs, penalty, matrix_size);

    // The fast kernel's chunk width and launch form are tuned once per shape, as for the dense
    // matrix, but on a slice of about 2e9 pairs of rows: every variant counts the slice's hits
    // into the sink (what it stores is overwritten by the passes below).
    {
        const bool has_prior = prior && prior_len > 0;
        const std::string skey = "sparse|" + gb_shape_key(qs, rs, has_prior);
        bool nonneg = qs.alphabet >= 0 && qs.alphabet == rs.alphabet &&
                      std::max(qs.max_len, rs.max_len) <= 64;
        const int A = nonneg ? alphabet_size(qs.alphabet) : 0;
        if (penalty && matrix_size != A) nonneg = false;
        if (nonneg && penalty)
            for (int i = 0; i < A * A; ++i) nonneg &= penalty[i] >= 0;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        STB_CUDA(cudaStreamIsCapturing(stream, &cs));
        if (nonneg && tuning_enabled() && cs == cudaStreamCaptureStatusNone && tuned_lookup(skey) < 0) {
            const int64_t tr1 = std::min<int64_t>(N, std::max<int64_t>(64, int64_t(2000000000) / K));
            const uint64_t tcap = std::min<uint64_t>(std::max<uint64_t>(hits.cap_hint, uint64_t(1) << 20),
                                                     kMaxBlockHits);
            SparseSink ts{};
            ts.count = count;
            ts.cap = tcap;
            ts.shift = shift;
            ts.thresh = max_penalty;
            if (ordered) {
                // room for hits at up to 1/8 density, so that the variants are timed with their
                // hit writes (a tile whose hits do not fit only counts them)
                ts.cap = std::min<uint64_t>(max_segment_hits(),
                                            std::max<uint64_t>(tcap, uint64_t(tr1) * uint64_t(K) / 8));
                ts.ordered = 1;
                ts.seg = ctx.sp_keys.as<int2>(size_t(ts.cap));
                ts.piece_cap = (tr1 == N ? N : tr1) * ceil_div(K, kRcCandidates[kNumRc - 1]);
                ts.piece_off = ctx.sp_sorted.as<int64_t>(size_t(ts.piece_cap));
                ts.piece_cnt = ctx.sp_vals.as<int32_t>(size_t(ts.piece_cap));
            } else {
                ts.keys = ctx.sp_keys.as<unsigned long long>(size_t(tcap));
                ts.vals = ctx.sp_vals.as<int32_t>(size_t(tcap));
            }
            tuned_run(skey, 2 * kNumRc, -1, [&](int c) {
                t_force_rc = c >= 0 ? kRcCandidates[c % kNumRc] : 0;
                t_force_persistent = c >= 0 ? c / kNumRc : -1;
                try {
                    STB_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned long long), stream));
                    gapblock_run(qs, rs, penalty, matrix_size, go, ge, prior, prior_len,
                                 prior_width, nullptr, &ts, stream, 0, tr1 == N ? -1 : tr1);
                } catch (...) {
                    t_force_rc = 0;
                    t_force_persistent = -1;
                    throw;
                }
                t_force_rc = 0;
                t_force_persistent = -1;
            }, stream);
        }
    }

    if (ordered) {
        // Ordered form: no sort.  One block of all rows in the usual case; blocks of rows when
        // the segments (max_segment_hits) or the piece table (2^28 entries) would not hold them.
        const uint64_t seg_cap_max = max_segment_hits();
        const int64_t most_chunks = ceil_div(K, kRcCandidates[kNumRc - 1]);
        const int64_t piece_rows = std::max<int64_t>(1, (int64_t(1) << 28) / most_chunks);
        int64_t r0 = 0, rows = std::min<int64_t>(
            hits.block_rows_hint > 0 ? hits.block_rows_hint : N, piece_rows);
        int64_t first_rows = 0, nblocks = 0, total = 0;
        uint64_t cap = std::min<uint64_t>(std::max<uint64_t>(hits.cap_hint, uint64_t(1) << 20),
                                          seg_cap_max);
        bool exact_retry = false;
        while (r0 < N) {
            const int64_t r1 = std::min<int64_t>(N, r0 + rows);
            SparseSink sink{};
            sink.ordered = 1;
            sink.count = count;
            sink.cap = cap;
            sink.shift = shift;
            sink.thresh = max_penalty;
            sink.seg = ctx.sp_keys.as<int2>(size_t(cap));
            sink.piece_cap = (r1 - r0) * most_chunks;
            sink.piece_off = ctx.sp_sorted.as<int64_t>(size_t(sink.piece_cap));
            sink.piece_cnt = ctx.sp_vals.as<int32_t>(size_t(sink.piece_cap));
            STB_CUDA(cudaMemsetAsync(ctx.flags_d + 8, 0, 8 * sizeof(int64_t), stream));
            gapblock_run(qs, rs, penalty, matrix_size, go, ge, prior, prior_len, prior_width,
                         nullptr, &sink, stream, r0, r1 == N && r0 == 0 ? -1 : r1);
            STB_CUDA(cudaMemcpyAsync(ctx.flags_h + 8, ctx.flags_d + 8, 8 * sizeof(int64_t),
                                     cudaMemcpyDeviceToHost, stream));
            STB_CUDA(cudaStreamSynchronize(stream));
            if (ctx.flags_h[8] != 0)
                fail(ST_ETIMEOUT,
                     "seqtree_b200: a bounded device-side wait gave up (shared-memory staging)");
            const uint64_t H = static_cast<uint64_t>(ctx.flags_h[10]);
            if (H > cap) {
                if (exact_retry) fail(ST_ECUDA, "seqtree_b200: sparse hit count changed between passes");
                const int64_t nrows = r1 - r0;
                if (H <= seg_cap_max || nrows == 1) {
                    cap = H;  // the same block at its exact size (one row holds < 2^31 hits)
                    exact_retry = true;
                } else {
                    const double per_row = double(H) / double(nrows);
                    rows = std::max<int64_t>(
                        1, std::min<int64_t>(nrows - 1, int64_t(0.75 * double(seg_cap_max) / per_row)));
                }
                continue;
            }
            exact_retry = false;
            const int64_t nrows = r1 - r0;
            const size_t need = size_t(total + int64_t(H) + 1);
            hits.ref_ids.grow_keep(need * sizeof(int32_t), size_t(total) * sizeof(int32_t), stream);
            hits.scores.grow_keep(need * sizeof(int32_t), size_t(total) * sizeof(int32_t), stream);
            int64_t* rowcnt = ctx.work_b.as<int64_t>(size_t(2 * (nrows + 1)));
            int64_t* start = rowcnt + (nrows + 1);
            const unsigned wblocks =
                unsigned(std::min<int64_t>(ceil_div(nrows * 32, 256), int64_t(ctx.num_sms) * 16));
            STB_CUDA(cudaMemsetAsync(rowcnt + nrows, 0, sizeof(int64_t), stream));
            piece_rows_kernel<<<wblocks, 256, 0, stream>>>(sink.piece_cnt, nrows, sink.nchunks,
                                                           rowcnt);
            STB_CUDA(cudaGetLastError());
            size_t temp = 0;
            STB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, rowcnt, start, int(nrows + 1),
                                                   stream));
            void* d_temp = ctx.sp_temp.as<uint8_t>(temp + 16);
            STB_CUDA(cub::DeviceScan::ExclusiveSum(d_temp, temp, rowcnt, start, int(nrows + 1),
                                                   stream));
            piece_copy_kernel<<<wblocks, 256, 0, stream>>>(
                sink.seg, sink.piece_off, sink.piece_cnt, start, nrows, sink.nchunks, r0, total,
                indptr, static_cast<int32_t*>(hits.ref_ids.ptr),
                static_cast<int32_t*>(hits.scores.ptr));
            STB_CUDA(cudaGetLastError());
            note_launch(nullptr, 2);
            total += int64_t(H);
            if (nblocks++ == 0) first_rows = nrows;
            const double per_row = double(std::max<uint64_t>(H, 1)) / double(nrows);
            rows = std::min<int64_t>(piece_rows,
                                     std::max<int64_t>(1, int64_t(0.75 * double(seg_cap_max) / per_row)));
            cap = std::min<uint64_t>(
                std::max<uint64_t>(cap, uint64_t(per_row * double(rows) * 1.25) + 1024), seg_cap_max);
            r0 = r1;
        }
        hits.nnz = total;
        hits.block_rows_hint = nblocks > 1 ? first_rows : 0;
        hits.cap_hint = std::max<uint64_t>(
            hits.cap_hint, std::min<uint64_t>(uint64_t(total) + uint64_t(total) / 8, seg_cap_max));
        return;
    }

    // One block of all rows when the hits fit one sort (the usual case: the set's cached plans
    // are used and nothing is copied); otherwise blocks sized from the hit density seen so far.
    int64_t r0 = 0, rows = hits.block_rows_hint > 0 ? hits.block_rows_hint : N;
    int64_t first_rows = 0, nblocks = 0;
    uint64_t cap = std::min<uint64_t>(std::max<uint64_t>(hits.cap_hint, uint64_t(1) << 20),
                                      kMaxBlockHits);
    int64_t total = 0;
    bool exact_retry = false;
    while (r0 < N) {
        const int64_t r1 = std::min<int64_t>(N, r0 + rows);
        SparseSink sink{};
        sink.keys = ctx.sp_keys.as<unsigned long long>(size_t(cap));
        sink.vals = ctx.sp_vals.as<int32_t>(size_t(cap));
        sink.count = count;
        sink.cap = cap;
        sink.shift = shift;
        sink.thresh = max_penalty;
        STB_CUDA(cudaMemsetAsync(ctx.flags_d + 8, 0, 8 * sizeof(int64_t), stream));
        gapblock_run(qs, rs, penalty, matrix_size, go, ge, prior, prior_len, prior_width, nullptr,
                     &sink, stream, r0, r1 == N && r0 == 0 ? -1 : r1);
        STB_CUDA(cudaMemcpyAsync(ctx.flags_h + 8, ctx.flags_d + 8, 8 * sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, stream));
        STB_CUDA(cudaStreamSynchronize(stream));
        if (ctx.flags_h[8] != 0)
            fail(ST_ETIMEOUT, "seqtree_b200: a bounded device-side wait gave up (shared-memory staging)");
        const uint64_t H = static_cast<uint64_t>(ctx.flags_h[10]);
        if (H > cap) {
            if (exact_retry) fail(ST_ECUDA, "seqtree_b200: sparse hit count changed between passes");
            const int64_t nrows = r1 - r0;
            if (H <= kMaxBlockHits || nrows == 1) {
                // same block at its exact size (a single row may exceed the block cap: its hits
                // are at most K < 2^31, what one sort takes)
                cap = H <= kMaxBlockHits ? std::min<uint64_t>(H + H / 8, kMaxBlockHits) : H;
                exact_retry = true;
            } else {  // fewer rows, sized to about 3/4 of a full sort
                const double per_row = double(H) / double(nrows);
                rows = std::max<int64_t>(
                    1, std::min<int64_t>(nrows - 1, int64_t(0.75 * double(kMaxBlockHits) / per_row)));
                cap = kMaxBlockHits;
            }
            continue;
        }
        exact_retry = false;
        // room for this block's results after the previous blocks'
        const size_t need = size_t(total + int64_t(H) + 1);
        hits.ref_ids.grow_keep(need * sizeof(int32_t), size_t(total) * sizeof(int32_t), stream);
        hits.scores.grow_keep(need * sizeof(int32_t), size_t(total) * sizeof(int32_t), stream);
        auto* ref_ids = static_cast<int32_t*>(hits.ref_ids.ptr);
        auto* scores = static_cast<int32_t*>(hits.scores.ptr);
        auto* sorted = ctx.sp_sorted.as<unsigned long long>(size_t(std::max<uint64_t>(H, 1)));
        if (H > 0) {
            size_t temp = 0;
            STB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, sink.keys, sorted, sink.vals,
                                                     scores + total, int(H), 0, end_bit, stream));
            void* d_temp = ctx.sp_temp.as<uint8_t>(temp + 16);
            STB_CUDA(cub::DeviceRadixSort::SortPairs(d_temp, temp, sink.keys, sorted, sink.vals,
                                                     scores + total, int(H), 0, end_bit, stream));
        }
        const int64_t work = std::max<int64_t>(r1 - r0 + 1, int64_t(H));
        const unsigned blocks =
            unsigned(std::min<int64_t>(ceil_div(work, 256), int64_t(ctx.num_sms) * 8));
        csr_block_kernel<<<blocks, 256, 0, stream>>>(sorted, int64_t(H), shift, r0, r1 - r0, total,
                                                     indptr, ref_ids);
        STB_CUDA(cudaGetLastError());
        note_launch(nullptr);
        total += int64_t(H);
        if (nblocks++ == 0) first_rows = r1 - r0;
        // next block: as many rows as this block's density says fit 3/4 of a sort
        const double per_row = double(std::max<uint64_t>(H, 1)) / double(r1 - r0);
        rows = std::max<int64_t>(1, int64_t(0.75 * double(kMaxBlockHits) / per_row));
        cap = std::min<uint64_t>(std::max<uint64_t>(cap, uint64_t(per_row * double(rows) * 1.25) + 1024),
                                 kMaxBlockHits);
        r0 = r1;
    }
    hits.nnz = total;
    hits.block_rows_hint = nblocks > 1 ? first_rows : 0;
    hits.cap_hint = std::max<uint64_t>(hits.cap_hint, std::min<uint64_t>(uint64_t(total) + uint64_t(total) / 8, kMaxBlockHits));
}

}  // namespace stb
