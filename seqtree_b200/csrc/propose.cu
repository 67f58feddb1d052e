// Learned candidate proposal: the top-k refs of every query by embedding dot product, on the
// 5th-generation tensor cores, without ever materialising the query x ref similarity matrix.
//
// Inputs are the encoder's 64-d unit embeddings in bf16, stored [n][64] with the eight 16-byte
// chunks of row r at chunk ^ (r & 7).  That is the 128-byte-swizzled K-major operand layout, so a
// linear bulk copy of 128 consecutive rows into 1024-byte-aligned shared memory is a ready
// tcgen05 operand tile and no tensor map is needed.
//
// One persistent CTA per SM (320 threads) walks query tiles of 256 rows:
//   warp 0     bulk-copies the tile's query rows once, then streams ref tiles of 128 rows
//              through a 6-stage shared-memory ring (cp.async.bulk + mbarrier complete_tx);
//   warp 1     allocates 512 TMEM columns and, from one thread, issues per ref tile two
//              M=128 N=128 K=64 bf16 MMAs (4 x tcgen05.mma K=16 each) into one of two
//              256-column fp32 accumulators, committing the stage and the accumulator to
//              mbarriers;
//   warps 2-9  own one query row each (TMEM lane = row, warp % 4 selects the lane quarter,
//              warps 2-5 read the first query half and 6-9 the second).  Each reads its row's
//              128 fp32 scores with tcgen05.ld, rejects a 32-column group with one 3-input max
//              tree against the running threshold, and otherwise builds the group's survivor bit
//              mask, parks the 32 scores in its own shared-memory row and appends only the set
//              bits (the loop stays small, which measured faster than unrolled or predicated
//              appends) to the query's candidate list in global scratch as 64-bit keys
//              (orderable score << 32 | ~ref_id: larger score first, then smaller ref id).
//              When a list passes kCap - 128 entries, the warp cooperatively radix-selects its
//              k-th largest key, keeps exactly k keys and raises the threshold to the smallest
//              kept score.  After the last ref tile each list is cut to k, sorted by key in
//              shared memory and written out.
//
// Refs are scanned in ascending id order, so a later ref with a score equal to the k-th kept
// one never ranks above it: the strict "score > threshold" test loses no member of the exact
// top-k under that order.  Every wait is bounded (a few seconds of %globaltimer); on time-out
// the CTA records the failure, drains its copies and MMAs with bounded waits, frees TMEM and
// returns.
//
// The threshold form (propose_range_kernel) keeps the producer and MMA warps and replaces the
// selection: a pair is proposed when its score reaches the threshold of its (query length, ref
// length) cell, read from a 33 x 33 table staged in shared memory.  Nothing is kept per query, so
// a group without a survivor costs one TMEM load and one max tree, and survivors are staged per
// warp in shared memory and flushed to global memory 512 pairs at a time (one atomicAdd each).
#include <cuda_bf16.h>

#include <cub/block/block_scan.cuh>

#include <cfloat>
#include <algorithm>
#include <cstdint>
#include <mutex>

#include "common.cuh"
#include "tc.cuh"

namespace stb {

namespace {

constexpr int kRowB = 128;                     // one 64-d bf16 embedding row
constexpr int kQT = 256;                       // queries per tile (two M=128 accumulators)
constexpr int kRT = 128;                       // refs per stage (MMA N)
constexpr int kStages = 6;
constexpr int kCap = 640;                      // candidate keys per query list
constexpr int kPer = kCap / 32;                // keys per lane in a cooperative pass
constexpr int kMaxK = 256;
constexpr int kThreads = 320;
constexpr int kEpiWarps = 8;
constexpr uint32_t kTmemCols = 512;
constexpr int kTileB = kRT * kRowB;            // 16 KB

constexpr int kSmA = 0;                                   // 32 KB: the query tile
constexpr int kSmB = kSmA + kQT * kRowB;                  // 96 KB: the ref ring
constexpr int kSmWarp = kSmB + kStages * kTileB;          // 8 x 2 KB: histogram / sort space
constexpr int kSmPark = kSmWarp + kEpiWarps * 2048;       // 8 x 32 x 128 B: parked scores
constexpr int kSmBar = kSmPark + kEpiWarps * 32 * 128;    // mbarriers and flags
constexpr int kSmTotal = kSmBar + 256;
constexpr size_t kSmemBytes = size_t(kSmTotal) + 1024;    // + alignment slack

// bf16 x bf16 -> fp32, both operands K-major, M = 128, N = 128.
constexpr uint32_t kIdesc = idesc_bf16(128, kRT);


constexpr int kLenSlots = 33;                  // lengths 0..32 of the threshold table
constexpr int kStageBytes = 32 * 128;          // threshold form: a warp's staging buffer (park row)
constexpr int kStage = kStageBytes / 8;        // pairs it holds

struct ProposeArgs {
    const uint8_t* qemb;
    const uint8_t* remb;
    int64_t nq, nr;
    int k;
    const int32_t* ranges;     // null, or per query tile [first, last) ref tile (2 ints)
    unsigned long long* cand;  // [gridDim.x][kQT][kCap]
    int32_t* out_ids;          // [nq][k]
    float* out_scores;         // [nq][k] or null
    unsigned long long* err;
    // threshold form
    const uint8_t* qlens;      // [nq] query lengths
    const uint8_t* rlens;      // [nr] ref lengths
    const float* thr;          // [kLenSlots][kLenSlots] dot-product threshold per length cell
    int32_t* pair_q;           // [cap] proposed pairs: query index
    int32_t* pair_r;           // [cap] proposed pairs: ref index
    unsigned long long cap;
    unsigned long long* count; // every proposed pair counted, the first cap written
    const int4* items;         // threshold form: (query tile, first, last ref tile) work items
    const int* nitems;         //   and their count (device), or null: one unit per query tile
};

// The ref tiles a query tile scans: the caller's [first, last) clamped into [0, ntr), so every
// copy stays inside the ref embeddings whatever the range array holds.
__device__ __forceinline__ int64_t tile_first(const ProposeArgs& a, int64_t qt, int64_t ntr) {
    if (!a.ranges) return 0;
    const int64_t f = a.ranges[2 * qt];
    return f < 0 ? 0 : (f > ntr ? ntr : f);
}
__device__ __forceinline__ int64_t tile_last(const ProposeArgs& a, int64_t qt, int64_t ntr) {
    if (!a.ranges) return ntr;
    const int64_t f = tile_first(a, qt, ntr), l = a.ranges[2 * qt + 1];
    return l < f ? f : (l > ntr ? ntr : l);
}

__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float m;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(m) : "f"(a), "f"(b), "f"(c));
    return m;
}

// Score <-> key half: an unsigned order that matches the float order (non-NaN).
__device__ __forceinline__ uint32_t ord_of(uint32_t u) {
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float score_of(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}
// Acceptance threshold for keys above `min_kept`: any score whose key can exceed it passes
// "s > thr" (a -0.0 threshold is lowered so that +0.0 passes; the test is a superset).
__device__ __forceinline__ float threshold_of(unsigned long long min_kept) {
    const float t = score_of(uint32_t(min_kept >> 32));
    return (t == 0.0f) ? -FLT_TRUE_MIN : t;
}

// ------------------------------------------------------------- warp selection ---------------
// The k-th largest of the n (<= kCap, distinct) keys at `list`, by one warp: 8-bit radix passes
// from the top with a 256-bin shared-memory histogram, stopping as soon as the bin holding the
// k-th key is entirely inside the top k.  Returns T with exactly k keys >= T.
__device__ unsigned long long warp_kth_largest(const unsigned long long (&key)[kPer], int n, int k,
                                               uint32_t* hist, int lane) {
    unsigned long long prefix = 0, pmask = 0;
    int krem = k;
#pragma unroll 1
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int i = lane; i < 256; i += 32) hist[i] = 0;
        __syncwarp();
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            const int idx = lane + 32 * i;
            if (idx < n && (key[i] & pmask) == prefix)
                atomicAdd(&hist[uint32_t(key[i] >> shift) & 255u], 1u);
        }
        __syncwarp();
        // lane l owns bins 255-8l .. 248-8l, highest first
        uint32_t c[8], sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c[j] = hist[255 - 8 * lane - j];
            sum += c[j];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const uint32_t excl = incl - sum;
        const uint32_t owner = __ballot_sync(0xffffffffu, excl < uint32_t(krem) && uint32_t(krem) <= incl);
        const int L = __ffs(owner) - 1;
        uint32_t bin = 0, above = 0, cb = 0;
        if (lane == L) {
            uint32_t acc = excl;
            bool found = false;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (!found && acc + c[j] >= uint32_t(krem)) {
                    found = true;
                    bin = uint32_t(255 - 8 * lane - j);
                    above = acc;
                    cb = c[j];
                }
                acc += c[j];
            }
        }
        bin = __shfl_sync(0xffffffffu, bin, L);
        above = __shfl_sync(0xffffffffu, above, L);
        cb = __shfl_sync(0xffffffffu, cb, L);
        krem -= int(above);
        prefix |= (unsigned long long)bin << shift;
        pmask |= 0xFFull << shift;
        __syncwarp();
        if (int(cb) == krem) break;
    }
    return prefix;
}

// Cuts the list of n > k keys to exactly its k largest (kept in list order) and returns the
// smallest kept key.  Warp-collective.
__device__ unsigned long long warp_cut(unsigned long long* list, int n, int k, uint32_t* hist,
                                       int lane) {
    unsigned long long key[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int idx = lane + 32 * i;
        key[i] = idx < n ? list[idx] : 0ull;
    }
    __syncwarp();
    const unsigned long long T = warp_kth_largest(key, n, k, hist, lane);
    unsigned long long mn = ~0ull;
    int base = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int idx = lane + 32 * i;
        const bool keep = idx < n && key[i] >= T;
        const uint32_t b = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            list[base + __popc(b & ((1u << lane) - 1u))] = key[i];
            mn = key[i] < mn ? key[i] : mn;
        }
        base += __popc(b);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, mn, o);
        mn = t < mn ? t : mn;
    }
    __syncwarp();
    return mn;
}

// Descending bitonic sort of 256 keys in shared memory by one warp.
__device__ void warp_sort256_desc(unsigned long long* s, int lane) {
#pragma unroll 1
    for (int k = 2; k <= 256; k <<= 1) {
#pragma unroll 1
        for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
            for (int t = lane; t < 128; t += 32) {
                const int i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                const int p = i + j;
                const unsigned long long a = s[i], b = s[p];
                const bool desc = (i & k) == 0;
                if (desc ? (a < b) : (a > b)) {
                    s[i] = b;
                    s[p] = a;
                }
            }
            __syncwarp();
        }
    }
}

// ------------------------------------------------------------------------ kernel ------------
// The body of both proposal kernels: the producer and MMA warps are shared; the selection warps
// keep a running top-k (RANGE false) or append every pair at or above its length cell's
// threshold (RANGE true).
template <bool RANGE>
__device__ __forceinline__ void propose_body(const ProposeArgs& a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((uintptr_t(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + kSmBar);
    // bars: [0,6) full, [6,12) empty, 12 a_full, 13 a_empty, 14-15 acc_full, 16-17 acc_empty,
    // 18 done
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + kSmBar + 8 * 20);
    volatile int* s_abort = reinterpret_cast<volatile int*>(smem + kSmBar + 8 * 20 + 4);
    const uint32_t bar0 = smem_u32(bars);
    auto BAR = [&](int i) { return bar0 + 8u * uint32_t(i); };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t ntq = (a.nq + kQT - 1) / kQT, ntr = (a.nr + kRT - 1) / kRT;
    // Work units: a query tile with its range of ref tiles, or (with an item list) a query tile
    // with one chunk of its range.  Every role walks the same units in the same order.
    const int64_t nunits = a.items ? int64_t(*a.nitems) : ntq;
    auto unit = [&](int64_t u, int64_t& qt, int64_t& rt0, int64_t& rt1) {
        if (a.items) {
            const int4 v = a.items[u];
            qt = v.x < 0 ? 0 : (v.x >= ntq ? ntq - 1 : v.x);
            rt0 = v.y < 0 ? 0 : (v.y > ntr ? ntr : v.y);
            rt1 = (v.z < rt0 || v.x < 0 || v.x >= ntq) ? rt0 : (v.z > ntr ? ntr : v.z);
        } else {
            qt = u;
            rt0 = tile_first(a, qt, ntr);
            rt1 = tile_last(a, qt, ntr);
        }
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            bar_init(BAR(s), 1);
            bar_init(BAR(kStages + s), 1);
        }
        bar_init(BAR(12), 1);
        bar_init(BAR(13), 1);
        bar_init(BAR(14), 1);
        bar_init(BAR(15), 1);
        bar_init(BAR(16), kEpiWarps);
        bar_init(BAR(17), kEpiWarps);
        bar_init(BAR(18), 1);
        *s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if constexpr (RANGE) {
        // the threshold table, in the selection warps' scratch (unused by this form)
        float* thr_s = reinterpret_cast<float*>(smem + kSmWarp);
        for (int i = threadIdx.x; i < kLenSlots * kLenSlots; i += kThreads) thr_s[i] = a.thr[i];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_tmem;

    if (warp == 0 && lane == 0) {
        // ---------------------------------------------------------------- producer --------
        const uint32_t sA = smem_u32(smem + kSmA), sB = smem_u32(smem + kSmB);
        uint32_t stage = 0, sphase = 0, aphase = 0;
        uint32_t issued = 0, par = 0;  // per stage: issued at least once, parity of last issue
        bool a_issued = false;
        uint32_t a_par = 0;
        for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
            int64_t qt, rt0, rt1;
            unit(u, qt, rt0, rt1);
            if (!bar_wait(BAR(13), aphase ^ 1u, s_abort, a.err)) break;
            const uint32_t rows = uint32_t((a.nq - qt * kQT < kQT ? a.nq - qt * kQT : kQT));
            bar_expect_tx(BAR(12), rows * kRowB);
            bulk_load(sA, a.qemb + qt * kQT * kRowB, rows * kRowB, BAR(12));
            a_issued = true;
            a_par = aphase;
            aphase ^= 1u;
            bool ok = true;
            for (int64_t rt = rt0; rt < rt1; ++rt) {
                if (!bar_wait(BAR(kStages + stage), sphase ^ 1u, s_abort, a.err)) {
                    ok = false;
                    break;
                }
                const uint32_t rr = uint32_t((a.nr - rt * kRT < kRT ? a.nr - rt * kRT : kRT));
                bar_expect_tx(BAR(stage), rr * kRowB);
                bulk_load(sB + stage * kTileB, a.remb + rt * kRT * kRowB, rr * kRowB, BAR(stage));
                issued |= 1u << stage;
                par = sphase ? (par | (1u << stage)) : (par & ~(1u << stage));
                if (++stage == kStages) {
                    stage = 0;
                    sphase ^= 1u;
                }
            }
            if (!ok) break;
        }
        // Drain: every copy this CTA issued has landed before the CTA can exit.
        for (int s = 0; s < kStages; ++s)
            if (issued & (1u << s)) bar_drain(BAR(s), (par >> s) & 1u);
        if (a_issued) bar_drain(BAR(12), a_par);
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------------------- MMA issuer ---------
        const uint32_t sA = smem_u32(smem + kSmA), sB = smem_u32(smem + kSmB);
        uint32_t stage = 0, sphase = 0, aphase = 0, acc = 0, accphase = 0;
        for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
            int64_t qt, rt0, rt1;
            unit(u, qt, rt0, rt1);
            if (!bar_wait(BAR(12), aphase, s_abort, a.err)) break;
            aphase ^= 1u;
            tc_fence_after();
            bool ok = true;
            for (int64_t rt = rt0; rt < rt1; ++rt) {
                if (!bar_wait(BAR(16 + acc), accphase ^ 1u, s_abort, a.err) ||
                    !bar_wait(BAR(stage), sphase, s_abort, a.err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t bbase = sB + stage * kTileB;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t d = tmem + acc * 256u + uint32_t(h) * 128u;
                    const uint32_t abase = sA + uint32_t(h) * kTileB;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                        tc_mma(d, sw128_desc(abase + 32u * kk), sw128_desc(bbase + 32u * kk),
                               kIdesc, kk > 0 ? 1u : 0u);
                }
                tc_commit(BAR(kStages + stage));  // stage free once these MMAs finish
                tc_commit(BAR(14 + acc));         // accumulator ready
                if (++stage == kStages) {
                    stage = 0;
                    sphase ^= 1u;
                }
                acc ^= 1u;
                if (acc == 0) accphase ^= 1u;
            }
            tc_commit(BAR(13));  // query tile free once the last MMA reading it finishes
            if (!ok) break;
        }
        tc_commit(BAR(18));
        bar_drain(BAR(18), 0);
    } else if (RANGE && warp >= 2) {
        // ------------------------------------------------------ threshold selection -------
        // Lane = query row, as below.  Each lane also loads one column's ref length and a warp
        // vote tells whether the 32-column group has a single length (nearly every group when
        // the refs are sorted by length; any order is correct).  Such a group is rejected by one
        // 3-input max tree against the row's threshold for that length; otherwise each column's
        // threshold is looked up with its length taken by shuffle.  Survivors are staged per
        // warp in shared memory and flushed to global memory with one atomicAdd per flush.
        const int ew = warp - 2, grp = ew >> 2, quarter = warp & 3;
        const int row = quarter * 32 + lane;
        const float* thr_s = reinterpret_cast<const float*>(smem + kSmWarp);
        const uint32_t tlane = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(grp) * 128u;
        // Survivors go to a warp-private staging buffer in shared memory (the park area,
        // unused by this form) and reach global memory in flushes of up to kStage pairs, one
        // atomicAdd each, so no tile waits for an atomic's round trip.  A tile with more
        // survivors than the buffer holds appends them to global memory directly.
        int2* wbuf = reinterpret_cast<int2*>(smem + kSmPark + ew * kStageBytes);
        int wcnt = 0;  // warp-uniform
        auto flush = [&] {
            __syncwarp();
            unsigned long long base = 0;
            if (lane == 0 && wcnt) base = atomicAdd(a.count, (unsigned long long)wcnt);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            for (int i = lane; i < wcnt; i += 32) {
                const unsigned long long pos = base + unsigned(i);
                if (pos < a.cap) {
                    const int2 e = wbuf[i];
                    a.pair_q[pos] = e.x;
                    a.pair_r[pos] = e.y;
                }
            }
            __syncwarp();
            wcnt = 0;
        };
        uint32_t acc = 0, accphase = 0;
        bool ok = true;
        for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
            int64_t qt, rt0, rt1;
            unit(u, qt, rt0, rt1);
            const int64_t q = qt * kQT + grp * 128 + row;
            const bool qvalid = q < a.nq;
            const int ql = qvalid ? min(int(a.qlens[q]), kLenSlots - 1) : 0;
            const float* trow = thr_s + ql * kLenSlots;
            // Survivor mask of one 32-column group.  `uni` / `t`: the group has one ref length
            // and its threshold; otherwise each column's threshold is looked up with its length
            // (`lcol`, -1 past the refs) taken by shuffle.
            auto group_mask = [&](const uint32_t (&v)[32], int lcol, bool uni, float t, int nv) {
                uint32_t mask = 0;
                if (uni) {
                    float m[11];
#pragma unroll
                    for (int j = 0; j < 10; ++j)
                        m[j] = fmax3(__uint_as_float(v[3 * j]), __uint_as_float(v[3 * j + 1]),
                                     __uint_as_float(v[3 * j + 2]));
                    m[10] = fmaxf(__uint_as_float(v[30]), __uint_as_float(v[31]));
                    const float mx = fmaxf(fmax3(fmax3(m[0], m[1], m[2]), fmax3(m[3], m[4], m[5]),
                                                 fmax3(m[6], m[7], m[8])),
                                           fmax3(m[9], m[10], -INFINITY));
                    if (mx >= t) {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            mask |= (__uint_as_float(v[j]) >= t) ? (1u << j) : 0u;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int lj = __shfl_sync(0xFFFFFFFFu, lcol, j);
                        if (lj >= 0) mask |= (__uint_as_float(v[j]) >= trow[lj]) ? (1u << j) : 0u;
                    }
                }
                const uint32_t vmask = nv >= 32 ? 0xFFFFFFFFu : (nv > 0 ? (1u << nv) - 1u : 0u);
                return qvalid ? (mask & vmask) : 0u;
            };
            auto append = [&](const uint32_t (&mk)[kRT / 32], int64_t r0) {
                uint32_t n = 0;
#pragma unroll
                for (int g = 0; g < kRT / 32; ++g) n += __popc(mk[g]);
                uint32_t incl = n;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                    if (lane >= o) incl += t;
                }
                const int tot = int(__shfl_sync(0xFFFFFFFFu, incl, 31));
                if (wcnt + tot > kStage) flush();
                if (tot <= kStage) {
                    int at = wcnt + int(incl - n);
#pragma unroll
                    for (int g = 0; g < kRT / 32; ++g) {
                        uint32_t mask = mk[g];
                        while (mask) {
                            const int j = __ffs(mask) - 1;
                            mask &= mask - 1;
                            wbuf[at++] = make_int2(int32_t(q), int32_t(r0 + g * 32 + j));
                        }
                    }
                    wcnt += tot;
                    return;
                }
                unsigned long long base = 0;
                if (lane == 31) base = atomicAdd(a.count, (unsigned long long)tot);
                base = __shfl_sync(0xFFFFFFFFu, base, 31);
                unsigned long long pos = base + (incl - n);
#pragma unroll
                for (int g = 0; g < kRT / 32; ++g) {
                    uint32_t mask = mk[g];
                    while (mask) {
                        const int j = __ffs(mask) - 1;
                        mask &= mask - 1;
                        if (pos < a.cap) {
                            a.pair_q[pos] = int32_t(q);
                            a.pair_r[pos] = int32_t(r0 + g * 32 + j);
                        }
                        ++pos;
                    }
                }
            };
            // Column lengths of a ref tile (lane l: columns l, l+32, l+64, l+96; -1 past the
            // refs), loaded one tile ahead so that their latency hides behind a whole tile.
            auto load_lens = [&](int64_t rt, int (&lc)[kRT / 32]) {
                const int64_t r0 = rt * kRT;
                const int nvalid = int((a.nr - r0 < kRT ? a.nr - r0 : kRT));
#pragma unroll
                for (int g = 0; g < kRT / 32; ++g) {
                    const int col = g * 32 + lane;
                    lc[g] = col < nvalid ? int(a.rlens[r0 + col]) : -1;
                }
            };
            int lnext[kRT / 32];
            if (rt0 < rt1) load_lens(rt0, lnext);
            for (int64_t rt = rt0; rt < rt1; ++rt) {
                const int64_t r0 = rt * kRT;
                const int nvalid = int((a.nr - r0 < kRT ? a.nr - r0 : kRT));
                // Before the accumulator wait: whether each group has a single length, and that
                // length's threshold for this row.
                int lc[kRT / 32];
                bool uni[kRT / 32];
                float tg[kRT / 32];
#pragma unroll
                for (int g = 0; g < kRT / 32; ++g) lc[g] = min(lnext[g], kLenSlots - 1);
                if (rt + 1 < rt1) load_lens(rt + 1, lnext);
#pragma unroll
                for (int g = 0; g < kRT / 32; ++g) {
                    const int l0 = __shfl_sync(0xFFFFFFFFu, lc[g], 0);
                    uni[g] = __all_sync(0xFFFFFFFFu, lc[g] == l0 || lc[g] < 0);
                    tg[g] = l0 >= 0 ? trow[l0] : INFINITY;
                }
                if (!bar_wait(BAR(14 + acc), accphase, s_abort, a.err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                // two groups per round: both TMEM loads in flight, then both masks
                uint32_t va[32], vb[32], mk[kRT / 32];
                const uint32_t tbase = tlane + acc * 256u;
                __syncwarp();
#pragma unroll
                for (int h = 0; h < kRT / 64; ++h) {
                    const int g0 = 2 * h, g1 = 2 * h + 1;
                    mk[g0] = mk[g1] = 0u;
                    if (nvalid > g0 * 32) {  // warp-uniform
                        tmem_ld32_issue(tbase + uint32_t(g0 * 32), va);
                        if (nvalid > g1 * 32) tmem_ld32_issue(tbase + uint32_t(g1 * 32), vb);
                        tmem_ld32_wait(va);
                        mk[g0] = group_mask(va, lc[g0], uni[g0], tg[g0], nvalid - g0 * 32);
                        if (nvalid > g1 * 32) {
                            tmem_ld32_wait(vb);
                            mk[g1] = group_mask(vb, lc[g1], uni[g1], tg[g1], nvalid - g1 * 32);
                        }
                    }
                }
                // the accumulator is free as soon as it has been read
                tc_fence_before();
                __syncwarp();
                if (lane == 0) bar_arrive(BAR(16 + acc));
                acc ^= 1u;
                if (acc == 0) accphase ^= 1u;
                if (__any_sync(0xFFFFFFFFu, (mk[0] | mk[1] | mk[2] | mk[3]) != 0u)) append(mk, r0);
            }
        }
        flush();
    } else if (!RANGE && warp >= 2) {
        // --------------------------------------------------------------- selection --------
        const int ew = warp - 2, grp = ew >> 2, quarter = warp & 3;
        const int row = quarter * 32 + lane;
        uint32_t* hist = reinterpret_cast<uint32_t*>(smem + kSmWarp + ew * 2048);
        unsigned long long* sortbuf = reinterpret_cast<unsigned long long*>(hist);
        unsigned long long* lists =
            a.cand + (int64_t(blockIdx.x) * kQT + grp * 128 + quarter * 32) * kCap;
        unsigned long long* mine = lists + int64_t(lane) * kCap;
        uint32_t* park = reinterpret_cast<uint32_t*>(smem + kSmPark + (ew * 32 + lane) * 128);
        const uint32_t tlane = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(grp) * 128u;
        uint32_t acc = 0, accphase = 0;
        bool ok = true;
        for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
            int64_t qt, rt0, rt1;
            unit(u, qt, rt0, rt1);
            const int64_t q = qt * kQT + grp * 128 + row;
            float thr = q < a.nq ? -INFINITY : INFINITY;
            int count = 0;
            for (int64_t rt = rt0; rt < rt1; ++rt) {
                if (!bar_wait(BAR(14 + acc), accphase, s_abort, a.err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int64_t r0 = rt * kRT;
                const int nvalid = int((a.nr - r0 < kRT ? a.nr - r0 : kRT));
#pragma unroll 1
                for (int c = 0; c < kRT / 32; ++c) {
                    uint32_t v[32];
                    __syncwarp();
                    tmem_ld32(tlane + acc * 256u + uint32_t(c) * 32u, v);
                    if (c * 32 + 32 > nvalid) {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (c * 32 + j >= nvalid) v[j] = 0xFF800000u;  // -inf
                    }
                    float m[11];
#pragma unroll
                    for (int j = 0; j < 10; ++j)
                        m[j] = fmax3(__uint_as_float(v[3 * j]), __uint_as_float(v[3 * j + 1]),
                                     __uint_as_float(v[3 * j + 2]));
                    m[10] = fmaxf(__uint_as_float(v[30]), __uint_as_float(v[31]));
                    const float mx = fmaxf(fmax3(fmax3(m[0], m[1], m[2]), fmax3(m[3], m[4], m[5]),
                                                 fmax3(m[6], m[7], m[8])),
                                           fmax3(m[9], m[10], -INFINITY));
                    if (mx > thr) {
                        // survivors as a bit mask; the 32 values parked in this thread's
                        // shared-memory row (16-byte chunks swizzled by lane) so that only the
                        // set bits are visited
                        uint32_t mask = 0;
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            mask |= (__uint_as_float(v[j]) > thr) ? (1u << j) : 0u;
#pragma unroll
                        for (int ch = 0; ch < 8; ++ch)
                            *reinterpret_cast<uint4*>(park + ((ch ^ (lane & 7)) << 2)) =
                                make_uint4(v[4 * ch], v[4 * ch + 1], v[4 * ch + 2], v[4 * ch + 3]);
                        const uint32_t rbase = uint32_t(r0 + c * 32);
                        while (mask) {
                            const int j = __ffs(mask) - 1;
                            mask &= mask - 1;
                            const uint32_t x = park[(((j >> 2) ^ (lane & 7)) << 2) | (j & 3)];
                            mine[count++] = ((unsigned long long)ord_of(x) << 32) |
                                            (unsigned long long)(~(rbase + uint32_t(j)));
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) bar_arrive(BAR(16 + acc));
                acc ^= 1u;
                if (acc == 0) accphase ^= 1u;
                // Lists about to overflow are cut back to k (room for a full tile remains).
                uint32_t need = __ballot_sync(0xffffffffu, count > kCap - kRT);
                while (need) {
                    const int L = __ffs(need) - 1;
                    need &= need - 1;
                    const int n = __shfl_sync(0xffffffffu, count, L);
                    const unsigned long long mn =
                        warp_cut(lists + int64_t(L) * kCap, n, a.k, hist, lane);
                    if (lane == L) {
                        count = a.k;
                        thr = threshold_of(mn);
                    }
                }
            }
            if (!ok) break;
            // Final lists: cut to k, sort by key (score descending, then ref ascending), store.
            __syncwarp();
            for (int L = 0; L < 32; ++L) {
                const int64_t qL = qt * kQT + grp * 128 + quarter * 32 + L;
                if (qL >= a.nq) break;
                int n = __shfl_sync(0xffffffffu, count, L);
                unsigned long long* list = lists + int64_t(L) * kCap;
                if (n > a.k) {
                    warp_cut(list, n, a.k, hist, lane);
                    n = a.k;
                }
                for (int i = lane; i < kMaxK; i += 32) sortbuf[i] = i < n ? list[i] : 0ull;
                __syncwarp();
                warp_sort256_desc(sortbuf, lane);
                for (int i = lane; i < a.k; i += 32) {
                    const unsigned long long key = sortbuf[i];
                    a.out_ids[qL * a.k + i] = i < n ? int32_t(~uint32_t(key)) : -1;
                    if (a.out_scores)
                        a.out_scores[qL * a.k + i] = i < n ? score_of(uint32_t(key >> 32)) : -INFINITY;
                }
                __syncwarp();
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols));
    }
}

__global__ void __launch_bounds__(kThreads, 1) propose_topk_kernel(ProposeArgs a) {
    propose_body<false>(a);
}

__global__ void __launch_bounds__(kThreads, 1) propose_range_kernel(ProposeArgs a) {
    propose_body<true>(a);
}

// The threshold form's work list: each query tile's ref-tile range [first, last) (every ref tile
// without ranges; clamped like tile_first / tile_last) cut into chunks of at most kItemTiles
// tiles, query tile by query tile.  One block of 1024 threads; a tile's pairs need no state
// across chunks, so any split gives the same pairs, and equal-sized items keep the persistent
// CTAs balanced whatever the ranges' lengths.
constexpr int kItemTiles = 32;
constexpr int kItemThreads = 1024;

__global__ void __launch_bounds__(kItemThreads) range_items_kernel(const int32_t* ranges,
                                                                   int64_t ntq, int64_t ntr,
                                                                   int4* items, int* nitems) {
    typedef cub::BlockScan<int, kItemThreads> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int s_base;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int64_t t0 = 0; t0 < ntq; t0 += kItemThreads) {
        const int64_t t = t0 + threadIdx.x;
        int64_t f = 0, l = 0;
        if (t < ntq) {
            if (ranges) {
                f = ranges[2 * t];
                f = f < 0 ? 0 : (f > ntr ? ntr : f);
                l = ranges[2 * t + 1];
                l = l < f ? f : (l > ntr ? ntr : l);
            } else {
                l = ntr;
            }
        }
        const int cnt = int((l - f + kItemTiles - 1) / kItemTiles);
        int excl = 0, total = 0;
        Scan(tmp).ExclusiveSum(cnt, excl, total);
        const int base = s_base;
        for (int c = 0; c < cnt; ++c) {
            const int64_t c0 = f + int64_t(c) * kItemTiles;
            items[base + excl + c] =
                make_int4(int(t), int(c0), int(c0 + kItemTiles < l ? c0 + kItemTiles : l), 0);
        }
        __syncthreads();
        if (threadIdx.x == 0) s_base = base + total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *nitems = s_base;
}

// Dot products of listed (query, ref) pairs of swizzled bf16 embeddings, one thread per pair,
// fp32 accumulation in chunk order.  An index outside its embedding set gives NaN.
__global__ void embed_dots_kernel(const uint4* __restrict__ qemb, int64_t nq,
                                  const uint4* __restrict__ remb, int64_t nr,
                                  const int32_t* __restrict__ qi, const int32_t* __restrict__ ri,
                                  int64_t n, float* __restrict__ out) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int64_t a = qi[p], b = ri[p];
    if (a < 0 || a >= nq || b < 0 || b >= nr) {
        out[p] = __int_as_float(0x7FC00000);
        return;
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint4 x = qemb[a * 8 + (c ^ int(a & 7))];
        const uint4 y = remb[b * 8 + (c ^ int(b & 7))];
        const uint32_t xs[4] = {x.x, x.y, x.z, x.w}, ys[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const float2 fx = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&xs[w]));
            const float2 fy = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&ys[w]));
            s = fmaf(fx.x, fy.x, s);
            s = fmaf(fx.y, fy.y, s);
        }
    }
    out[p] = s;
}

}  // namespace

// Top-k refs of every query by dot product of the swizzled bf16 embeddings (device memory, 16-byte
// aligned).  ids[q][i] / scores[q][i] hold the i-th best ref of query q (score descending, ties by
// ascending ref id); entries past the number of refs are -1 / -inf.
void propose_topk(const void* qemb, int64_t nq, const void* remb, int64_t nr, int k, int32_t* ids,
                  float* scores, cudaStream_t stream, const int32_t* ranges) {
    if (nq < 0 || nr < 0) fail(ST_EINVAL, "seqtree_b200: negative embedding count");
    if (k < 1 || k > kMaxK) fail(ST_EINVAL, "seqtree_b200: k must be in 1..256");
    if (nr >= (int64_t(1) << 31)) fail(ST_EINVAL, "seqtree_b200: at most 2^31 - 1 refs");
    if (nq == 0) return;
    if (!qemb || !ids || (nr > 0 && !remb)) fail(ST_EINVAL, "seqtree_b200: null embedding or output");
    if ((uintptr_t(qemb) | uintptr_t(remb)) & 15)
        fail(ST_EINVAL, "seqtree_b200: embeddings must be 16-byte aligned");
    Context& ctx = context();
    ensure_smem_limit(reinterpret_cast<const void*>(propose_topk_kernel), kSmemBytes);
    const int64_t ntq = (nq + kQT - 1) / kQT;
    const int grid = int(std::min<int64_t>(ntq, ctx.num_sms));
    ProposeArgs a{};
    a.qemb = static_cast<const uint8_t*>(qemb);
    a.remb = static_cast<const uint8_t*>(remb);
    a.nq = nq;
    a.nr = nr;
    a.k = k;
    a.ranges = ranges;
    a.cand = ctx.topk_cand.as<unsigned long long>(size_t(grid) * kQT * kCap);
    a.out_ids = ids;
    a.out_scores = scores;
    a.err = reinterpret_cast<unsigned long long*>(ctx.flags_d + 8);
    propose_topk_kernel<<<grid, kThreads, kSmemBytes, stream>>>(a);
    STB_CUDA(cudaGetLastError());
    note_launch("propose_topk_kernel");
}

// Every (query, ref) pair whose embedding dot product is >= thr[qlen][rlen] (host float
// [33][33]; lengths above 32 use row / column 32).  Writes the first `cap` pairs found (in no
// particular order) to pq / pr and returns how many pairs pass in all.  Synchronous on `stream`.
int64_t propose_range(const void* qemb, int64_t nq, const uint8_t* qlens, const void* remb,
                      int64_t nr, const uint8_t* rlens, const float* thr, int32_t* pq, int32_t* pr,
                      int64_t cap, cudaStream_t stream, const int32_t* ranges) {
    if (nq < 0 || nr < 0) fail(ST_EINVAL, "seqtree_b200: negative embedding count");
    if (cap < 0) fail(ST_EINVAL, "seqtree_b200: negative pair capacity");
    if (nq >= (int64_t(1) << 31) || nr >= (int64_t(1) << 31))
        fail(ST_EINVAL, "seqtree_b200: at most 2^31 - 1 queries and refs");
    if (!thr) fail(ST_EINVAL, "seqtree_b200: null threshold table");
    if (nq == 0 || nr == 0) return 0;
    if (!qemb || !remb || !qlens || !rlens || (cap > 0 && (!pq || !pr)))
        fail(ST_EINVAL, "seqtree_b200: null embedding, length or output");
    if ((uintptr_t(qemb) | uintptr_t(remb)) & 15)
        fail(ST_EINVAL, "seqtree_b200: embeddings must be 16-byte aligned");
    Context& ctx = context();
    constexpr size_t kThrBytes = sizeof(float) * kLenSlots * kLenSlots;
    float* d_thr = ctx.prop_thr.as<float>(kLenSlots * kLenSlots);
    if (!same_as_last(ctx.prop_thr_key, thr, kThrBytes)) h2d(d_thr, thr, kThrBytes, stream);
    ensure_smem_limit(reinterpret_cast<const void*>(propose_range_kernel), kSmemBytes);
    const int64_t ntq = (nq + kQT - 1) / kQT, ntr = (nr + kRT - 1) / kRT;
    const int64_t max_items = ntq * ((ntr + kItemTiles - 1) / kItemTiles);
    if (max_items >= (int64_t(1) << 31)) fail(ST_EINVAL, "seqtree_b200: too many proposal work items");
    int4* items = ctx.prop_items.as<int4>(size_t(max_items));
    int* nitems = reinterpret_cast<int*>(ctx.flags_d + 12);
    range_items_kernel<<<1, kItemThreads, 0, stream>>>(ranges, ntq, ntr, items, nitems);
    STB_CUDA(cudaGetLastError());
    note_launch(nullptr);
    const int grid = int(std::min<int64_t>(max_items, ctx.num_sms));
    ProposeArgs a{};
    a.qemb = static_cast<const uint8_t*>(qemb);
    a.remb = static_cast<const uint8_t*>(remb);
    a.nq = nq;
    a.nr = nr;
    a.ranges = ranges;
    a.err = reinterpret_cast<unsigned long long*>(ctx.flags_d + 8);
    a.qlens = qlens;
    a.rlens = rlens;
    a.thr = d_thr;
    a.pair_q = pq;
    a.pair_r = pr;
    a.cap = static_cast<unsigned long long>(cap);
    a.count = reinterpret_cast<unsigned long long*>(ctx.flags_d + 11);
    a.items = items;
    a.nitems = nitems;
    STB_CUDA(cudaMemsetAsync(ctx.flags_d + 8, 0, 4 * sizeof(int64_t), stream));
    propose_range_kernel<<<grid, kThreads, kSmemBytes, stream>>>(a);
    STB_CUDA(cudaGetLastError());
    note_launch("propose_range_kernel");
    STB_CUDA(cudaMemcpyAsync(ctx.flags_h + 8, ctx.flags_d + 8, 8 * sizeof(int64_t),
                             cudaMemcpyDeviceToHost, stream));
    STB_CUDA(cudaStreamSynchronize(stream));
    if (ctx.flags_h[8] != 0)
        fail(ST_ETIMEOUT, "seqtree_b200: a bounded device-side wait gave up (proposal)");
    return ctx.flags_h[11];
}

// Dot products of listed pairs of swizzled bf16 embeddings (asynchronous on `stream`).
void embed_dots(const void* qemb, int64_t nq, const void* remb, int64_t nr, const int32_t* qi,
                const int32_t* ri, int64_t n, float* out, cudaStream_t stream) {
    if (nq < 0 || nr < 0 || n < 0) fail(ST_EINVAL, "seqtree_b200: negative count");
    if (n == 0) return;
    if (!qemb || !remb || !qi || !ri || !out)
        fail(ST_EINVAL, "seqtree_b200: null embedding, index or output");
    if ((uintptr_t(qemb) | uintptr_t(remb)) & 15)
        fail(ST_EINVAL, "seqtree_b200: embeddings must be 16-byte aligned");
    context();
    const int threads = 256;
    const int64_t blocks = (n + threads - 1) / threads;
    if (blocks > 0x7FFFFFFF) fail(ST_EINVAL, "seqtree_b200: too many pairs for one call");
    embed_dots_kernel<<<unsigned(blocks), threads, 0, stream>>>(
        static_cast<const uint4*>(qemb), nq, static_cast<const uint4*>(remb), nr, qi, ri, n, out);
    STB_CUDA(cudaGetLastError());
    note_launch("embed_dots_kernel");
}

}  // namespace stb
