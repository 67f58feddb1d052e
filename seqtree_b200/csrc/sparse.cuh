// Thresholded sparse output of the all-vs-all kernels: the cells whose score passes a threshold.
// Two forms:
//   * append: (row << shift | column, score) pairs appended to a device buffer in any order and
//     later radix-sorted into CSR (any kernel);
//   * ordered (the fast gap-block kernel): a CTA owns whole (row, column chunk) pieces of the
//     matrix, so it reserves one contiguous segment for its tile, writes each of its rows' hits
//     there in ascending column order as (ref id, score), and records where each piece starts and
//     how many hits it holds.  The CSR is then a prefix sum over the pieces and a segmented copy,
//     with no sort.
#pragma once

#include <cstdint>

namespace stb {

struct SparseSink {
    unsigned long long* keys = nullptr;   // row << shift | column
    int32_t* vals = nullptr;              // score
    unsigned long long* count = nullptr;  // hits found (may exceed cap; only cap are stored)
    unsigned long long cap = 0;
    int shift = 0;                        // bits of the column index
    int32_t thresh = 0;                   // keep score <= thresh
    // ordered form (cap counts hits of 8 bytes in seg)
    int ordered = 0;
    int2* seg = nullptr;                  // (ref id, score), one segment per tile
    int64_t* piece_off = nullptr;         // [(row - row0) * nchunks + chunk]: start in seg
    int32_t* piece_cnt = nullptr;         // [(row - row0) * nchunks + chunk]: hits of the piece
    int64_t piece_cap = 0;                // entries of piece_off / piece_cnt
    int64_t row0 = 0;                     // first row of the block
    int nchunks = 0;                      // column chunks of the plan (set by the launcher)
};

__device__ __forceinline__ unsigned long long sink_key(const SparseSink& s, int64_t row,
                                                       int64_t col) {
    return (static_cast<unsigned long long>(row) << s.shift) | static_cast<unsigned long long>(col);
}

// Warp-collective append: every lane of the warp calls it (with `hitmask` 0 when it has nothing);
// bit b of a lane's mask asks for entry b, which get(b, key, val) produces.  One atomic per warp
// reserves the warp's slots; entries past the capacity are counted but not stored.
template <class F>
__device__ __forceinline__ void sink_append(const SparseSink& s, uint32_t hitmask, int lane,
                                            F&& get) {
    const unsigned full = 0xffffffffu;
    const int cnt = __popc(hitmask);
    if (!__any_sync(full, cnt != 0)) return;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(full, incl, o);
        if (lane >= o) incl += v;
    }
    unsigned long long base = 0;
    if (lane == 31) base = atomicAdd(s.count, static_cast<unsigned long long>(incl));
    base = __shfl_sync(full, base, 31);
    unsigned long long pos = base + static_cast<unsigned long long>(incl - cnt);
    while (hitmask) {
        const int b = __ffs(int(hitmask)) - 1;
        hitmask &= hitmask - 1;
        if (pos < s.cap) {
            unsigned long long key;
            int32_t val;
            get(b, key, val);
            s.keys[pos] = key;
            s.vals[pos] = val;
        }
        ++pos;
    }
}

}  // namespace stb
