// IslandProfile scoring (seqtree python/seqtree/gapblock.py:365-377, score / score_batch): the
// penalty of each sequence in a profile's frame, as a GPU map over a raw-byte sequence set.
//
// A sequence of length L fits the frame when L <= width and c <= L; it is embedded as its first
// c symbols, width - L gap symbols, then the rest (embed_in_frame, gapblock.py:186-205), and its
// score is the sum over columns of table[j][symbol]; one that does not fit scores `unreachable`.
// The table carries the column penalty of every byte (the profile's `cap` for symbols it does
// not list), so the lookup is one load per column.  One thread per sequence.
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>

#include "common.cuh"

namespace stb {

namespace {

__global__ void profile_score_kernel(const uint8_t* __restrict__ bytes, const int64_t* __restrict__ off,
                                     int64_t n, const int32_t* __restrict__ table, int width, int c,
                                     uint8_t gap, int32_t unreachable, int32_t* __restrict__ out) {
    for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < n;
         s += int64_t(gridDim.x) * blockDim.x) {
        const uint8_t* p = bytes + off[s];
        const int L = int(off[s + 1] - off[s]);
        if (L > width || c > L) {
            out[s] = unreachable;
            continue;
        }
        const int d = width - L;
        int32_t acc = 0;
        for (int j = 0; j < width; ++j) {
            const uint8_t ch = j < c ? p[j] : (j < c + d ? gap : p[j - d]);
            acc += __ldg(table + j * 256 + ch);
        }
        out[s] = acc;
    }
}

struct ProfileTable {
    std::vector<uint8_t> key;
    DevBuf table;
};

}  // namespace

void profile_scores(const int32_t* table, int32_t width, int32_t c, uint8_t gap, int32_t unreachable,
                    const st_seqset_s& set, int32_t* out_d, cudaStream_t stream) {
    if (width < 0 || c < 0 || c > width) fail(ST_EINVAL, "seqtree_b200: frame column outside [0, width]");
    if (set.alphabet != -1) fail(ST_EINVAL, "seqtree_b200: profile scoring takes a raw-byte set");
    if (!table && width > 0) fail(ST_EINVAL, "seqtree_b200: null profile table");
    if (set.count == 0) return;
    Context& ctx = context();
    static std::mutex mu;
    static std::map<int, std::unique_ptr<ProfileTable>> tables;
    ProfileTable* pt;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto& slot = tables[ctx.device];
        if (!slot) slot = std::make_unique<ProfileTable>();
        pt = slot.get();
    }
    const size_t bytes = size_t(std::max(width, 1)) * 256 * sizeof(int32_t);
    int32_t* d_table = pt->table.as<int32_t>(bytes / 4);
    if (width > 0 && !same_as_last(pt->key, table, size_t(width) * 256 * sizeof(int32_t))) {
        try {
            h2d(d_table, table, size_t(width) * 256 * sizeof(int32_t), stream);
        } catch (...) {
            pt->key.clear();
            throw;
        }
    }
    const int64_t blocks = std::min<int64_t>(ceil_div(set.count, 256), int64_t(ctx.num_sms) * 8);
    profile_score_kernel<<<unsigned(blocks), 256, 0, stream>>>(set.d_bytes, set.d_off, set.count,
                                                               d_table, width, c, gap, unreachable,
                                                               out_d);
    STB_CUDA(cudaGetLastError());
    note_launch("profile_score_kernel");
}

}  // namespace stb
