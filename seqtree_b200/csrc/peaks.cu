// Peak issue rates of the instructions the scoring kernels are built from, measured on the
// current device: the integer ALU pipe (LOP3, IADD3), the integer multiply-add (IMAD), the DPX
// operations (__viaddmin_s16x2, __viaddmax_s32, __vimax3_s32) and the conflict-free 32-bit
// shared-memory load.  These are the denominators of the scoring kernels' own rooflines: the
// gap-block sweep is one LDS.32 plus one __viaddmin_s16x2 per pair of cells
// (src/gapblock.cpp:119-125 is the loop it replaces), the Gotoh wavefront is DPX add-max
// operations (src/pairwise.cpp:106-117) and the Levenshtein bit-vector step is LOP3/IADD3 work
// (src/distance.cpp:78-95).
//
// Each thread keeps eight accumulators and updates each from itself and its neighbour every
// iteration, x[j] = op(x[j], x[j+1], c), so no chain is a closed form the compiler could fold and
// four or more updates are independent at any time.  The shared-memory probe walks eight
// independent chains through a table whose rows hold one warp-uniform next-row index, so every
// load of a warp touches 32 distinct banks.  One launch covers one SM (a single 1,024-thread
// block) or every SM (two such blocks per SM); the span of each block is read with clock64, so
// the per-SM-cycle rate does not depend on the clock, and CUDA events give the rate per second
// at the clock the launch ran.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../include/seqtree_b200.h"

namespace {

constexpr int kThreads = 1024;
constexpr int kRows = 128;  // shared-memory table rows of 32 words (16 KB)

int32_t peak_error(st_error* err, int32_t code, const char* msg) {
    if (err) {
        err->code = code;
        std::snprintf(err->message, sizeof err->message, "%s", msg);
    }
    return code;
}

template <int OP>
__device__ __forceinline__ uint32_t step(uint32_t x, uint32_t y, uint32_t c) {
    if constexpr (OP == ST_PEAK_LOP3) {
        uint32_t r;  // one three-input logic operation (x ^ y ^ c), written so it stays one
        asm("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(x), "r"(y), "r"(c));
        return r;
    } else if constexpr (OP == ST_PEAK_IADD3) {
        return x + y + c;
    } else if constexpr (OP == ST_PEAK_IMAD) {
        return x * y + c;
    } else if constexpr (OP == ST_PEAK_VIADDMIN_S16X2) {
        return __viaddmin_s16x2(x, y, c);
    } else if constexpr (OP == ST_PEAK_VIADDMAX_S32) {
        return uint32_t(__viaddmax_s32(int(x), int(y), int(c)));
    } else {
        return uint32_t(__vimax3_s32(int(x), int(y), int(c)));
    }
}

template <int OP>
__global__ void __launch_bounds__(kThreads, 2)
peak_kernel(uint32_t seed, int iters, uint32_t* sink, unsigned long long* cycles) {
    __shared__ uint32_t tab[kRows * 32];
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t x[8];
    if constexpr (OP == ST_PEAK_LDS32) {
        for (int w = threadIdx.x; w < kRows * 32; w += blockDim.x)
            tab[w] = (uint32_t(w >> 5) * 37u + 11u) & (kRows - 1);
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = uint32_t(j * (kRows / 8));
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = seed * (threadIdx.x + 1u) + uint32_t(j) * 0x9E3779B9u;
    }
    const uint32_t c = seed ^ 0x5bd1e995u;
    __syncthreads();
    const unsigned long long t0 = clock64();
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if constexpr (OP == ST_PEAK_LDS32)
                x[j] = tab[(x[j] << 5) | lane];  // x[j] < kRows: in bounds, warp-uniform row
            else
                x[j] = step<OP>(x[j], x[(j + 1) & 7], c);
        }
    }
    __syncthreads();
    const unsigned long long t1 = clock64();
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s ^= x[j];
    if (s == seed + 1u) sink[0] = s;  // keeps the work; practically never taken
    if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
}

template <int OP>
cudaError_t launch_peak(int blocks, int iters, uint32_t seed, uint32_t* sink,
                        unsigned long long* cycles, cudaStream_t s) {
    peak_kernel<OP><<<blocks, kThreads, 0, s>>>(seed, iters, sink, cycles);
    return cudaGetLastError();
}

cudaError_t launch_op(int op, int blocks, int iters, uint32_t seed, uint32_t* sink,
                      unsigned long long* cycles, cudaStream_t s) {
    switch (op) {
        case ST_PEAK_LOP3: return launch_peak<ST_PEAK_LOP3>(blocks, iters, seed, sink, cycles, s);
        case ST_PEAK_IADD3: return launch_peak<ST_PEAK_IADD3>(blocks, iters, seed, sink, cycles, s);
        case ST_PEAK_IMAD: return launch_peak<ST_PEAK_IMAD>(blocks, iters, seed, sink, cycles, s);
        case ST_PEAK_VIADDMIN_S16X2:
            return launch_peak<ST_PEAK_VIADDMIN_S16X2>(blocks, iters, seed, sink, cycles, s);
        case ST_PEAK_VIADDMAX_S32:
            return launch_peak<ST_PEAK_VIADDMAX_S32>(blocks, iters, seed, sink, cycles, s);
        case ST_PEAK_VIMAX3_S32:
            return launch_peak<ST_PEAK_VIMAX3_S32>(blocks, iters, seed, sink, cycles, s);
        default: return launch_peak<ST_PEAK_LDS32>(blocks, iters, seed, sink, cycles, s);
    }
}

}  // namespace

extern "C" int32_t st_measure_peak(int32_t op, int32_t all_sms, st_peak* out, st_error* err) {
    if (op < 0 || op > ST_PEAK_LDS32 || !out)
        return peak_error(err, ST_EINVAL, "seqtree_b200: unknown peak probe or null output");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return peak_error(err, ST_ENODEV, "seqtree_b200: no usable CUDA device");
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) return peak_error(err, ST_ENODEV, "seqtree_b200: no multiprocessors reported");
    const int blocks = all_sms ? 2 * sms : 1;
    const int iters = 16384;
    uint32_t* sink = nullptr;
    unsigned long long* cycles = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<unsigned long long> cyc(size_t(blocks), 0ull);
    float best_ms = 0.f;
    unsigned long long best_cyc = 0ull;
    cudaError_t e = cudaMalloc(&sink, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&cycles, sizeof(unsigned long long) * size_t(blocks));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = launch_op(op, blocks, iters, 0x1234567u, sink, cycles, s);  // warm-up
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
        e = cudaEventRecord(e0, s);
        if (e == cudaSuccess) e = launch_op(op, blocks, iters, 0x1234567u + rep, sink, cycles, s);
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess)
            e = cudaMemcpy(cyc.data(), cycles, sizeof(unsigned long long) * size_t(blocks),
                           cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) break;
        unsigned long long span = 0ull;
        for (auto v : cyc) span = v > span ? v : span;
        if (rep == 0 || ms < best_ms) {
            best_ms = ms;
            best_cyc = span;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (sink) cudaFree(sink);
    if (cycles) cudaFree(cycles);
    if (e != cudaSuccess) {
        char msg[200];
        std::snprintf(msg, sizeof msg, "CUDA error: %s", cudaGetErrorString(e));
        cudaGetLastError();
        return peak_error(err, ST_ECUDA, msg);
    }
    const double lane_ops = double(blocks) * kThreads * double(iters) * 8.0;
    const int used = all_sms ? sms : 1;
    out->lane_ops_per_s = best_ms > 0.f ? lane_ops / (double(best_ms) * 1e-3) : 0.0;
    out->lane_ops_per_sm_clk = best_cyc ? lane_ops / double(used) / double(best_cyc) : 0.0;
    out->ms = double(best_ms);
    out->sms = used;
    out->threads = blocks * kThreads;
    return peak_error(err, ST_OK, "");
}
