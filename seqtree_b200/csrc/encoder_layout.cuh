// Fixed shape and flat parameter layout of the sequence encoder (shared by the fp32 training
// kernels and the bf16 inference kernels).
#pragma once

#include <cstdint>

namespace stb {
namespace enc {

constexpr int kA = 24, kW = 128, kE = 64, kP = 32;

// flat parameter offsets: W1[3][24][128], b1, W2[384][128], b2, (Wqkv[128][384], bqkv,
// Wo[128][128], bo) x 2, Wout[128][64], bout
constexpr int64_t oW1 = 0, ob1 = oW1 + 3 * kA * kW, oW2 = ob1 + kW, ob2 = oW2 + 3 * kW * kW;
constexpr int64_t oL0 = ob2 + kW;                                   // attention layer 0
constexpr int64_t kLayer = kW * 3 * kW + 3 * kW + kW * kW + kW;     // Wqkv, bqkv, Wo, bo
constexpr int64_t oWout = oL0 + 2 * kLayer, obout = oWout + kW * kE;
constexpr int64_t kParams = obout + kE;
constexpr int64_t lWqkv = 0, lbqkv = kW * 3 * kW, lWo = lbqkv + 3 * kW, lbo = lWo + kW * kW;

}  // namespace enc
}  // namespace stb
