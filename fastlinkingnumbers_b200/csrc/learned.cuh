// Learned opening criterion for the two-tree Barnes–Hut traversal: a small
// MLP (8 -> 64 -> 64 -> 1, ReLU) that predicts log10 of the far-field error
// of a node pair, so that the traversal can accept as far-field a pair the
// beta test would open when the predicted error is below a threshold.
//
// Shared between bh.cu (inference inside the traversal, sampling of training
// node pairs) and learned.cu (features, exact errors, training kernels).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.hpp"

namespace fln {

constexpr int kMlpIn = 8, kMlpHidden = 64;
// FP32 master parameters, contiguous: W1[8][64], b1[64], W2[64][64], b2[64], w3[64], b3.
constexpr int kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpIn * kMlpHidden, kMlpW2 = kMlpB1 + kMlpHidden,
              kMlpB2 = kMlpW2 + kMlpHidden * kMlpHidden, kMlpW3 = kMlpB2 + kMlpHidden,
              kMlpB3 = kMlpW3 + kMlpHidden, kMlpParams = kMlpB3 + 1;

// Inference copy: BF16 weights laid out as mma.sync m16n8k16 B fragments
// (one 32-bit register pair per lane per tile) plus FP32 biases.
struct MlpFrag {
  uint32_t w1[8][32][2];     // layer 1: K = 16 (8 inputs + 8 zero rows), 8 n-tiles
  uint32_t w2[4][8][32][2];  // layer 2: 4 k-tiles x 8 n-tiles
  float w3f[64];             // layer 3 (64 -> 1), BF16-rounded, in FP32
  float b1[64], b2[64], b3;
};

// Node-pair features (dimensionless), computed identically for training and
// inference from the two nodes' centres, radii and moment norms:
//   0 s = |dr| / (r1 + r2)            1 r1 / (r1 + r2)
//   2 log10 |c1||c2| / (4 pi d^2) / 4 3 log10 (Eq. 14 estimate x 1/(4 pi d^3)) / 4
//   4 min(|c1| / 2 r1, 2)             5 min(|c2| / 2 r2, 2)
//   6 min(D1 / (|c1| r1), 4)          7 min(D2 / (|c2| r2), 4)
__device__ __forceinline__ void mlp_features(float s, float r1, float r2, double dsq, float tn1, float tn2,
                                             float dn1, float dn2, float qn1, float qn2, float *f) {
  const float inv4pi = 0.0795774715459476678844f;
  const float d2 = (float)dsq, d = sqrtf(d2);
  const float est = (1.f / d2) * (qn1 * (r1 * tn2 + 3.f * dn2) + qn2 * (r2 * tn1 + 3.f * dn1)) * inv4pi / (d2 * d);
  f[0] = s;
  f[1] = r1 / (r1 + r2 + 1e-30f);
  f[2] = log10f(tn1 * tn2 * inv4pi / d2 + 1e-30f) * 0.25f;
  f[3] = log10f(est + 1e-30f) * 0.25f;
  f[4] = fminf(tn1 / (2.f * r1 + 1e-30f), 2.f);
  f[5] = fminf(tn2 / (2.f * r2 + 1e-30f), 2.f);
  f[6] = fminf(dn1 / (tn1 * r1 + 1e-30f), 4.f);
  f[7] = fminf(dn2 / (tn2 * r2 + 1e-30f), 4.f);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float *d, const uint32_t *a, const uint32_t *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Warp-wide MLP over 32 candidates (lane l holds candidate l's features in
// f[0..7]); returns the prediction of the calling lane's candidate. Layers 1
// and 2 run on the tensor cores (mma.sync m16n8k16, BF16 operands, FP32
// accumulation): the warp's batch is 32 x 8 -> 64 -> 64, far too small for a
// TMEM-based tcgen05 pipeline inside a warp-independent traversal. The C
// fragments of layer 1 are repacked in registers as layer 2's A fragments;
// layer 3 (64 -> 1) is folded into layer 2's epilogue with FP32 FMAs and a
// 4-lane reduction. W lives in shared memory.
static __device__ __noinline__ float mlp_warp_predict(const MlpFrag &W, const float *f) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float y[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // [m-tile][row g, row g + 8]
  for (int m = 0; m < 2; ++m) {
    // Layer 1 A fragment: rows g and g + 8 of m-tile m, features 2t and 2t + 1.
    const int r0 = 16 * m + g, r1 = r0 + 8;
    float p0 = 0.f, p1 = 0.f, q0 = 0.f, q1 = 0.f;
    for (int k = 0; k < 8; ++k) {
      const float x0 = __shfl_sync(0xffffffffu, f[k], r0), x1 = __shfl_sync(0xffffffffu, f[k], r1);
      if (k == 2 * t) {
        p0 = x0;
        q0 = x1;
      }
      if (k == 2 * t + 1) {
        p1 = x0;
        q1 = x1;
      }
    }
    const uint32_t a1[4] = {pack_bf16(p0, p1), pack_bf16(q0, q1), 0u, 0u};
    // Layer 1 -> layer 2 A fragments (k-tile kk = layer-1 n-tiles 2kk, 2kk+1).
    uint32_t a2[4][4];
    for (int kk = 0; kk < 4; ++kk) {
      float c[2][4];
      for (int h = 0; h < 2; ++h) {
        const int n = 2 * kk + h;
        const float bb0 = W.b1[8 * n + 2 * t], bb1 = W.b1[8 * n + 2 * t + 1];
        c[h][0] = bb0;
        c[h][1] = bb1;
        c[h][2] = bb0;
        c[h][3] = bb1;
        mma_bf16(c[h], a1, W.w1[n][lane]);
      }
      a2[kk][0] = pack_bf16(fmaxf(c[0][0], 0.f), fmaxf(c[0][1], 0.f));
      a2[kk][1] = pack_bf16(fmaxf(c[0][2], 0.f), fmaxf(c[0][3], 0.f));
      a2[kk][2] = pack_bf16(fmaxf(c[1][0], 0.f), fmaxf(c[1][1], 0.f));
      a2[kk][3] = pack_bf16(fmaxf(c[1][2], 0.f), fmaxf(c[1][3], 0.f));
    }
    // Layer 2 per n-tile, folded into layer 3.
    for (int n = 0; n < 8; ++n) {
      const float bb0 = W.b2[8 * n + 2 * t], bb1 = W.b2[8 * n + 2 * t + 1];
      float c[4] = {bb0, bb1, bb0, bb1};
      for (int kk = 0; kk < 4; ++kk) mma_bf16(c, a2[kk], W.w2[kk][n][lane]);
      const float w0 = W.w3f[8 * n + 2 * t], w1 = W.w3f[8 * n + 2 * t + 1];
      y[m][0] += fmaxf(c[0], 0.f) * w0 + fmaxf(c[1], 0.f) * w1;
      y[m][1] += fmaxf(c[2], 0.f) * w0 + fmaxf(c[3], 0.f) * w1;
    }
  }
  // Sum over the 4 lanes of a group: lane 4g' then holds rows g' and g' + 8.
  for (int o = 1; o < 4; o <<= 1)
    for (int m = 0; m < 2; ++m) {
      y[m][0] += __shfl_xor_sync(0xffffffffu, y[m][0], o);
      y[m][1] += __shfl_xor_sync(0xffffffffu, y[m][1], o);
    }
  // Candidate r = lane: m-tile r / 16, row r % 16 -> group (r % 8), half r % 16 >= 8.
  const int row = lane & 15, src = 4 * (row & 7);
  const float v00 = __shfl_sync(0xffffffffu, y[0][0], src), v01 = __shfl_sync(0xffffffffu, y[0][1], src);
  const float v10 = __shfl_sync(0xffffffffu, y[1][0], src), v11 = __shfl_sync(0xffffffffu, y[1][1], src);
  const float v = lane < 16 ? (row < 8 ? v00 : v01) : (row < 8 ? v10 : v11);
  return v + W.b3;
}

}  // namespace fln
