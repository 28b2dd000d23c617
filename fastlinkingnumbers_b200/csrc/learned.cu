// Learned opening criterion: training, inference checks and packing.
//
// Training data (bh.cu, learned_collect). While the Barnes–Hut traversal runs
// in recording mode it samples node pairs with separation s = |dr| / (r1 +
// r2) in [s_min, 1.25 beta] (pairs it opens and far-field pairs near the beta
// threshold). Each sample gets the 8 features of learned.cuh and the true
// far-field error: |multipole value - exact sum|, the exact sum being the
// FP64 sum over the two nodes' segment ranges (in a curve-order tree a node
// is a contiguous segment range). Target: log10(error + 1e-14).
//
// Training. Our own kernels: `mlp_train_step` runs forward and backward of a
// mini-batch (one sample per thread, parameters and activations in shared
// memory) with the pinball loss at quantile q (a conservative, upper-
// quantile regression of the log error) and accumulates the gradient;
// `mlp_adam` applies Adam. `mlp_pack` converts the FP32 master weights into
// the BF16 mma.sync fragments the traversal uses.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <vector>

#include "engine.hpp"
#include "learned.cuh"

namespace fln {

namespace learned {

constexpr int kTrainBlock = 128;

// Forward + backward of one mini-batch; pinball loss at quantile q on
// y = prediction, t = target. One sample per thread; activations and
// per-sample gradients in (dynamic) shared memory; each CTA adds its
// parameter gradient of d(mean loss)/d(params) into grad and its loss share
// into loss.
constexpr int kLd = kMlpHidden + 1;  // padded row (no bank conflicts)
constexpr size_t kTrainSmem = sizeof(float) * (kMlpParams + kTrainBlock * (kMlpIn + 4 * kLd + 1));

__global__ void __launch_bounds__(kTrainBlock) mlp_train_step(const float *params, const float *X, const float *T,
                                                              const int32_t *idx, int64_t nbatch, float q,
                                                              float *grad, float *loss) {
  extern __shared__ float smem[];
  float *sp = smem;                          // parameters
  float *sx = sp + kMlpParams;               // [B][8]
  float *sh1 = sx + kTrainBlock * kMlpIn;    // [B][kLd] layer-1 activations
  float *sh2 = sh1 + kTrainBlock * kLd;      // [B][kLd] layer-2 activations
  float *sd2 = sh2 + kTrainBlock * kLd;      // [B][kLd] dL/d(pre-activation 2)
  float *sd1 = sd2 + kTrainBlock * kLd;      // [B][kLd] dL/d(pre-activation 1)
  float *sdy = sd1 + kTrainBlock * kLd;      // [B]
  for (int p = threadIdx.x; p < kMlpParams; p += blockDim.x) sp[p] = params[p];
  __syncthreads();
  const int me = threadIdx.x;
  const int64_t b = (int64_t)blockIdx.x * kTrainBlock + me;
  const bool act = b < nbatch;
  const int64_t row = act ? idx[b] : 0;
  for (int i = 0; i < kMlpIn; ++i) sx[me * kMlpIn + i] = act ? X[row * kMlpIn + i] : 0.f;
  for (int j = 0; j < kMlpHidden; ++j) {
    float a = sp[kMlpB1 + j];
    for (int i = 0; i < kMlpIn; ++i) a += sx[me * kMlpIn + i] * sp[kMlpW1 + i * kMlpHidden + j];
    sh1[me * kLd + j] = fmaxf(a, 0.f);
  }
  float y = sp[kMlpB3];
  for (int k = 0; k < kMlpHidden; ++k) {
    float a = sp[kMlpB2 + k];
    for (int j = 0; j < kMlpHidden; ++j) a += sh1[me * kLd + j] * sp[kMlpW2 + j * kMlpHidden + k];
    const float h = fmaxf(a, 0.f);
    sh2[me * kLd + k] = h;
    y += h * sp[kMlpW3 + k];
  }
  const float inv_n = 1.f / (float)nbatch;
  float dy = 0.f;
  if (act) {
    const float e = T[row] - y;
    atomicAdd(loss, (e >= 0.f ? q * e : (q - 1.f) * e) * inv_n);
    dy = (e > 0.f ? -q : (1.f - q)) * inv_n;
  }
  sdy[me] = dy;
  for (int k = 0; k < kMlpHidden; ++k) sd2[me * kLd + k] = sh2[me * kLd + k] > 0.f ? dy * sp[kMlpW3 + k] : 0.f;
  for (int j = 0; j < kMlpHidden; ++j) {
    float a = 0.f;
    if (sh1[me * kLd + j] > 0.f)
      for (int k = 0; k < kMlpHidden; ++k) a += sd2[me * kLd + k] * sp[kMlpW2 + j * kMlpHidden + k];
    sd1[me * kLd + j] = a;
  }
  __syncthreads();
  // Parameter gradients: threads split the parameters and sum over samples.
  for (int p = me; p < kMlpParams; p += blockDim.x) {
    float a = 0.f;
    if (p < kMlpB1) {  // W1[i][j]
      const int i = p / kMlpHidden, j = p % kMlpHidden;
      for (int s = 0; s < kTrainBlock; ++s) a += sx[s * kMlpIn + i] * sd1[s * kLd + j];
    } else if (p < kMlpW2) {  // b1[j]
      const int j = p - kMlpB1;
      for (int s = 0; s < kTrainBlock; ++s) a += sd1[s * kLd + j];
    } else if (p < kMlpB2) {  // W2[j][k]
      const int j = (p - kMlpW2) / kMlpHidden, k = (p - kMlpW2) % kMlpHidden;
      for (int s = 0; s < kTrainBlock; ++s) a += sh1[s * kLd + j] * sd2[s * kLd + k];
    } else if (p < kMlpW3) {  // b2[k]
      const int k = p - kMlpB2;
      for (int s = 0; s < kTrainBlock; ++s) a += sd2[s * kLd + k];
    } else if (p < kMlpB3) {  // w3[k]
      const int k = p - kMlpW3;
      for (int s = 0; s < kTrainBlock; ++s) a += sdy[s] * sh2[s * kLd + k];
    } else {  // b3
      for (int s = 0; s < kTrainBlock; ++s) a += sdy[s];
    }
    if (a != 0.f) atomicAdd(&grad[p], a);
  }
}

// Adam (Kingma & Ba 2015) with bias correction; clears the gradient.
__global__ void mlp_adam(float *params, float *grad, float *m, float *v, int step, float lr, float b1, float b2,
                         float eps) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpParams) return;
  const float g = grad[p];
  m[p] = b1 * m[p] + (1.f - b1) * g;
  v[p] = b2 * v[p] + (1.f - b2) * g * g;
  const float mh = m[p] / (1.f - powf(b1, (float)step)), vh = v[p] / (1.f - powf(b2, (float)step));
  params[p] -= lr * mh / (sqrtf(vh) + eps);
  grad[p] = 0.f;
}

// FP32 forward (evaluation and the gradient check).
__global__ void mlp_predict(const float *params, const float *X, int64_t n, float *Y) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float h1[kMlpHidden];
  for (int j = 0; j < kMlpHidden; ++j) {
    float a = params[kMlpB1 + j];
    for (int i = 0; i < kMlpIn; ++i) a += X[s * kMlpIn + i] * params[kMlpW1 + i * kMlpHidden + j];
    h1[j] = fmaxf(a, 0.f);
  }
  float y = params[kMlpB3];
  for (int k = 0; k < kMlpHidden; ++k) {
    float a = params[kMlpB2 + k];
    for (int j = 0; j < kMlpHidden; ++j) a += h1[j] * params[kMlpW2 + j * kMlpHidden + k];
    y += fmaxf(a, 0.f) * params[kMlpW3 + k];
  }
  Y[s] = y;
}

// BF16 mma.sync B fragments from the FP32 master weights.
__global__ void mlp_pack(const float *P, MlpFrag *F) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  for (int n = 0; n < 8; ++n) {
    const int col = 8 * n + g;
    F->w1[n][lane][0] = pack_bf16(P[kMlpW1 + (2 * t) * kMlpHidden + col], P[kMlpW1 + (2 * t + 1) * kMlpHidden + col]);
    F->w1[n][lane][1] = 0u;  // input rows 8..15 are padding
  }
  for (int kk = 0; kk < 4; ++kk)
    for (int n = 0; n < 8; ++n) {
      const int col = 8 * n + g, r = 16 * kk + 2 * t;
      F->w2[kk][n][lane][0] = pack_bf16(P[kMlpW2 + r * kMlpHidden + col], P[kMlpW2 + (r + 1) * kMlpHidden + col]);
      F->w2[kk][n][lane][1] =
          pack_bf16(P[kMlpW2 + (r + 8) * kMlpHidden + col], P[kMlpW2 + (r + 9) * kMlpHidden + col]);
    }
  for (int j = lane; j < kMlpHidden; j += 32) F->w3f[j] = __bfloat162float(__float2bfloat16_rn(P[kMlpW3 + j]));
  for (int j = lane; j < kMlpHidden; j += 32) {
    F->b1[j] = P[kMlpB1 + j];
    F->b2[j] = P[kMlpB2 + j];
  }
  if (lane == 0) F->b3 = P[kMlpB3];
}

// Batched warp MLP inference: the traversal's BF16 fragment path, 32 samples
// per warp.
__global__ void mlp_predict_mma(const MlpFrag *W, const float *X, int64_t n, float *Y) {
  __shared__ MlpFrag s;
  const uint32_t *src = reinterpret_cast<const uint32_t *>(W);
  uint32_t *dst = reinterpret_cast<uint32_t *>(&s);
  for (int x = threadIdx.x; x < (int)(sizeof(MlpFrag) / 4); x += blockDim.x) dst[x] = src[x];
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float f[kMlpIn];
  for (int k = 0; k < kMlpIn; ++k) f[k] = i < n ? X[i * kMlpIn + k] : 0.f;
  const float y = mlp_warp_predict(s, f);
  if (i < n) Y[i] = y;
}

}  // namespace learned

using namespace learned;

static void upload(Context &ctx, DevBuf &b, const void *src, size_t bytes) {
  void *d = b.need(bytes + 16);
  FLN_CUDA(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, ctx.stream));
}

static MlpFrag *pack_device(Context &ctx, const float *d_params) {
  MlpFrag *F = static_cast<MlpFrag *>(ctx.d_mlp.need(sizeof(MlpFrag)));
  mlp_pack<<<1, 32, 0, ctx.stream>>>(d_params, F);
  FLN_CUDA(cudaGetLastError());
  return F;
}

double learned_train(Context &ctx, const std::vector<float> &X, const std::vector<float> &T,
                     const std::vector<int32_t> &idx_train, const TrainOptions &opt, std::vector<float> &params) {
  const int64_t n = (int64_t)idx_train.size();
  if (n == 0) return 0.0;
  if ((int64_t)params.size() != kMlpParams) throw Error(FLN_ERR_INVALID_ARGUMENT, "MLP parameter count");
  cudaStream_t st = ctx.stream;
  upload(ctx, ctx.d_learn[3], X.data(), X.size() * sizeof(float));
  upload(ctx, ctx.d_learn[5], T.data(), T.size() * sizeof(float));
  const float *d_X = static_cast<const float *>(ctx.d_learn[3].ptr);
  const float *d_T = static_cast<const float *>(ctx.d_learn[5].ptr);
  // params | grad | m | v | loss
  float *d_p = ctx.d_learn[7].as<float>(4 * kMlpParams + 4);
  float *d_g = d_p + kMlpParams, *d_m = d_g + kMlpParams, *d_v = d_m + kMlpParams, *d_loss = d_v + kMlpParams;
  FLN_CUDA(cudaMemcpyAsync(d_p, params.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemsetAsync(d_g, 0, (3 * kMlpParams + 4) * sizeof(float), st));
  int32_t *d_idx = ctx.d_learn[6].as<int32_t>(n);
  FLN_CUDA(cudaFuncSetAttribute(mlp_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
  std::mt19937_64 rng(opt.seed);
  std::vector<int32_t> perm(idx_train);
  const int batch = std::max(kTrainBlock, opt.batch);
  const int64_t steps_per_epoch = (n + batch - 1) / batch;
  const int64_t total_steps = steps_per_epoch * std::max(1, opt.epochs);
  int step = 0;
  for (int ep = 0; ep < std::max(1, opt.epochs); ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    // perm must stay alive until the copy has run: it is reshuffled only after the sync below.
    FLN_CUDA(cudaMemcpyAsync(d_idx, perm.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    for (int64_t b0 = 0; b0 < n; b0 += batch) {
      const int64_t nb = std::min<int64_t>(batch, n - b0);
      FLN_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(float), st));
      mlp_train_step<<<(int)((nb + kTrainBlock - 1) / kTrainBlock), kTrainBlock, kTrainSmem, st>>>(
          d_p, d_X, d_T, d_idx + b0, nb, opt.quantile, d_g, d_loss);
      ++step;
      // Cosine decay of the step size.
      const float lr = (float)(opt.lr * 0.5 * (1.0 + std::cos(3.141592653589793 * (double)(step - 1) / total_steps)));
      mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(d_p, d_g, d_m, d_v, step, lr, 0.9f, 0.999f, 1e-7f);
      FLN_CUDA(cudaGetLastError());
    }
    FLN_CUDA(cudaStreamSynchronize(st));
  }
  // Mean loss over the training rows at the final parameters (chunks of up
  // to 2^20 rows, each launch averaging over its chunk).
  double total = 0.0;
  for (int64_t b0 = 0; b0 < n; b0 += (int64_t)1 << 20) {
    const int64_t nb = std::min<int64_t>((int64_t)1 << 20, n - b0);
    FLN_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(float), st));
    mlp_train_step<<<(int)((nb + kTrainBlock - 1) / kTrainBlock), kTrainBlock, kTrainSmem, st>>>(
        d_p, d_X, d_T, d_idx + b0, nb, opt.quantile, d_g, d_loss);
    FLN_CUDA(cudaGetLastError());
    float l = 0.f;
    FLN_CUDA(cudaMemcpyAsync(&l, d_loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaStreamSynchronize(st));
    total += (double)l * (double)nb / (double)n;
  }
  FLN_CUDA(cudaMemcpyAsync(params.data(), d_p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaStreamSynchronize(st));
  return total;
}

void learned_predict(Context &ctx, const float *params, const float *X, int64_t n, int mma, float *Y) {
  if (n <= 0) return;
  cudaStream_t st = ctx.stream;
  float *d_p = ctx.d_learn[7].as<float>(4 * kMlpParams + 4);
  FLN_CUDA(cudaMemcpyAsync(d_p, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, st));
  upload(ctx, ctx.d_learn[3], X, (size_t)n * kMlpIn * sizeof(float));
  float *d_Y = ctx.d_learn[5].as<float>(n);
  const float *d_X = static_cast<const float *>(ctx.d_learn[3].ptr);
  if (mma) {
    MlpFrag *F = static_cast<MlpFrag *>(ctx.d_learn[4].need(sizeof(MlpFrag)));
    mlp_pack<<<1, 32, 0, st>>>(d_p, F);
    mlp_predict_mma<<<(int)((n + 127) / 128), 128, 0, st>>>(F, d_X, n, d_Y);
  } else {
    mlp_predict<<<(int)((n + 127) / 128), 128, 0, st>>>(d_p, d_X, n, d_Y);
  }
  FLN_CUDA(cudaGetLastError());
  FLN_CUDA(cudaMemcpyAsync(Y, d_Y, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaStreamSynchronize(st));
}

double learned_gradients(Context &ctx, const float *params, const float *X, const float *T, int64_t n, float q,
                         float *grad) {
  if (n <= 0 || n > ((int64_t)1 << 24)) throw Error(FLN_ERR_INVALID_ARGUMENT, "gradient batch size");
  cudaStream_t st = ctx.stream;
  float *d_p = ctx.d_learn[7].as<float>(4 * kMlpParams + 4);
  float *d_g = d_p + kMlpParams, *d_loss = d_p + 4 * kMlpParams;
  FLN_CUDA(cudaMemcpyAsync(d_p, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemsetAsync(d_g, 0, kMlpParams * sizeof(float), st));
  FLN_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(float), st));
  upload(ctx, ctx.d_learn[3], X, (size_t)n * kMlpIn * sizeof(float));
  upload(ctx, ctx.d_learn[5], T, (size_t)n * sizeof(float));
  std::vector<int32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  int32_t *d_idx = ctx.d_learn[6].as<int32_t>(n);
  FLN_CUDA(cudaMemcpyAsync(d_idx, idx.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaFuncSetAttribute(mlp_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
  mlp_train_step<<<(int)((n + kTrainBlock - 1) / kTrainBlock), kTrainBlock, kTrainSmem, st>>>(
      d_p, static_cast<const float *>(ctx.d_learn[3].ptr), static_cast<const float *>(ctx.d_learn[5].ptr), d_idx, n,
      q, d_g, d_loss);
  FLN_CUDA(cudaGetLastError());
  float loss = 0.f;
  FLN_CUDA(cudaMemcpyAsync(grad, d_g, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaMemcpyAsync(&loss, d_loss, sizeof(float), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaStreamSynchronize(st));
  return loss;
}

void learned_enable(Context &ctx, const float *params, float s_min, float log10_tau, int32_t min_cand,
                    int32_t min_seg) {
  if (!params) {
    ctx.learned = LearnedCfg{nullptr, 0.f, 0.f, 0, 0};
    return;
  }
  float *d_p = ctx.d_learn[7].as<float>(4 * kMlpParams + 4);
  FLN_CUDA(cudaMemcpyAsync(d_p, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, ctx.stream));
  MlpFrag *F = pack_device(ctx, d_p);
  FLN_CUDA(cudaStreamSynchronize(ctx.stream));
  ctx.learned = LearnedCfg{F, s_min, log10_tau, std::max<int32_t>(1, min_cand), std::max<int32_t>(0, min_seg)};
}

}  // namespace fln
