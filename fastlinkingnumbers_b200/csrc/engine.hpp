// Device side of the engine: context, device buffers and the launchers of
// the linking-number kernels (direct sum: direct.cu; Barnes–Hut: bh.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>
#include <string>
#include <vector>

#include "host.hpp"

namespace fln {

#define FLN_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::fln::Error(e_ == cudaErrorMemoryAllocation ? FLN_ERR_OUT_OF_MEMORY : FLN_ERR_CUDA, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));              \
  } while (0)

// Grow-only device buffer.
struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  void *need(size_t n) {
    if (n > bytes) {
      if (ptr) cudaFree(ptr);
      ptr = nullptr;
      bytes = 0;
      FLN_CUDA(cudaMalloc(&ptr, n));
      bytes = n;
    }
    return ptr;
  }
  template <class T>
  T *as(size_t count) {
    return static_cast<T *>(need(count * sizeof(T) + 16));
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
};

// Grow-only pinned host buffer (for the host-array entry points).
struct HostBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  void *need(size_t n) {
    if (n > bytes) {
      if (ptr) cudaFreeHost(ptr);
      ptr = nullptr;
      bytes = 0;
      FLN_CUDA(cudaMallocHost(&ptr, n));
      bytes = n;
    }
    return ptr;
  }
  ~HostBuf() {
    if (ptr) cudaFreeHost(ptr);
  }
};

// Direct-sum schedule: the pair list oriented and ordered for the kernel,
// and the work items (pair, block of kBlockSegs curve-1 segments).
struct DirectPlan {
  std::vector<int32_t> order;       // kernel slot -> caller pair index
  std::vector<int32_t> loops;       // 2 per slot: (curve-1 loop, curve-2 loop)
  std::vector<int64_t> item_start;  // slot -> first item; size nslots + 1
  int64_t items = 0;
  double segment_pairs = 0;
};

// Learned opening criterion of the Barnes–Hut traversal (learned.cuh has the
// weight layout; frag == nullptr: off).
struct MlpFrag;
struct LearnedCfg {
  const MlpFrag *frag;  // device copy of the packed BF16 weights
  float s_min;          // candidates: separation |dr| / (r1 + r2) at least this
  float log10_tau;      // accept when the predicted log10 error is below this (at beta0)
  int32_t min_cand;     // run the MLP only when a warp step has at least this many candidates
  int32_t min_seg;      // candidates: the smaller node holds at least this many segments
};

// Sampling of node pairs for training, during the first Barnes–Hut pass
// (rec == nullptr: off). Pairs are (slot, node 1, node 2, 0).
struct Recording {
  int4 *rec = nullptr;
  unsigned long long *count = nullptr;
  int64_t cap = 0;
  float s_min = 0.f;
  uint32_t keep = 0;  // keep a candidate when its 32-bit hash is below this
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  fln_stats stats{};
  // Device buffers.
  DevBuf d_xyz, d_off, d_pairs, d_loops, d_items, d_partial, d_counter, d_lk, d_err, d_flags, d_near;
  DevBuf d_bh[28];
  int64_t bh_front_hint = 0;  // frontier records of the largest Barnes–Hut first pass so far
  // CTAs per SM of the traversal kernels (per occupancy set), of the learned
  // traversal and of bh_classify; 0 until first queried.
  int bh_per_sm[3] = {0, 0, 0};
  int bh_per_sm_learned = 0, bh_per_sm_classify = 0;
  HostBuf h_in, h_out;  // pinned staging of copy_h2d / copy_d2h
  cudaEvent_t ev_stage[2] = {nullptr, nullptr};
  // The exact-list launches of the fused Barnes–Hut rounds run on their own
  // stream, beside the next round's traversal; ev_round holds an event pair
  // around each (grown on demand, kept for later calls).
  cudaStream_t exact_stream = nullptr;
  std::vector<cudaEvent_t> ev_round;
  // Vertices from host arrays arrive in pieces on a copy stream (split at
  // loop boundaries); the Barnes–Hut tree build of each piece's loops waits
  // only for its piece. xyz_pieces = 0: the vertices are resident.
  static constexpr int kXyzPieces = 8;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_piece[kXyzPieces] = {};
  cudaEvent_t ev_before_copy = nullptr;
  int64_t xyz_piece_end[kXyzPieces] = {};  // vertex index at which each piece ends
  int xyz_pieces = 0;
  // Learned criterion in use on this context, and training buffers.
  DevBuf d_mlp, d_learn[8];
  // Device Discretize (discretize.cu).
  DevBuf d_disc[37];
  LearnedCfg learned{nullptr, 0.f, 0.f, 0};
  Recording recording;

  explicit Context(int dev, void *user_stream);
  // Device time between two events recorded around launches on `stream`.
  float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~Context();
};

// The context's stream waits for every piece of the vertices still on its
// way (Context::xyz_pieces); afterwards they are resident.
inline void wait_xyz_pieces(Context &c) {
  for (int i = 0; i < c.xyz_pieces; ++i) cudaStreamWaitEvent(c.stream, c.ev_piece[i], 0);
  c.xyz_pieces = 0;
}

// Resident CTAs per SM of `kernel` at `block` threads (at least 1), asked of
// the driver once per kernel and block size: the library is built for one
// architecture, and a driver query on every call costs host time while the
// GPU waits.
inline int occupancy_of(const void *kernel, int block) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(kernel, block);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, 0) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return cache[key] = std::max(n, 1);
}

// Mixed direct sum: a segment pair whose closest endpoint distance is below
// this multiple of the longer segment's length is evaluated in FP64 (the
// default of fln_params.near_factor, and the factor of the allocation-free
// entry point).
constexpr double kDefaultNearFactor = 4.0;
// Barnes–Hut round budget (traversal steps a warp spends on a batch per
// launch) when fln_params.bh_budget is 0: on the polymer step with the exact
// list, 128 ran the traversal in 48.0 ms against 49.6 ms at 256.
constexpr int kDefaultBhBudget = 128;

// Plans and runs the direct sum over `npairs` pairs of the loops in device
// memory. d_xyz/d_off describe the loops; h_off is the host copy of the
// offsets; h_pairs the host copy of the pairs. Writes lk (per caller pair) to
// d_lk_out. Returns the number of kernel launches.
// tile_shape: index into the direct sum's tile shapes (fln_params.direct_tile).
constexpr int kDirectTileShapes = 6;
int direct_sum_device(Context &ctx, const double *d_xyz, const int64_t *d_off, const std::vector<int64_t> &h_off,
                      const std::vector<int32_t> &h_pairs, int precision, double near_factor, double *d_lk_out,
                      double *near_terms_out, int tile_shape = 0);

// Barnes–Hut over the same inputs; err per pair after ERROR_EST_SCALE and the
// reference's beta retry; flags gets FLN_PAIR_BETA_RETRIED. Returns launches.
int barnes_hut_device(Context &ctx, const double *d_xyz, const int64_t *d_off, const std::vector<int64_t> &h_off,
                      const std::vector<int32_t> &h_pairs, const fln_params &prm, double *d_lk_out,
                      double *d_err_out, int32_t *d_flags_out);

// Runs the Barnes–Hut stage (curve-order trees, beta0, learned criterion off)
// while sampling node pairs with separation in [s_min, 1.25 beta0] (opened
// pairs and far-field pairs near the threshold; a fraction `keep` of them by
// a hash of (pair, node, node), lowered and rerun until at most `cap` are
// recorded), then computes for each sample its features (learned.cuh) and
// the log10 of the true far-field error: |multipole value - FP64 exact sum
// over the two nodes' segment ranges| + 1e-14. Samples whose ranges hold more
// than max_terms segment pairs are dropped. X gets 8 floats per sample, T the
// target, S the separation, E log10 of the Eq. 14 estimate x err_scale (the
// reference's error measure for the same pair).
void learned_collect(Context &ctx, const double *d_xyz, const int64_t *d_off, const std::vector<int64_t> &h_off,
                     const std::vector<int32_t> &h_pairs, const fln_params &prm, float s_min, double keep,
                     int64_t cap, int64_t max_terms, std::vector<float> &X, std::vector<float> &T,
                     std::vector<float> &S, std::vector<float> &E, int64_t *recorded);

// Training of the MLP on (X, T): pinball loss at quantile q, Adam, our own
// kernels (learned.cu), on the rows idx_train. params holds kMlpParams FP32
// values (initialised by the caller) and is updated; returns the mean loss of
// the last epoch.
struct TrainOptions {
  int epochs = 40;
  int batch = 4096;
  float lr = 2e-3f;
  float quantile = 0.9f;
  uint64_t seed = 1;
};
double learned_train(Context &ctx, const std::vector<float> &X, const std::vector<float> &T,
                     const std::vector<int32_t> &idx_train, const TrainOptions &opt, std::vector<float> &params);
// FP32 (mma = 0) or BF16 warp-MMA (mma = 1, the traversal's path) predictions.
void learned_predict(Context &ctx, const float *params, const float *X, int64_t n, int mma, float *Y);
// Mean pinball loss and its gradient (d loss / d params) at params.
double learned_gradients(Context &ctx, const float *params, const float *X, const float *T, int64_t n, float q,
                         float *grad);
// Discretize (discretize.cpp:103-281) and the potential-link searches before
// and after it, on the GPU: the same closed polylines (CSR offsets, xyz) and
// sorted unique pairs (i < j) as the host path, bit for bit; rounds = the
// refinement rounds run. Throws Error on the reference's failure conditions.
// bcc_f32: the same control points as float32 (curves in order, 3 per
// point), or nullptr; when given they are uploaded as such and widened on the
// device (the same doubles, half the copy).
void discretize_device(Context &ctx, const std::vector<CurveData> &curves, const float *bcc_f32,
                       std::vector<int64_t> &offsets, DoubleArray &xyz, std::vector<int32_t> &pairs, int32_t &rounds);

// Host<->device copies on ctx.stream that return when the data has arrived.
// Pinned host memory is copied directly; pageable memory goes in 64 MB
// chunks through two pinned buffers, the host side by all threads (a single
// pageable DMA copy runs at a few GB/s, slower still into fresh pages).
void copy_h2d(Context &ctx, void *d_dst, const void *h_src, size_t bytes);
void copy_d2h(Context &ctx, void *h_dst, const void *d_src, size_t bytes);
// memcpy by all host threads.
void parallel_memcpy(void *dst, const void *src, size_t bytes);

// Packs params into the context's device weights and enables the criterion.
void learned_enable(Context &ctx, const float *params, float s_min, float log10_tau, int32_t min_cand,
                    int32_t min_seg);

}  // namespace fln
