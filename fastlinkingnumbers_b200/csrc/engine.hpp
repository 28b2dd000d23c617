// Device side of the engine: context, device buffers and the launchers of
// the linking-number kernels (direct sum: direct.cu; Barnes–Hut: bh.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
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

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  fln_stats stats{};
  // Device buffers.
  DevBuf d_xyz, d_off, d_pairs, d_loops, d_items, d_partial, d_counter, d_lk, d_err, d_flags, d_near;
  DevBuf d_bh[24];
  HostBuf h_in, h_out;

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

// Plans and runs the direct sum over `npairs` pairs of the loops in device
// memory. d_xyz/d_off describe the loops; h_off is the host copy of the
// offsets; h_pairs the host copy of the pairs. Writes lk (per caller pair) to
// d_lk_out. Returns the number of kernel launches.
int direct_sum_device(Context &ctx, const double *d_xyz, const int64_t *d_off, const std::vector<int64_t> &h_off,
                      const std::vector<int32_t> &h_pairs, int precision, double near_factor, double *d_lk_out,
                      double *near_terms_out);

// Barnes–Hut over the same inputs; err per pair after ERROR_EST_SCALE and the
// reference's beta retry; flags gets FLN_PAIR_BETA_RETRIED. Returns launches.
int barnes_hut_device(Context &ctx, const double *d_xyz, const int64_t *d_off, const std::vector<int64_t> &h_off,
                      const std::vector<int32_t> &h_pairs, const fln_params &prm, double *d_lk_out,
                      double *d_err_out, int32_t *d_flags_out);

}  // namespace fln
