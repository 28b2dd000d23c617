// The C ABI of include/fln.h: argument checks, host<->device staging, the
// FP64 recompute of low-margin pairs, certificates. No exception crosses it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "engine.hpp"

namespace fln {

Context::Context(int dev, void *user_stream) : device(dev) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw Error(FLN_ERR_NO_DEVICE, "No CUDA device is visible.");
  if (dev < 0 || dev >= n) throw Error(FLN_ERR_INVALID_ARGUMENT, "Device index out of range.");
  FLN_CUDA(cudaSetDevice(dev));
  FLN_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
  if (user_stream) {
    stream = static_cast<cudaStream_t>(user_stream);
  } else {
    FLN_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own_stream = true;
  }
  FLN_CUDA(cudaEventCreate(&ev0));
  FLN_CUDA(cudaEventCreate(&ev1));
  FLN_CUDA(cudaEventCreate(&ev2));
  FLN_CUDA(cudaEventCreate(&ev3));
}

Context::~Context() {
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  if (exact_stream) cudaStreamSynchronize(exact_stream);
  if (copy_stream) cudaStreamSynchronize(copy_stream);
  for (DevBuf *b : {&d_xyz, &d_off, &d_pairs, &d_loops, &d_items, &d_partial, &d_counter, &d_lk, &d_err, &d_flags,
                    &d_near})
    b->release();
  for (auto &b : d_bh) b.release();
  d_mlp.release();
  for (auto &b : d_learn) b.release();
  for (auto &b : d_disc) b.release();
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (ev2) cudaEventDestroy(ev2);
  if (ev3) cudaEventDestroy(ev3);
  for (cudaEvent_t e : ev_stage)
    if (e) cudaEventDestroy(e);
  if (exact_stream) cudaStreamDestroy(exact_stream);
  for (cudaEvent_t e : ev_round)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ev_piece)
    if (e) cudaEventDestroy(e);
  if (ev_before_copy) cudaEventDestroy(ev_before_copy);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

void parallel_memcpy(void *dst, const void *src, size_t bytes) {
  const size_t kBlock = size_t(1) << 20;
  const int64_t nb = (int64_t)((bytes + kBlock - 1) / kBlock);
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nb; ++b) {
    const size_t o = (size_t)b * kBlock;
    std::memcpy(static_cast<char *>(dst) + o, static_cast<const char *>(src) + o, std::min(kBlock, bytes - o));
  }
}

static bool is_pinned(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

static constexpr size_t kStage = size_t(64) << 20;

static void stage_setup(Context &ctx) {
  ctx.h_in.need(kStage);
  ctx.h_out.need(kStage);
  for (cudaEvent_t &e : ctx.ev_stage)
    if (!e) FLN_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

void copy_h2d(Context &ctx, void *d_dst, const void *h_src, size_t bytes) {
  if (bytes == 0) return;
  if (bytes <= kStage / 4 || is_pinned(h_src)) {
    FLN_CUDA(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, ctx.stream));
    FLN_CUDA(cudaStreamSynchronize(ctx.stream));
    return;
  }
  stage_setup(ctx);
  void *stage[2] = {ctx.h_in.ptr, ctx.h_out.ptr};
  for (size_t o = 0, k = 0; o < bytes; o += kStage, ++k) {
    const size_t len = std::min(kStage, bytes - o);
    FLN_CUDA(cudaEventSynchronize(ctx.ev_stage[k & 1]));  // the copy that last used this buffer is done
    parallel_memcpy(stage[k & 1], static_cast<const char *>(h_src) + o, len);
    FLN_CUDA(cudaMemcpyAsync(static_cast<char *>(d_dst) + o, stage[k & 1], len, cudaMemcpyHostToDevice, ctx.stream));
    FLN_CUDA(cudaEventRecord(ctx.ev_stage[k & 1], ctx.stream));
  }
  FLN_CUDA(cudaStreamSynchronize(ctx.stream));
}

void copy_d2h(Context &ctx, void *h_dst, const void *d_src, size_t bytes) {
  if (bytes == 0) return;
  if (bytes <= kStage / 4 || is_pinned(h_dst)) {
    FLN_CUDA(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, ctx.stream));
    FLN_CUDA(cudaStreamSynchronize(ctx.stream));
    return;
  }
  stage_setup(ctx);
  void *stage[2] = {ctx.h_in.ptr, ctx.h_out.ptr};
  const size_t nchunks = (bytes + kStage - 1) / kStage;
  for (size_t k = 0; k <= nchunks; ++k) {
    if (k < nchunks) {
      const size_t o = k * kStage, len = std::min(kStage, bytes - o);
      FLN_CUDA(cudaMemcpyAsync(stage[k & 1], static_cast<const char *>(d_src) + o, len, cudaMemcpyDeviceToHost,
                               ctx.stream));
      FLN_CUDA(cudaEventRecord(ctx.ev_stage[k & 1], ctx.stream));
    }
    if (k > 0) {
      const size_t j = k - 1, o = j * kStage, len = std::min(kStage, bytes - o);
      FLN_CUDA(cudaEventSynchronize(ctx.ev_stage[j & 1]));
      parallel_memcpy(static_cast<char *>(h_dst) + o, stage[j & 1], len);
    }
  }
}

// Scatters src[k] into dst[idx[k]] for the FP64 recompute (defined in bh.cu).
void scatter_doubles(Context &ctx, const double *src, const int32_t *idx, int64_t n, double *dst);

// Runs the requested method over device-resident loops and pairs, then the
// margin check and FP64 direct-sum recompute of the pairs that fail it.
static int run_pairs(Context &ctx, const double *d_xyz, const int64_t *d_off, const std::vector<int64_t> &h_off,
                     const std::vector<int32_t> &h_pairs, fln_method method, const fln_params &prm,
                     double *d_lk, double *d_err, int32_t *d_flags) {
  const int64_t np = (int64_t)h_pairs.size() / 2;
  int launches = 0;
  double near_terms = 0;
  ctx.stats.ms_main_kernel = 0;
  ctx.stats.ms_tree_build = 0;
  ctx.stats.bh_far_evals = ctx.stats.bh_leaf_evals = 0;
  ctx.stats.ms_exact = ctx.stats.bh_exact_entries = ctx.stats.ms_traverse = 0;
  ctx.stats.ms_retry = 0;
  ctx.stats.bh_front_records = ctx.stats.bh_retry_from_roots = 0;
  ctx.stats.bh_wait_timeouts = 0;
  ctx.stats.bh_far_reused = ctx.stats.bh_far_subtracted = 0;
  ctx.stats.beta_retried = 0;
  ctx.stats.bh_escalated = 0;
  if (!d_err) d_err = ctx.d_err.as<double>(std::max<int64_t>(np, 1));  // Barnes–Hut needs one
  if (method == FLN_METHOD_DIRECTSUM) {
    launches += direct_sum_device(ctx, d_xyz, d_off, h_off, h_pairs, prm.precision, prm.near_factor, d_lk,
                                  prm.precision == FLN_PREC_MIXED ? &near_terms : nullptr, prm.direct_tile);
    if (d_err) FLN_CUDA(cudaMemsetAsync(d_err, 0, np * sizeof(double), ctx.stream));
    if (d_flags) FLN_CUDA(cudaMemsetAsync(d_flags, 0, np * sizeof(int32_t), ctx.stream));
  } else {
    launches += barnes_hut_device(ctx, d_xyz, d_off, h_off, h_pairs, prm, d_lk, d_err, d_flags);
  }
  ctx.stats.near_fp64_terms = near_terms;
  const bool checked = !(method == FLN_METHOD_DIRECTSUM && prm.precision == FLN_PREC_FP64);
  ctx.stats.fp64_recomputed = 0;
  if (checked && np > 0) {
    std::vector<double> lk(np), err(np, 0.0);
    FLN_CUDA(cudaMemcpyAsync(lk.data(), d_lk, np * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    if (d_err) FLN_CUDA(cudaMemcpyAsync(err.data(), d_err, np * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    FLN_CUDA(cudaStreamSynchronize(ctx.stream));
    std::vector<int32_t> redo_idx, redo_pairs;
    for (int64_t p = 0; p < np; ++p) {
      const double r = std::round(lk[p]);
      const double margin = 0.5 - std::fabs(lk[p] - r);
      // Low margin, non-finite, or a Barnes–Hut error estimate that could
      // reach the rounding boundary: recompute in FP64 direct sum.
      if (!(margin >= prm.fp64_margin) || (method == FLN_METHOD_BARNESHUT && !(err[p] <= prm.bh_err_limit))) {
        redo_idx.push_back((int32_t)p);
        redo_pairs.push_back(h_pairs[2 * p]);
        redo_pairs.push_back(h_pairs[2 * p + 1]);
      }
    }
    if (!redo_idx.empty()) {
      const int64_t nr = (int64_t)redo_idx.size();
      double *d_tmp = ctx.d_near.as<double>(nr + nr / 2 + 2);
      int32_t *d_idx = reinterpret_cast<int32_t *>(d_tmp + nr);
      launches += direct_sum_device(ctx, d_xyz, d_off, h_off, redo_pairs, FLN_PREC_FP64, 0.0, d_tmp, nullptr);
      FLN_CUDA(cudaMemcpyAsync(d_idx, redo_idx.data(), nr * sizeof(int32_t), cudaMemcpyHostToDevice, ctx.stream));
      scatter_doubles(ctx, d_tmp, d_idx, nr, d_lk);
      ++launches;
      if (d_flags) {
        std::vector<int32_t> fl(np, 0);
        FLN_CUDA(cudaMemcpyAsync(fl.data(), d_flags, np * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
        FLN_CUDA(cudaStreamSynchronize(ctx.stream));
        for (int32_t p : redo_idx) fl[p] |= FLN_PAIR_FP64_RECOMPUTED;
        FLN_CUDA(cudaMemcpyAsync(d_flags, fl.data(), np * sizeof(int32_t), cudaMemcpyHostToDevice, ctx.stream));
      }
      ctx.stats.fp64_recomputed = nr;
    }
  }
  double sp = 0;
  for (int64_t p = 0; p < np; ++p)
    sp += (double)(h_off[h_pairs[2 * p] + 1] - h_off[h_pairs[2 * p]]) *
          (double)(h_off[h_pairs[2 * p + 1] + 1] - h_off[h_pairs[2 * p + 1]]);
  ctx.stats.segment_pairs = sp;
  ctx.stats.pairs = np;
  return launches;
}

static void check_inputs(const std::vector<int64_t> &h_off, int32_t nloops, const std::vector<int32_t> &h_pairs) {
  if (h_off.size() != (size_t)nloops + 1 || h_off[0] != 0)
    throw Error(FLN_ERR_INVALID_ARGUMENT, "loop_offsets must start at 0 and hold nloops + 1 entries.");
  for (int32_t l = 0; l < nloops; ++l)
    if (h_off[l + 1] < h_off[l]) throw Error(FLN_ERR_INVALID_ARGUMENT, "loop_offsets must be non-decreasing.");
  for (size_t k = 0; k < h_pairs.size(); ++k) {
    const int32_t l = h_pairs[k];
    if (l < 0 || l >= nloops) throw Error(FLN_ERR_INVALID_ARGUMENT, "pair index out of range.");
    if (h_off[l + 1] - h_off[l] < 2)
      throw Error(FLN_ERR_INVALID_ARGUMENT, "every loop in a pair needs at least two vertices.");
  }
  for (size_t p = 0; p + 1 < h_pairs.size(); p += 2)
    if (h_pairs[p] == h_pairs[p + 1]) throw Error(FLN_ERR_INVALID_ARGUMENT, "a pair must name two different loops.");
}

static fln_params resolved(const fln_params *p) {
  fln_params r;
  fln_default_params(&r);
  if (p) r = *p;
  if (r.precision != FLN_PREC_FP64 && r.precision != FLN_PREC_MIXED)
    throw Error(FLN_ERR_INVALID_ARGUMENT, "unknown precision");
  if (!(r.barnes_hut_init_beta > 0) || !(r.barnes_hut_beta_limit > 0))
    throw Error(FLN_ERR_INVALID_ARGUMENT, "Barnes-Hut beta must be positive");
  if (r.bh_escalations < 0 || r.bh_escalations > 8) throw Error(FLN_ERR_INVALID_ARGUMENT, "bh_escalations in [0, 8]");
  if (r.bh_schedule < 0 || r.bh_schedule > 2) throw Error(FLN_ERR_INVALID_ARGUMENT, "bh_schedule in [0, 2]");
  if (r.bh_budget != 0 && (r.bh_budget < 16 || r.bh_budget > 4096))
    throw Error(FLN_ERR_INVALID_ARGUMENT, "bh_budget 0 or in [16, 4096]");
  if (r.bh_bucket < 0 || r.bh_bucket > 16) throw Error(FLN_ERR_INVALID_ARGUMENT, "bh_bucket in [0, 16]");
  if (r.bh_retry_from_roots != 0 && r.bh_retry_from_roots != 1)
    throw Error(FLN_ERR_INVALID_ARGUMENT, "bh_retry_from_roots is 0 or 1");
  if (r.bh_spill_cap < 0 || r.bh_spill_cap > 8192) throw Error(FLN_ERR_INVALID_ARGUMENT, "bh_spill_cap in [0, 8192]");
  if (r.bh_wait_polls < 0) throw Error(FLN_ERR_INVALID_ARGUMENT, "bh_wait_polls must not be negative");
  if (r.bh_occupancy != 0 && (r.bh_occupancy < 5 || r.bh_occupancy > 7))
    throw Error(FLN_ERR_INVALID_ARGUMENT, "bh_occupancy 0 or in [5, 7]");
  if (r.direct_tile < 0 || r.direct_tile >= kDirectTileShapes)
    throw Error(FLN_ERR_INVALID_ARGUMENT, "direct_tile in [0, " + std::to_string(kDirectTileShapes - 1) + "]");
  return r;
}

}  // namespace fln

using namespace fln;

struct fln_ctx {
  std::unique_ptr<Context> c;
};
struct fln_model {
  Model m;
  int prepared_disc = -1;
};
struct fln_certificate {
  Certificate c;
};
struct fln_learned {
  std::vector<float> params;
  fln_learned_info info{};
};

namespace fln {
void set_last_error(const std::string &msg);

// prepare() with Discretize and both potential-link searches on the GPU.
static void prepare_device(Context &ctx, Model &m, bool discretize_on) {
  if (!discretize_on) {
    prepare(m, false);
    return;
  }
  discretize_device(ctx, m.curves, m.bcc_xyz.empty() ? nullptr : m.bcc_xyz.data(), m.poly_offsets, m.poly_xyz,
                    m.pairs, m.rounds);
  // An open curve that reaches the linking-number stage is an error there
  // (Curve::GetStartPoints, curve.cpp:126-128); one without pairs is not.
  for (size_t p = 0; p < m.pairs.size(); ++p)
    if (!m.curves[m.pairs[p]].closed)
      throw Error(FLN_ERR_UNLOOPED, "Curve::GetStartPoints() does not support unlooped curves.");
  m.prepared = true;
}
}  // namespace fln

namespace {
thread_local std::string g_last_error;

template <class F>
fln_status guarded(F &&f) {
  try {
    f();
    return FLN_OK;
  } catch (const Error &e) {
    g_last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc &) {
    g_last_error = "host out of memory";
    return FLN_ERR_OUT_OF_MEMORY;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return FLN_ERR_INTERNAL;
  }
}

// Pinned vertices for a Barnes–Hut call go up in Context::kXyzPieces pieces
// on the copy stream, split at loop boundaries, after the work already queued
// on the context's stream (which may still read the previous vertices); the
// tree build of each piece's loops waits only for its piece, so the copy
// overlaps the build.
bool copy_xyz_pieces(Context &ctx, double *d_xyz, const double *xyz, const std::vector<int64_t> &h_off) {
  const int32_t nloops = (int32_t)h_off.size() - 1;
  const int64_t nv = h_off[nloops];
  if (nloops < Context::kXyzPieces || 3 * nv * sizeof(double) < (size_t(64) << 20) || !is_pinned(xyz)) return false;
  if (!ctx.copy_stream) FLN_CUDA(cudaStreamCreateWithFlags(&ctx.copy_stream, cudaStreamNonBlocking));
  if (!ctx.ev_before_copy) FLN_CUDA(cudaEventCreateWithFlags(&ctx.ev_before_copy, cudaEventDisableTiming));
  for (cudaEvent_t &e : ctx.ev_piece)
    if (!e) FLN_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  FLN_CUDA(cudaEventRecord(ctx.ev_before_copy, ctx.stream));
  FLN_CUDA(cudaStreamWaitEvent(ctx.copy_stream, ctx.ev_before_copy, 0));
  int64_t start = 0;
  int32_t l = 0;
  for (int i = 0; i < Context::kXyzPieces; ++i) {
    const int64_t want = nv * (i + 1) / Context::kXyzPieces;
    while (l < nloops && h_off[l] < want) ++l;  // each piece ends at a loop boundary
    const int64_t end = i + 1 == Context::kXyzPieces ? nv : std::max(start, h_off[l]);
    if (end > start)
      FLN_CUDA(cudaMemcpyAsync(d_xyz + 3 * start, xyz + 3 * start, 3 * (end - start) * sizeof(double),
                               cudaMemcpyHostToDevice, ctx.copy_stream));
    FLN_CUDA(cudaEventRecord(ctx.ev_piece[i], ctx.copy_stream));
    ctx.xyz_piece_end[i] = end;
    start = end;
  }
  ctx.xyz_pieces = Context::kXyzPieces;
  return true;
}

void compute_pairs_host(Context &ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                        const int32_t *pairs, int64_t npairs, fln_method method, const fln_params &prm,
                        double *lk_out, double *err_out, int32_t *flags_out) {
  const double t0 = now_ms();
  FLN_CUDA(cudaSetDevice(ctx.device));
  std::vector<int64_t> h_off(loop_offsets, loop_offsets + nloops + 1);
  std::vector<int32_t> h_pairs(pairs, pairs + 2 * npairs);
  check_inputs(h_off, nloops, h_pairs);
  const int64_t nv = h_off[nloops];
  double *d_xyz = ctx.d_xyz.as<double>(3 * std::max<int64_t>(nv, 1));
  int64_t *d_off = ctx.d_off.as<int64_t>(nloops + 1);
  double *d_lk = ctx.d_lk.as<double>(std::max<int64_t>(npairs, 1));
  double *d_err = ctx.d_err.as<double>(std::max<int64_t>(npairs, 1));
  int32_t *d_flags = ctx.d_flags.as<int32_t>(std::max<int64_t>(npairs, 1));
  FLN_CUDA(cudaEventRecord(ctx.ev0, ctx.stream));
  ctx.xyz_pieces = 0;
  if (!(method == FLN_METHOD_BARNESHUT && prm.bh_tree == 0 && copy_xyz_pieces(ctx, d_xyz, xyz, h_off)))
    copy_h2d(ctx, d_xyz, xyz, 3 * nv * sizeof(double));
  FLN_CUDA(cudaMemcpyAsync(d_off, h_off.data(), (nloops + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, ctx.stream));
  int launches = 0;
  try {
    launches = run_pairs(ctx, d_xyz, d_off, h_off, h_pairs, method, prm, d_lk, d_err, d_flags);
  } catch (...) {
    wait_xyz_pieces(ctx);
    throw;
  }
  wait_xyz_pieces(ctx);
  FLN_CUDA(cudaEventRecord(ctx.ev1, ctx.stream));
  FLN_CUDA(cudaMemcpyAsync(lk_out, d_lk, npairs * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
  if (err_out) FLN_CUDA(cudaMemcpyAsync(err_out, d_err, npairs * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
  if (flags_out)
    FLN_CUDA(cudaMemcpyAsync(flags_out, d_flags, npairs * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
  FLN_CUDA(cudaStreamSynchronize(ctx.stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1);
  ctx.stats.ms_kernels = ms;
  ctx.stats.kernel_launches = launches;
  ctx.stats.ms_total = now_ms() - t0;
}
// A seeded sample (12345) of `want` pairs (0 = 2048; all when fewer), in
// their original order, for the autotuners.
static std::vector<int32_t> sample_of(const std::vector<int32_t> &h_all, int64_t npairs, int64_t want) {
  if (want <= 0) want = 2048;
  std::vector<int64_t> idx(npairs);
  std::iota(idx.begin(), idx.end(), 0);
  std::mt19937_64 rng(12345);
  std::shuffle(idx.begin(), idx.end(), rng);
  idx.resize(std::min(want, npairs));
  std::sort(idx.begin(), idx.end());
  std::vector<int32_t> out(2 * idx.size());
  for (size_t k = 0; k < idx.size(); ++k) {
    out[2 * k] = h_all[2 * idx[k]];
    out[2 * k + 1] = h_all[2 * idx[k] + 1];
  }
  return out;
}

// Host loops and pairs -> the context's device buffers (checked).
void upload_loops(Context &ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops, const int32_t *pairs,
                  int64_t npairs, std::vector<int64_t> &h_off, std::vector<int32_t> &h_pairs, double **d_xyz,
                  int64_t **d_off) {
  if (!xyz || !loop_offsets || !pairs || nloops < 0 || npairs < 0) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
  FLN_CUDA(cudaSetDevice(ctx.device));
  h_off.assign(loop_offsets, loop_offsets + nloops + 1);
  h_pairs.assign(pairs, pairs + 2 * npairs);
  check_inputs(h_off, nloops, h_pairs);
  const int64_t nv = h_off[nloops];
  *d_xyz = ctx.d_xyz.as<double>(3 * std::max<int64_t>(nv, 1));
  *d_off = ctx.d_off.as<int64_t>(nloops + 1);
  ctx.xyz_pieces = 0;
  FLN_CUDA(cudaMemcpyAsync(*d_xyz, xyz, 3 * nv * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));
  FLN_CUDA(cudaMemcpyAsync(*d_off, h_off.data(), (nloops + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, ctx.stream));
}

double pinball(float y, float t, double q) {
  const double e = (double)t - (double)y;
  return e >= 0 ? q * e : (q - 1.0) * e;
}
}  // namespace

void fln::set_last_error(const std::string &msg) { g_last_error = msg; }

extern "C" {

const char *fln_status_string(fln_status s) {
  switch (s) {
    case FLN_OK: return "ok";
    case FLN_ERR_INVALID_ARGUMENT: return "invalid argument";
    case FLN_ERR_IO: return "i/o error";
    case FLN_ERR_FORMAT: return "format error";
    case FLN_ERR_CUDA: return "CUDA error";
    case FLN_ERR_NO_DEVICE: return "no CUDA device";
    case FLN_ERR_OUT_OF_MEMORY: return "out of memory";
    case FLN_ERR_SEGMENT_TOO_SMALL: return "segment smaller than eps * average coordinate";
    case FLN_ERR_MAX_RECURSION: return "Discretize reached its maximum number of rounds";
    case FLN_ERR_UNLOOPED: return "open curve in the linking-number stage";
    case FLN_ERR_NONFINITE: return "non-finite linking number";
    case FLN_ERR_STACK_OVERFLOW: return "traversal stack overflow";
    case FLN_ERR_TIMEOUT: return "bounded device wait ran out";
    default: return "internal error";
  }
}

const char *fln_last_error(void) { return g_last_error.c_str(); }
int fln_abi_version(void) { return FLN_ABI_VERSION; }

void fln_default_params(fln_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->barnes_hut_init_beta = 2.0;
  p->barnes_hut_beta_limit = 10.0;
  p->epssq = 1e-24;
  p->target_error = 0.1;
  p->error_est_scale = 0.05;
  p->precision = FLN_PREC_MIXED;
  p->fp64_margin = 0.25;
  p->near_factor = kDefaultNearFactor;
  p->bh_tree = 0;
  p->bh_escalations = 2;
  p->bh_err_limit = 0.25;
}

fln_status fln_ctx_create(int device, void *stream, fln_ctx **out) {
  return guarded([&] {
    if (!out) throw Error(FLN_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    auto *c = new fln_ctx;
    try {
      c->c.reset(new Context(device, stream));
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
  });
}

void fln_ctx_destroy(fln_ctx *ctx) { delete ctx; }

fln_status fln_ctx_stats(const fln_ctx *ctx, fln_stats *out) {
  return guarded([&] {
    if (!ctx || !out) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = ctx->c->stats;
  });
}

fln_status fln_linking_numbers(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                               const int32_t *pairs, int64_t npairs, fln_method method, const fln_params *params,
                               double *lk_out, double *err_out, int32_t *flags_out) {
  return guarded([&] {
    if (!ctx || !loop_offsets || nloops < 0 || npairs < 0 || (npairs && (!pairs || !lk_out)) ||
        (!xyz && nloops && loop_offsets[nloops] > 0))
      throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL or negative argument");
    if (method != FLN_METHOD_DIRECTSUM && method != FLN_METHOD_BARNESHUT)
      throw Error(FLN_ERR_INVALID_ARGUMENT, "Invalid method");
    const fln_params prm = resolved(params);
    compute_pairs_host(*ctx->c, xyz, loop_offsets, nloops, pairs, npairs, method, prm, lk_out, err_out, flags_out);
  });
}

fln_status fln_linking_numbers_device(fln_ctx *ctx, const double *d_xyz, const int64_t *d_loop_offsets,
                                      int32_t nloops, const int32_t *d_pairs, int64_t npairs, fln_method method,
                                      const fln_params *params, double *d_lk_out, double *d_err_out,
                                      int32_t *d_flags_out) {
  return guarded([&] {
    if (!ctx || !d_loop_offsets || nloops < 0 || npairs < 0 || (npairs && (!d_pairs || !d_lk_out)))
      throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL or negative argument");
    if (method != FLN_METHOD_DIRECTSUM && method != FLN_METHOD_BARNESHUT)
      throw Error(FLN_ERR_INVALID_ARGUMENT, "Invalid method");
    const fln_params prm = resolved(params);
    Context &c = *ctx->c;
    const double t0 = now_ms();
    FLN_CUDA(cudaSetDevice(c.device));
    std::vector<int64_t> h_off(nloops + 1);
    std::vector<int32_t> h_pairs(2 * npairs);
    FLN_CUDA(cudaEventRecord(c.ev0, c.stream));
    FLN_CUDA(cudaMemcpyAsync(h_off.data(), d_loop_offsets, (nloops + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                             c.stream));
    if (npairs)
      FLN_CUDA(cudaMemcpyAsync(h_pairs.data(), d_pairs, 2 * npairs * sizeof(int32_t), cudaMemcpyDeviceToHost,
                               c.stream));
    FLN_CUDA(cudaStreamSynchronize(c.stream));
    check_inputs(h_off, nloops, h_pairs);
    const int launches = run_pairs(c, d_xyz, d_loop_offsets, h_off, h_pairs, method, prm, d_lk_out, d_err_out,
                                   d_flags_out);
    FLN_CUDA(cudaEventRecord(c.ev1, c.stream));
    FLN_CUDA(cudaStreamSynchronize(c.stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, c.ev0, c.ev1);
    c.stats.ms_kernels = ms;
    c.stats.kernel_launches = launches;
    c.stats.ms_total = now_ms() - t0;
  });
}

fln_status fln_direct_pair(fln_ctx *ctx, const double *xyz1, int64_t n1, const double *xyz2, int64_t n2,
                           int32_t precision, double *lk_out) {
  return guarded([&] {
    if (!ctx || !xyz1 || !xyz2 || !lk_out || n1 < 2 || n2 < 2)
      throw Error(FLN_ERR_INVALID_ARGUMENT, "each loop needs at least two vertices");
    std::vector<double> xyz(3 * (n1 + n2));
    std::memcpy(xyz.data(), xyz1, 3 * n1 * sizeof(double));
    std::memcpy(xyz.data() + 3 * n1, xyz2, 3 * n2 * sizeof(double));
    const int64_t off[3] = {0, n1, n1 + n2};
    const int32_t pr[2] = {0, 1};
    fln_params prm;
    fln_default_params(&prm);
    prm.precision = precision;
    const fln_params r = resolved(&prm);
    compute_pairs_host(*ctx->c, xyz.data(), off, 2, pr, 1, FLN_METHOD_DIRECTSUM, r, lk_out, nullptr, nullptr);
  });
}

void fln_learned_default_options(fln_learned_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->s_min = 1.5;
  o->sample_keep = 0.05;
  o->max_samples = int64_t(1) << 20;
  o->max_terms = int64_t(1) << 16;
  o->epochs = 40;
  o->batch = 4096;
  o->learning_rate = 2e-3;
  o->quantile = 0.9;
  o->tau_quantile = 0.5;
  o->val_fraction = 0.1;
  o->min_candidates = 4;
  o->seed = 1;
}

fln_status fln_learned_collect(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                               const int32_t *pairs, int64_t npairs, const fln_params *params, double s_min,
                               double sample_keep, int64_t cap, int64_t max_terms, float *features_out,
                               float *target_out, float *sep_out, float *est_out, int64_t *n_out) {
  return guarded([&] {
    if (!ctx || !n_out || cap < 0 || (cap > 0 && (!features_out || !target_out))) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    const fln_params prm = resolved(params);
    std::vector<int64_t> h_off;
    std::vector<int32_t> h_pairs;
    double *d_xyz;
    int64_t *d_off;
    upload_loops(*ctx->c, xyz, loop_offsets, nloops, pairs, npairs, h_off, h_pairs, &d_xyz, &d_off);
    std::vector<float> X, T, S, E;
    int64_t recorded = 0;
    learned_collect(*ctx->c, d_xyz, d_off, h_off, h_pairs, prm, (float)s_min, sample_keep, cap, max_terms, X, T, S,
                    E, &recorded);
    const int64_t n = (int64_t)T.size();
    if (n > 0) {
      std::memcpy(features_out, X.data(), X.size() * sizeof(float));
      std::memcpy(target_out, T.data(), T.size() * sizeof(float));
      if (sep_out) std::memcpy(sep_out, S.data(), S.size() * sizeof(float));
      if (est_out) std::memcpy(est_out, E.data(), E.size() * sizeof(float));
    }
    *n_out = n;
  });
}

fln_status fln_learned_train(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                             const int32_t *pairs, int64_t npairs, const fln_params *params,
                             const fln_learned_options *options, fln_learned **out) {
  return guarded([&] {
    if (!ctx || !out) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    fln_learned_options o;
    fln_learned_default_options(&o);
    if (options) o = *options;
    if (!(o.s_min > 0) || !(o.sample_keep > 0 && o.sample_keep <= 1) || o.max_samples <= 0 || o.max_terms <= 0 ||
        o.epochs <= 0 || o.batch <= 0 || !(o.learning_rate > 0) || !(o.quantile > 0 && o.quantile < 1) ||
        !(o.tau_quantile >= 0 && o.tau_quantile <= 1) || !(o.val_fraction >= 0 && o.val_fraction < 1))
      throw Error(FLN_ERR_INVALID_ARGUMENT, "learned options out of range");
    const fln_params prm = resolved(params);
    Context &c = *ctx->c;
    std::vector<int64_t> h_off;
    std::vector<int32_t> h_pairs;
    double *d_xyz;
    int64_t *d_off;
    const double t0 = now_ms();
    upload_loops(c, xyz, loop_offsets, nloops, pairs, npairs, h_off, h_pairs, &d_xyz, &d_off);
    std::vector<float> X, T, S, E;
    int64_t recorded = 0;
    learned_collect(c, d_xyz, d_off, h_off, h_pairs, prm, (float)o.s_min, o.sample_keep, o.max_samples, o.max_terms,
                    X, T, S, E, &recorded);
    const double t1 = now_ms();
    const int64_t n = (int64_t)T.size();
    if (n < 256) throw Error(FLN_ERR_INVALID_ARGUMENT, "too few training samples (" + std::to_string(n) + ")");
    // Threshold: the tau_quantile of the true errors of accepted far-field pairs.
    const double b0 = prm.barnes_hut_init_beta;
    std::vector<float> acc;
    for (int64_t k = 0; k < n; ++k)
      if (S[k] >= b0) acc.push_back(T[k]);
    if (acc.empty()) throw Error(FLN_ERR_INVALID_ARGUMENT, "no recorded far-field pairs to set the threshold");
    std::sort(acc.begin(), acc.end());
    const double log10_tau = acc[std::min<size_t>(acc.size() - 1, (size_t)(o.tau_quantile * (acc.size() - 1) + 0.5))];
    // Split, initialise (He normal), train.
    std::mt19937_64 rng(o.seed);
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::shuffle(idx.begin(), idx.end(), rng);
    const int64_t nval = (int64_t)(o.val_fraction * n);
    std::vector<int32_t> val(idx.begin(), idx.begin() + nval), train(idx.begin() + nval, idx.end());
    std::vector<float> prm_mlp(FLN_MLP_PARAMS, 0.f);
    std::normal_distribution<float> nd(0.f, 1.f);
    const int kIn = 8, kH = 64;
    for (int k = 0; k < kIn * kH; ++k) prm_mlp[k] = nd(rng) * std::sqrt(2.f / kIn);
    const int w2 = kIn * kH + kH, b2 = w2 + kH * kH, w3 = b2 + kH, b3 = w3 + kH;
    for (int k = 0; k < kH * kH; ++k) prm_mlp[w2 + k] = nd(rng) * std::sqrt(2.f / kH);
    for (int k = 0; k < kH; ++k) prm_mlp[w3 + k] = nd(rng) * std::sqrt(1.f / kH);
    {
      std::vector<float> tt;
      for (int32_t r : train) tt.push_back(T[r]);
      std::nth_element(tt.begin(), tt.begin() + tt.size() / 2, tt.end());
      prm_mlp[b3] = tt[tt.size() / 2];
    }
    TrainOptions to;
    to.epochs = o.epochs;
    to.batch = o.batch;
    to.lr = (float)o.learning_rate;
    to.quantile = (float)o.quantile;
    to.seed = o.seed;
    const double train_loss = learned_train(c, X, T, train, to, prm_mlp);
    double val_loss = 0, cover = 0;
    if (nval > 0) {
      std::vector<float> xv((size_t)kIn * nval), yv(nval);
      for (int64_t k = 0; k < nval; ++k) std::memcpy(&xv[kIn * k], &X[(size_t)kIn * val[k]], kIn * sizeof(float));
      learned_predict(c, prm_mlp.data(), xv.data(), nval, 0, yv.data());
      for (int64_t k = 0; k < nval; ++k) {
        val_loss += pinball(yv[k], T[val[k]], o.quantile);
        cover += T[val[k]] <= yv[k] ? 1.0 : 0.0;
      }
      val_loss /= nval;
      cover /= nval;
    }
    auto *m = new fln_learned;
    m->params = std::move(prm_mlp);
    fln_learned_info &inf = m->info;
    inf.recorded = recorded;
    inf.samples = n;
    inf.train_samples = (int64_t)train.size();
    inf.val_samples = nval;
    inf.s_min = o.s_min;
    inf.log10_tau = log10_tau;
    inf.min_candidates = std::max(1, o.min_candidates);
    inf.min_node_segments = std::max(0, o.min_node_segments);
    inf.epochs = o.epochs;
    inf.train_loss = train_loss;
    inf.val_loss = val_loss;
    inf.val_coverage = cover;
    inf.ms_collect = t1 - t0;
    inf.ms_train = now_ms() - t1;
    *out = m;
  });
}

fln_status fln_learned_create(const float *params, double s_min, double log10_tau, int32_t min_candidates,
                              fln_learned **out) {
  return guarded([&] {
    if (!params || !out) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!(s_min > 0) || !std::isfinite(log10_tau)) throw Error(FLN_ERR_INVALID_ARGUMENT, "s_min or log10_tau");
    for (int k = 0; k < FLN_MLP_PARAMS; ++k)
      if (!std::isfinite(params[k])) throw Error(FLN_ERR_INVALID_ARGUMENT, "non-finite MLP parameter");
    auto *m = new fln_learned;
    m->params.assign(params, params + FLN_MLP_PARAMS);
    m->info.s_min = s_min;
    m->info.log10_tau = log10_tau;
    m->info.min_candidates = std::max(1, min_candidates);
    *out = m;
  });
}

void fln_learned_destroy(fln_learned *m) { delete m; }

fln_status fln_learned_configure(fln_learned *m, int32_t min_candidates, int32_t min_node_segments) {
  return guarded([&] {
    if (!m) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL model");
    if (min_candidates < 1 || min_candidates > 32 || min_node_segments < 0)
      throw Error(FLN_ERR_INVALID_ARGUMENT, "min_candidates in [1, 32], min_node_segments >= 0");
    m->info.min_candidates = min_candidates;
    m->info.min_node_segments = min_node_segments;
  });
}

fln_status fln_learned_get(const fln_learned *m, float *params_out, fln_learned_info *info_out) {
  return guarded([&] {
    if (!m) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL model");
    if (params_out) std::memcpy(params_out, m->params.data(), FLN_MLP_PARAMS * sizeof(float));
    if (info_out) *info_out = m->info;
  });
}

fln_status fln_ctx_set_learned(fln_ctx *ctx, const fln_learned *m) {
  return guarded([&] {
    if (!ctx) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL context");
    FLN_CUDA(cudaSetDevice(ctx->c->device));
    if (!m) learned_enable(*ctx->c, nullptr, 0.f, 0.f, 0, 0);
    else
      learned_enable(*ctx->c, m->params.data(), (float)m->info.s_min, (float)m->info.log10_tau,
                     m->info.min_candidates, m->info.min_node_segments);
  });
}

fln_status fln_learned_predict(fln_ctx *ctx, const float *params, const float *features, int64_t n,
                               int32_t use_mma, float *y_out) {
  return guarded([&] {
    if (!ctx || !params || (n > 0 && (!features || !y_out)) || n < 0) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    FLN_CUDA(cudaSetDevice(ctx->c->device));
    learned_predict(*ctx->c, params, features, n, use_mma ? 1 : 0, y_out);
  });
}

fln_status fln_learned_gradients(fln_ctx *ctx, const float *params, const float *features,
                                 const float *targets, int64_t n, double quantile, float *grad_out,
                                 double *loss_out) {
  return guarded([&] {
    if (!ctx || !params || !features || !targets || !grad_out || n <= 0) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!(quantile > 0 && quantile < 1)) throw Error(FLN_ERR_INVALID_ARGUMENT, "quantile in (0, 1)");
    FLN_CUDA(cudaSetDevice(ctx->c->device));
    const double l = learned_gradients(*ctx->c, params, features, targets, n, (float)quantile, grad_out);
    if (loss_out) *loss_out = l;
  });
}

fln_status fln_autotune_direct(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                               const int32_t *pairs, int64_t npairs, const fln_params *params, int64_t sample_pairs,
                               fln_params *out, fln_tune_result *result) {
  return guarded([&] {
    if (!ctx || !out || npairs <= 0) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument or no pairs");
    const fln_params base = resolved(params);
    Context &c = *ctx->c;
    std::vector<int64_t> h_off;
    std::vector<int32_t> h_all;
    double *d_xyz;
    int64_t *d_off;
    upload_loops(c, xyz, loop_offsets, nloops, pairs, npairs, h_off, h_all, &d_xyz, &d_off);
    const std::vector<int32_t> h_pairs = sample_of(h_all, npairs, sample_pairs);
    const int64_t np = (int64_t)h_pairs.size() / 2;
    double *d_lk = c.d_lk.as<double>(np), *d_err = c.d_err.as<double>(np);
    int32_t *d_fl = c.d_flags.as<int32_t>(np);
    auto time_of = [&](const fln_params &p) {
      double best = 1e300;
      for (int rep = 0; rep < 3; ++rep) {
        FLN_CUDA(cudaEventRecord(c.ev0, c.stream));
        run_pairs(c, d_xyz, d_off, h_off, h_pairs, FLN_METHOD_DIRECTSUM, p, d_lk, d_err, d_fl);
        FLN_CUDA(cudaEventRecord(c.ev1, c.stream));
        best = std::min(best, (double)c.elapsed(c.ev0, c.ev1));
      }
      return best;
    };
    time_of(base);  // warm-up
    fln_tune_result r{};
    r.sample_pairs = (int32_t)np;
    r.default_ms = time_of(base);
    fln_params best = base;
    r.best_ms = r.default_ms;
    r.trials = 1;
    for (int t = 0; t < kDirectTileShapes; ++t) {
      if (t == base.direct_tile) continue;
      fln_params p = base;
      p.direct_tile = t;
      const double ms = time_of(p);
      ++r.trials;
      if (ms < r.best_ms) {
        r.best_ms = ms;
        best = p;
      }
    }
    r.best_direct_tile = best.direct_tile;
    r.best_budget = best.bh_budget > 0 ? best.bh_budget : kDefaultBhBudget;
    r.best_beta = best.barnes_hut_init_beta;
    r.best_bucket = best.bh_bucket > 0 ? best.bh_bucket : 8;
    r.best_occupancy = best.bh_occupancy > 0 ? best.bh_occupancy : 5;
    *out = best;
    if (result) *result = r;
  });
}

fln_status fln_autotune(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                        const int32_t *pairs, int64_t npairs, const fln_params *params, int32_t tune_beta,
                        int64_t sample_pairs, fln_params *out, fln_tune_result *result) {
  return guarded([&] {
    if (!ctx || !out || npairs <= 0) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument or no pairs");
    const fln_params base = resolved(params);
    Context &c = *ctx->c;
    std::vector<int64_t> h_off;
    std::vector<int32_t> h_all;
    double *d_xyz;
    int64_t *d_off;
    upload_loops(c, xyz, loop_offsets, nloops, pairs, npairs, h_off, h_all, &d_xyz, &d_off);
    const std::vector<int32_t> h_pairs = sample_of(h_all, npairs, sample_pairs);
    const int64_t np = (int64_t)h_pairs.size() / 2;
    double *d_lk = c.d_lk.as<double>(np), *d_err = c.d_err.as<double>(np);
    int32_t *d_fl = c.d_flags.as<int32_t>(np);
    auto time_of = [&](const fln_params &p) {
      double best = 1e300;
      for (int rep = 0; rep < 3; ++rep) {
        FLN_CUDA(cudaEventRecord(c.ev0, c.stream));
        run_pairs(c, d_xyz, d_off, h_off, h_pairs, FLN_METHOD_BARNESHUT, p, d_lk, d_err, d_fl);
        FLN_CUDA(cudaEventRecord(c.ev1, c.stream));
        best = std::min(best, (double)c.elapsed(c.ev0, c.ev1));
      }
      return best;
    };
    time_of(base);  // warm-up: trees, buffers, kernel loading
    // A setting replaces the best so far only when it is faster by more than
    // the run-to-run spread of the timing (about 1 %), so noise does not pick
    // among settings that tie.
    constexpr double kTuneMargin = 0.985;
    fln_tune_result r{};
    r.sample_pairs = (int32_t)np;
    r.default_ms = time_of(base);
    fln_params best = base;
    r.best_ms = r.default_ms;
    r.trials = 1;
    const bool t_beta = (tune_beta & 1) != 0, t_bucket = (tune_beta & 2) != 0 && base.bh_tree == 0;
    const double betas[] = {1.5, 2.0, 2.5, 3.0};
    const int budgets[] = {128, 256, 512};
    auto try_budgets = [&](fln_params p) {
      for (int bud : budgets) {
        p.bh_budget = bud;
        const double ms = time_of(p);
        ++r.trials;
        if (ms < kTuneMargin * r.best_ms) {
          r.best_ms = ms;
          best = p;
        }
      }
    };
    for (double b : betas) {
      if (!t_beta && b != base.barnes_hut_init_beta) continue;
      fln_params p = base;
      if (t_beta) p.barnes_hut_init_beta = b;
      try_budgets(p);
    }
    if (!t_beta && base.barnes_hut_init_beta != 1.5 && base.barnes_hut_init_beta != 2.0 &&
        base.barnes_hut_init_beta != 2.5 && base.barnes_hut_init_beta != 3.0)
      try_budgets(base);  // the caller's own beta
    {  // traversal occupancy at the best setting (the same node pairs)
      const fln_params around = best;
      for (int occ : {6, 7}) {
        fln_params p = around;
        p.bh_occupancy = occ;
        const double ms = time_of(p);
        ++r.trials;
        if (ms < kTuneMargin * r.best_ms) {
          r.best_ms = ms;
          best = p;
        }
      }
    }
    if (t_bucket) {
      // Exact buckets of other sizes around the best setting so far (the
      // node pairs change: real sums move within the Barnes-Hut error).
      const fln_params around = best;
      for (int bk : {4, 6, 10, 12, 16}) {
        fln_params p = around;
        p.bh_bucket = bk;
        const double ms = time_of(p);
        ++r.trials;
        if (ms < kTuneMargin * r.best_ms) {
          r.best_ms = ms;
          best = p;
        }
      }
    }
    if (best.bh_budget <= 0) best.bh_budget = kDefaultBhBudget;  // the tuned parameters name their budget
    r.best_budget = best.bh_budget;
    r.best_beta = best.barnes_hut_init_beta;
    r.best_bucket = best.bh_bucket > 0 ? best.bh_bucket : 8;
    r.best_occupancy = best.bh_occupancy > 0 ? best.bh_occupancy : 5;
    *out = best;
    if (result) *result = r;
  });
}

fln_status fln_model_create(fln_model **out) {
  return guarded([&] {
    if (!out) throw Error(FLN_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = new fln_model;
  });
}
void fln_model_destroy(fln_model *m) { delete m; }

fln_status fln_model_load_bcc(fln_model *m, const char *path) {
  return guarded([&] {
    if (!m || !path) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    const std::string p(path);
    const size_t dot = p.rfind('.');
    std::string ext = dot == std::string::npos ? "" : p.substr(dot);
    for (auto &ch : ext) ch = (char)std::tolower((unsigned char)ch);
    if (ext != ".bcc") throw Error(FLN_ERR_FORMAT, "File extension for import must be .bcc: " + p);
    load_bcc(p, m->m);
    m->prepared_disc = -1;
  });
}

fln_status fln_model_save_bcc(const fln_model *m, const char *path) {
  return guarded([&] {
    if (!m || !path) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    save_bcc(path, m->m);
  });
}

fln_status fln_model_set_curves(fln_model *m, fln_seg_type type, int32_t ncurves, const int32_t *counts,
                                const double *xyz) {
  return guarded([&] {
    if (!m || ncurves < 0 || (ncurves && !counts)) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    if ((int)type < 0 || (int)type > 3) throw Error(FLN_ERR_INVALID_ARGUMENT, "unknown segment type");
    std::vector<CurveData> cs(ncurves);
    int64_t at = 0;
    for (int32_t i = 0; i < ncurves; ++i) {
      const int64_t n = counts[i] < 0 ? -(int64_t)counts[i] : counts[i];
      cs[i].kind = (SegKind)type;
      cs[i].closed = counts[i] < 0;
      cs[i].q.resize(n);
      if (n && !xyz) throw Error(FLN_ERR_INVALID_ARGUMENT, "xyz is NULL");
      for (int64_t k = 0; k < n; ++k, ++at) cs[i].q[k] = {xyz[3 * at], xyz[3 * at + 1], xyz[3 * at + 2]};
    }
    m->m.curves.swap(cs);
    m->m.bcc_xyz.clear();
    m->m.bcc_xyz.shrink_to_fit();
    m->m.prepared = false;
    m->prepared_disc = -1;
  });
}

int32_t fln_model_num_curves(const fln_model *m) { return m ? (int32_t)m->m.curves.size() : 0; }
int64_t fln_model_num_points(const fln_model *m) {
  int64_t t = 0;
  if (m)
    for (auto &c : m->m.curves) t += (int64_t)c.q.size();
  return t;
}

fln_status fln_model_get_curves(const fln_model *m, int32_t *type_out, int32_t *counts_out, double *xyz_out) {
  return guarded([&] {
    if (!m) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL model");
    if (type_out) *type_out = m->m.curves.empty() ? FLN_SEG_CATMULLROM : (int32_t)m->m.curves[0].kind;
    int64_t at = 0;
    for (size_t i = 0; i < m->m.curves.size(); ++i) {
      const auto &c = m->m.curves[i];
      if (counts_out) counts_out[i] = c.closed ? -(int32_t)c.q.size() : (int32_t)c.q.size();
      for (auto &v : c.q) {
        if (xyz_out) {
          xyz_out[3 * at] = v.x;
          xyz_out[3 * at + 1] = v.y;
          xyz_out[3 * at + 2] = v.z;
        }
        ++at;
      }
    }
  });
}

fln_status fln_model_prepare(fln_model *m, int discretize, int32_t *rounds_out) {
  return guarded([&] {
    if (!m) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL model");
    prepare(m->m, discretize != 0);
    m->prepared_disc = discretize != 0;
    if (rounds_out) *rounds_out = m->m.rounds;
  });
}

fln_status fln_model_prepare_device(fln_ctx *ctx, fln_model *m, int discretize, int32_t *rounds_out) {
  return guarded([&] {
    if (!ctx || !m) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    FLN_CUDA(cudaSetDevice(ctx->c->device));
    prepare_device(*ctx->c, m->m, discretize != 0);
    m->prepared_disc = discretize != 0;
    if (rounds_out) *rounds_out = m->m.rounds;
  });
}

fln_status fln_model_prepared_sizes(const fln_model *m, int64_t *num_vertices, int64_t *num_pairs) {
  return guarded([&] {
    if (!m || !m->m.prepared) throw Error(FLN_ERR_INVALID_ARGUMENT, "model not prepared");
    if (num_vertices) *num_vertices = m->m.poly_offsets.empty() ? 0 : m->m.poly_offsets.back();
    if (num_pairs) *num_pairs = (int64_t)m->m.pairs.size() / 2;
  });
}

fln_status fln_model_get_prepared(const fln_model *m, int64_t *loop_offsets_out, double *xyz_out,
                                  int32_t *pairs_out) {
  return guarded([&] {
    if (!m || !m->m.prepared) throw Error(FLN_ERR_INVALID_ARGUMENT, "model not prepared");
    if (loop_offsets_out)
      std::memcpy(loop_offsets_out, m->m.poly_offsets.data(), m->m.poly_offsets.size() * sizeof(int64_t));
    if (xyz_out) parallel_memcpy(xyz_out, m->m.poly_xyz.data(), m->m.poly_xyz.size() * sizeof(double));
    if (pairs_out) std::memcpy(pairs_out, m->m.pairs.data(), m->m.pairs.size() * sizeof(int32_t));
  });
}

fln_status fln_certificate_compute(fln_ctx *ctx, const fln_model *model, int force_direct_sum, int discretize,
                                   const fln_params *params, fln_certificate **out) {
  return guarded([&] {
    if (!ctx || !model || !out) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    const fln_params prm = resolved(params);
    auto *mm = const_cast<fln_model *>(model);  // the prepared polylines are a cache
    const double t0 = now_ms();
    if (!mm->m.prepared || mm->prepared_disc != (discretize != 0)) {
      FLN_CUDA(cudaSetDevice(ctx->c->device));
      if (prm.host_prepare) prepare(mm->m, discretize != 0);
      else prepare_device(*ctx->c, mm->m, discretize != 0);
      mm->prepared_disc = discretize != 0;
    }
    const double t1 = now_ms();
    const Model &m = mm->m;
    const int32_t nc = (int32_t)m.curves.size();
    const int64_t np = (int64_t)m.pairs.size() / 2;
    std::unique_ptr<fln_certificate> cert(new fln_certificate);
    cert->c.pairs = m.pairs;
    cert->c.lk.assign(np, 0.0);
    cert->c.err.assign(np, 0.0);
    cert->c.flags.assign(np, 0);
    Context &c = *ctx->c;
    if (np)
      compute_pairs_host(c, m.poly_xyz.data(), m.poly_offsets.data(), nc, m.pairs.data(), np,
                         force_direct_sum ? FLN_METHOD_DIRECTSUM : FLN_METHOD_BARNESHUT, prm, cert->c.lk.data(),
                         cert->c.err.data(), cert->c.flags.data());
    else
      c.stats = fln_stats{};
    fill_certificate(cert->c, nc, m.pairs, cert->c.lk);
    c.stats.ms_discretize = t1 - t0;
    c.stats.discretize_rounds = m.rounds;
    c.stats.mean_off_integer = cert->c.mean_off;
    c.stats.max_off_integer = cert->c.max_off;
    c.stats.ms_total = now_ms() - t0;
    *out = cert.release();
  });
}

fln_status fln_certificate_load(const char *path, fln_certificate **out) {
  return guarded([&] {
    if (!path || !out) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    std::unique_ptr<fln_certificate> c(new fln_certificate);
    c->c = read_certificate(path);
    *out = c.release();
  });
}

void fln_certificate_destroy(fln_certificate *c) { delete c; }

fln_status fln_certificate_save(const fln_certificate *c, const char *path) {
  return guarded([&] {
    if (!c || !path) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    FILE *f = std::fopen(path, "wb");
    if (!f) throw Error(FLN_ERR_IO, std::string("Cannot write certificate: ") + path);
    const std::string t = c->c.text();
    const bool ok = std::fwrite(t.data(), 1, t.size(), f) == t.size();
    std::fclose(f);
    if (!ok) throw Error(FLN_ERR_IO, std::string("Cannot write certificate: ") + path);
  });
}

int64_t fln_certificate_text(const fln_certificate *c, char *buf, int64_t cap) {
  if (!c) return -1;
  const std::string t = c->c.text();
  if (buf && cap > 0) {
    const int64_t k = std::min<int64_t>(cap - 1, (int64_t)t.size());
    std::memcpy(buf, t.data(), k);
    buf[k] = 0;
  }
  return (int64_t)t.size();
}

int32_t fln_certificate_num_curves(const fln_certificate *c) { return c ? c->c.ncurves : 0; }
int64_t fln_certificate_num_entries(const fln_certificate *c) { return c ? (int64_t)c->c.entries.size() : 0; }

fln_status fln_certificate_entries(const fln_certificate *c, int32_t *entries_out) {
  return guarded([&] {
    if (!c || !entries_out) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL argument");
    for (size_t k = 0; k < c->c.entries.size(); ++k) {
      entries_out[3 * k] = c->c.entries[k].i;
      entries_out[3 * k + 1] = c->c.entries[k].j;
      entries_out[3 * k + 2] = c->c.entries[k].lk;
    }
  });
}

int64_t fln_certificate_num_pairs(const fln_certificate *c) { return c ? (int64_t)c->c.lk.size() : 0; }

fln_status fln_certificate_pairs(const fln_certificate *c, int32_t *pairs_out, double *lk_out, double *err_out,
                                 int32_t *flags_out) {
  return guarded([&] {
    if (!c) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL certificate");
    const size_t np = c->c.lk.size();
    if (pairs_out) std::memcpy(pairs_out, c->c.pairs.data(), 2 * np * sizeof(int32_t));
    if (lk_out) std::memcpy(lk_out, c->c.lk.data(), np * sizeof(double));
    if (err_out) std::memcpy(err_out, c->c.err.data(), np * sizeof(double));
    if (flags_out) std::memcpy(flags_out, c->c.flags.data(), np * sizeof(int32_t));
  });
}

int fln_certificate_equals(const fln_certificate *a, const fln_certificate *b) {
  if (!a || !b || a->c.ncurves != b->c.ncurves || a->c.entries.size() != b->c.entries.size()) return 0;
  for (size_t k = 0; k < a->c.entries.size(); ++k) {
    const auto &x = a->c.entries[k], &y = b->c.entries[k];
    if (x.i != y.i || x.j != y.j || x.lk != y.lk) return 0;
  }
  return 1;
}

fln_status fln_certificate_export_diffs(const fln_certificate *self, const fln_certificate *other,
                                        const char *diff_pairs_path, const char *diff_curves_path) {
  return guarded([&] {
    if (!self || !other) throw Error(FLN_ERR_INVALID_ARGUMENT, "NULL certificate");
    export_diffs(self->c, other->c, diff_pairs_path ? diff_pairs_path : "", diff_curves_path ? diff_curves_path : "");
  });
}

}  // extern "C"
