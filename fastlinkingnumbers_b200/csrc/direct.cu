// Direct summation of the Gauss linking integral on B200 (sm_100a).
//
// Work: every potential loop pair (i, j) is split into items of kBlockSegs
// consecutive segments of its longer loop ("curve 1"); one CTA of kBlockSegs
// threads takes items from a device work queue (an atomic counter) until it
// runs dry, so all pairs — 16-segment rings to 2^18-segment loops — run in
// one persistent launch. Each thread owns one curve-1 segment and walks all
// curve-2 segments, which the CTA stages tile by tile in shared memory
// (coalesced loads, broadcast reads). Per segment pair it evaluates the
// closed-form solid-angle term of Arai 2013 as the reference does
// (src/compute_link.cpp:126-178, :200-280): with a = q_k - p_i,
// b = q_k - p_{i+1}, c = q_{k+1} - p_{i+1}, d = q_{k+1} - p_i,
//   det  = a . (b x c)
//   div1 = |a||b||c| + (a.b)|c| + (c.a)|b| + (c.b)|a|
//   div2 = |a||d||c| + (a.d)|c| + (c.a)|d| + (c.d)|a|
//   term = atan2(det (div1 + div2), div1 div2 - det^2) / 2pi
//          + [det (div1 + div2) det < 0] sign(det)          (in full turns).
// Consecutive steps share vertices: step k+1's a, b are step k's d, c, so
// each step computes two new difference vectors and two norms.
//
// Two precisions:
//  * FP64 ("plain FP64 GPU direct sum"): every operation in FP64; the per-
//    thread terms are combined by the arctangent-addition recurrence of
//    ComputeLinkingNumberDirectFast (Bertolazzi et al. 2019) — a running
//    complex product with a count of negative-x-axis crossings — and one
//    atan2 per thread per item. The product is rescaled by an exact power of
//    two each step instead of the reference's division.
//  * MIXED: coordinates relative to the tile's first vertex in FP32, one
//    FP32 atan2 per segment pair, FP32 sums over one tile of kTile terms and
//    FP64 sums above that. det uses the identity det = a . (f x e) with
//    e = p_{i+1} - p_i and f = q_{k+1} - q_k, which keeps its relative
//    accuracy for distant pairs. A segment pair whose closest endpoint
//    distance is below near_factor x (longer segment length) is recomputed
//    in FP64 (near-singular terms).
// Item results go to one FP64 partial per item; a second kernel sums them
// per pair in a fixed order, so results are deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>
#include <string>

#include "engine.hpp"

namespace fln {
namespace {

constexpr int kBlockSegs = 128;  // default: threads per CTA = curve-1 segments per item
constexpr int kTile = 256;       // default: curve-2 vertices per shared-memory tile
constexpr double kInvTwoPi = 0.15915494309189533576888376337251436;

struct DirectArgs {
  const double *xyz;          // 3 doubles per vertex
  const int64_t *off;         // loop offsets
  const int32_t *loops;       // per slot: (curve-1 loop, curve-2 loop)
  const int64_t *item_start;  // per slot: first item; nslots + 1 entries
  int32_t nslots;
  int64_t items;
  double *partial;                   // per item
  unsigned long long *counter;       // [0] work queue head, [1] near-term count
  float near_factor;
};

__device__ __forceinline__ int find_slot(const int64_t *start, int n, int64_t item) {
  int lo = 0, hi = n;  // start[lo] <= item < start[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(start + mid) <= item) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ double3 load_v(const double *xyz, int64_t v) {
  return make_double3(__ldg(xyz + 3 * v), __ldg(xyz + 3 * v + 1), __ldg(xyz + 3 * v + 2));
}

// Sum over the CTA of kB threads; the result is valid in thread 0.
template <int kB>
__device__ __forceinline__ double block_sum(double v, double *s_red) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kB / 32; ++w) r += s_red[w];
  return r;
}

// One segment pair in FP64, in full turns (OneArctanPerPair form,
// compute_link.cpp:151-175 divided by 4 pi).
__device__ __noinline__ double term_fp64(double3 p0, double3 p1, double3 q0, double3 q1) {
  const double ax = q0.x - p0.x, ay = q0.y - p0.y, az = q0.z - p0.z;
  const double bx = q0.x - p1.x, by = q0.y - p1.y, bz = q0.z - p1.z;
  const double cx = q1.x - p1.x, cy = q1.y - p1.y, cz = q1.z - p1.z;
  const double dx = q1.x - p0.x, dy = q1.y - p0.y, dz = q1.z - p0.z;
  const double la = sqrt(ax * ax + ay * ay + az * az), lb = sqrt(bx * bx + by * by + bz * bz);
  const double lc = sqrt(cx * cx + cy * cy + cz * cz), ld = sqrt(dx * dx + dy * dy + dz * dz);
  const double ca = cx * ax + cy * ay + cz * az;
  const double div1 = la * lb * lc + (ax * bx + ay * by + az * bz) * lc + ca * lb + (cx * bx + cy * by + cz * bz) * la;
  const double div2 = la * ld * lc + (ax * dx + ay * dy + az * dz) * lc + ca * ld + (cx * dx + cy * dy + cz * dz) * la;
  const double det = ax * (by * cz - bz * cy) + az * (bx * cy - by * cx) + ay * (bz * cx - bx * cz);
  const double xp = div1 * div2 - det * det, yp = det * (div1 + div2);
  double r = atan2(yp, xp) * kInvTwoPi;
  if (yp * det < 0) r += (det > 0) ? 1.0 : -1.0;
  return r;
}

// Rescales (x, y) by the power of two that brings max(|x|, |y|) into [1, 2).
__device__ __forceinline__ void renorm(double &x, double &y) {
  const double m = fmax(fabs(x), fabs(y));
  int e = (__double2hiint(m) >> 20) & 0x7ff;
  e = min(max(e, 1), 2045);
  const double s = __hiloint2double((2046 - e) << 20, 0);
  x *= s;
  y *= s;
}

// ------------------------------------------------------------------ FP64
// Tile shape: kB threads per CTA (= curve-1 segments per item), kT curve-2
// vertices per shared-memory tile.
template <int kB, int kT>
__global__ void __launch_bounds__(kB) direct_fp64_kernel(DirectArgs A) {
  __shared__ double sx[kT + 1], sy[kT + 1], sz[kT + 1];
  __shared__ double s_red[kB / 32];
  __shared__ long long s_item;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(A.counter, 1ULL);
    __syncthreads();
    const int64_t item = s_item;
    if (item >= A.items) break;
    const int slot = find_slot(A.item_start, A.nslots, item);
    const int64_t blk = item - A.item_start[slot];
    const int l1 = A.loops[2 * slot], l2 = A.loops[2 * slot + 1];
    const int64_t o1 = A.off[l1], n1 = A.off[l1 + 1] - o1;
    const int64_t o2 = A.off[l2], n2 = A.off[l2 + 1] - o2;
    const int64_t i = blk * kB + threadIdx.x;
    const bool active = i < n1;
    double3 p0 = make_double3(0, 0, 0), p1 = p0;
    if (active) {
      p0 = load_v(A.xyz, o1 + i);
      p1 = load_v(A.xyz, o1 + (i + 1 == n1 ? 0 : i + 1));
    }
    double xs = 1.0, ys = 0.0, S = -1.0, turns = 0.0;
    for (int64_t k0 = 0; k0 < n2; k0 += kT) {
      const int kt = (int)(n2 - k0 < kT ? n2 - k0 : kT);
      __syncthreads();
      for (int t = threadIdx.x; t <= kt; t += kB) {
        const int64_t kk = k0 + t;
        const double3 v = load_v(A.xyz, o2 + (kk == n2 ? 0 : kk));
        sx[t] = v.x;
        sy[t] = v.y;
        sz[t] = v.z;
      }
      __syncthreads();
      if (!active) continue;
      double ax = sx[0] - p0.x, ay = sy[0] - p0.y, az = sz[0] - p0.z;
      double bx = sx[0] - p1.x, by = sy[0] - p1.y, bz = sz[0] - p1.z;
      double la = sqrt(ax * ax + ay * ay + az * az), lb = sqrt(bx * bx + by * by + bz * bz);
      double ab = ax * bx + ay * by + az * bz;
      for (int k = 0; k < kt; ++k) {
        const double qx = sx[k + 1], qy = sy[k + 1], qz = sz[k + 1];
        const double cx = qx - p1.x, cy = qy - p1.y, cz = qz - p1.z;
        const double dx = qx - p0.x, dy = qy - p0.y, dz = qz - p0.z;
        const double lc = sqrt(cx * cx + cy * cy + cz * cz), ld = sqrt(dx * dx + dy * dy + dz * dz);
        const double ca = cx * ax + cy * ay + cz * az;
        const double cb = cx * bx + cy * by + cz * bz;
        const double ad = ax * dx + ay * dy + az * dz;
        const double cd = cx * dx + cy * dy + cz * dz;
        const double det = ax * (by * cz - bz * cy) + az * (bx * cy - by * cx) + ay * (bz * cx - bx * cz);
        const double t = la * lc;
        const double div1 = t * lb + ab * lc + ca * lb + cb * la;
        const double div2 = t * ld + ad * lc + ca * ld + cd * la;
        const double xp = div1 * div2 - det * det;
        const double yp = det * (div1 + div2);
        // Arctangent addition: (xs + i ys) *= (xp + i yp), tracking crossings
        // of the negative real axis (compute_link.cpp:245-269).
        double ny = xs * yp + xp * ys;
        double nx = xs * xp - ys * yp;
        renorm(nx, ny);
        if (yp * det < 0) turns += (det > 0) ? 1.0 : -1.0;
        const double s3 = (ny > 0.0 || (ny == 0.0 && nx < 0.0)) ? 1.0 : -1.0;
        if (s3 * S < 0 && yp * S >= 0) turns += S;
        xs = nx;
        ys = ny;
        S = s3;
        ax = dx; ay = dy; az = dz;
        bx = cx; by = cy; bz = cz;
        la = ld; lb = lc; ab = cd;
      }
    }
    const double v = active ? atan2(ys, xs) * kInvTwoPi + turns : 0.0;
    const double s = block_sum<kB>(v, s_red);
    if (threadIdx.x == 0) A.partial[item] = s;
  }
}

// ------------------------------------------------------------------ mixed
// arctan(t) for |t| <= 1/4 from its Maclaurin series t - t^3/3 + t^5/5 - t^7/7
// + t^9/9; the first omitted term is below 2.2e-8 |t|, under FP32 rounding.
__device__ __forceinline__ float atan_small(float t) {
  const float u = t * t;
  float p = fmaf(u, 1.0f / 9.0f, -1.0f / 7.0f);
  p = fmaf(p, u, 1.0f / 5.0f);
  p = fmaf(p, u, -1.0f / 3.0f);
  p = fmaf(p, u, 1.0f);
  return p * t;
}

// Minimum and maximum over the CTA of 7 values each (a box and a length);
// the result is in out[0..6] (min) and out[7..13] (max) for every thread.
template <int kB>
__device__ __forceinline__ void block_minmax7(float *lo, float *hi, float (*s_box)[14], float *out) {
  for (int o = 16; o; o >>= 1)
    for (int v = 0; v < 7; ++v) {
      lo[v] = fminf(lo[v], __shfl_xor_sync(0xffffffffu, lo[v], o));
      hi[v] = fmaxf(hi[v], __shfl_xor_sync(0xffffffffu, hi[v], o));
    }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int v = 0; v < 7; ++v) {
      s_box[warp][v] = lo[v];
      s_box[warp][7 + v] = hi[v];
    }
  __syncthreads();
  for (int v = 0; v < 14; ++v) {
    float r = s_box[0][v];
    for (int w = 1; w < kB / 32; ++w) r = v < 7 ? fminf(r, s_box[w][v]) : fmaxf(r, s_box[w][v]);
    out[v] = r;
  }
}

// Accumulation of a thread's terms over a tile: 0 = FP32 over the tile
// (up to kT terms), 1 = FP32 with Kahan compensation, 2 = FP64 per term,
// 3 = FP32 runs of 32 terms folded into FP64 (the rounding error of a run is
// bounded by 32 terms instead of kT, for one FP64 add per 32 terms).
#ifndef FLN_MIXED_ACC
#define FLN_MIXED_ACC 3
#endif

template <int kB, int kT>
__global__ void __launch_bounds__(kB) direct_mixed_kernel(DirectArgs A) {
  __shared__ float4 sq[kT + 1];  // xyz relative to the tile origin; w = length of segment t
  __shared__ double s_red[kB / 32];
  __shared__ float s_box[kB / 32][14];
  __shared__ long long s_item;
  const float INF = __int_as_float(0x7f800000);
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(A.counter, 1ULL);
    __syncthreads();
    const int64_t item = s_item;
    if (item >= A.items) break;
    const int slot = find_slot(A.item_start, A.nslots, item);
    const int64_t blk = item - A.item_start[slot];
    const int l1 = A.loops[2 * slot], l2 = A.loops[2 * slot + 1];
    const int64_t o1 = A.off[l1], n1 = A.off[l1 + 1] - o1;
    const int64_t o2 = A.off[l2], n2 = A.off[l2 + 1] - o2;
    const int64_t i = blk * kB + threadIdx.x;
    const bool active = i < n1;
    double3 p0 = make_double3(0, 0, 0), p1 = p0;
    if (active) {
      p0 = load_v(A.xyz, o1 + i);
      p1 = load_v(A.xyz, o1 + (i + 1 == n1 ? 0 : i + 1));
    }
    const float ex = (float)(p1.x - p0.x), ey = (float)(p1.y - p0.y), ez = (float)(p1.z - p0.z);
    const float len1 = sqrtf(ex * ex + ey * ey + ez * ez);
    double acc = 0.0, near_turns = 0.0;
    int turns = 0;
    unsigned near_count = 0;
    for (int64_t k0 = 0; k0 < n2; k0 += kT) {
      const int kt = (int)(n2 - k0 < kT ? n2 - k0 : kT);
      const double3 O = load_v(A.xyz, o2 + k0);
      __syncthreads();
      for (int t = threadIdx.x; t <= kt; t += kB) {
        const int64_t kk = k0 + t;
        const double3 v = load_v(A.xyz, o2 + (kk == n2 ? 0 : kk));
        sq[t] = make_float4((float)(v.x - O.x), (float)(v.y - O.y), (float)(v.z - O.z), 0.f);
      }
      __syncthreads();
      const float r0x = (float)(p0.x - O.x), r0y = (float)(p0.y - O.y), r0z = (float)(p0.z - O.z);
      const float r1x = (float)(p1.x - O.x), r1y = (float)(p1.y - O.y), r1z = (float)(p1.z - O.z);
      // Boxes of this thread's curve-1 segment (slots 0-2, length 3) and of
      // its curve-2 tile vertices (slots 4-6, length 3 of the max).
      float lo[7], hi[7];
      for (int v = 0; v < 7; ++v) {
        lo[v] = INF;
        hi[v] = -INF;
      }
      if (active) {
        lo[0] = fminf(r0x, r1x); hi[0] = fmaxf(r0x, r1x);
        lo[1] = fminf(r0y, r1y); hi[1] = fmaxf(r0y, r1y);
        lo[2] = fminf(r0z, r1z); hi[2] = fmaxf(r0z, r1z);
        hi[3] = len1;
      }
      for (int t = threadIdx.x; t < kt; t += kB) {
        const float4 a = sq[t], b = sq[t + 1];
        const float fx = b.x - a.x, fy = b.y - a.y, fz = b.z - a.z;
        const float len = sqrtf(fx * fx + fy * fy + fz * fz);
        sq[t].w = len;
        lo[4] = fminf(lo[4], fminf(a.x, b.x)); hi[4] = fmaxf(hi[4], fmaxf(a.x, b.x));
        lo[5] = fminf(lo[5], fminf(a.y, b.y)); hi[5] = fmaxf(hi[5], fmaxf(a.y, b.y));
        lo[6] = fminf(lo[6], fminf(a.z, b.z)); hi[6] = fmaxf(hi[6], fmaxf(a.z, b.z));
        hi[3] = fmaxf(hi[3], len);
      }
      float bx[14];
      block_minmax7<kB>(lo, hi, s_box, bx);
      __syncthreads();
      // Box gap between the CTA's curve-1 segments and this tile: no segment
      // pair can be near-singular when it exceeds near_factor x (longest segment).
      const float gx = fmaxf(0.f, fmaxf(bx[4] - bx[7], bx[0] - bx[11]));
      const float gy = fmaxf(0.f, fmaxf(bx[5] - bx[8], bx[1] - bx[12]));
      const float gz = fmaxf(0.f, fmaxf(bx[6] - bx[9], bx[2] - bx[13]));
      const float lim = A.near_factor * bx[10];
      const bool far_tile = gx * gx + gy * gy + gz * gz > 1.0001f * lim * lim;
      if (!active) continue;
      float4 q = sq[0];
      float ax = q.x - r0x, ay = q.y - r0y, az = q.z - r0z;
      float bx_ = q.x - r1x, by = q.y - r1y, bz = q.z - r1z;
      float la = sqrtf(ax * ax + ay * ay + az * az), lb = sqrtf(bx_ * bx_ + by * by + bz * bz);
      float ab = ax * bx_ + ay * by + az * bz;
      float accf = 0.f;
#if FLN_MIXED_ACC == 1
      float comp = 0.f;  // Kahan compensation of accf
#elif FLN_MIXED_ACC == 2
      double accd = 0.0;
#endif
      for (int k = 0; k < kt; ++k) {
        const float4 qn = sq[k + 1];
        const float cx = qn.x - r1x, cy = qn.y - r1y, cz = qn.z - r1z;
        const float dx = qn.x - r0x, dy = qn.y - r0y, dz = qn.z - r0z;
        const float cc = cx * cx + cy * cy + cz * cz, dd = dx * dx + dy * dy + dz * dz;
        const float lc = cc * rsqrtf(cc), ld = dd * rsqrtf(dd);
        const float cd = cx * dx + cy * dy + cz * dz;
        bool near = false;
        if (!far_tile) near = fminf(fminf(la, lb), fminf(lc, ld)) < A.near_factor * fmaxf(len1, q.w);
        if (near) {
          const int64_t kk = k0 + k, kn = kk + 1;
          near_turns += term_fp64(p0, p1, load_v(A.xyz, o2 + kk), load_v(A.xyz, o2 + (kn == n2 ? 0 : kn)));
          ++near_count;
        } else {
          const float ca = cx * ax + cy * ay + cz * az;
          const float cb = cx * bx_ + cy * by + cz * bz;
          const float ad = ax * dx + ay * dy + az * dz;
          const float fx = qn.x - q.x, fy = qn.y - q.y, fz = qn.z - q.z;
          const float det = ax * (fy * ez - fz * ey) + ay * (fz * ex - fx * ez) + az * (fx * ey - fy * ex);
          const float t = la * lc;
          const float div1 = t * lb + ab * lc + ca * lb + cb * la;
          const float div2 = t * ld + ad * lc + ca * ld + cd * la;
          const float sdiv = div1 + div2;
          const float xp = div1 * div2 - det * det;
          const float yp = det * sdiv;
          float term;
          if (sdiv > 0.f && fabsf(yp) < 0.25f * xp) {
            term = atan_small(__fdividef(yp, xp));  // principal branch, |angle| < 0.245
          } else {
            term = atan2f(yp, xp);
            if (sdiv < 0.f && det != 0.f) turns += (det > 0.f) ? 1 : -1;
          }
#if FLN_MIXED_ACC == 1
          const float y_ = term - comp;
          const float t_ = accf + y_;
          comp = (t_ - accf) - y_;
          accf = t_;
#elif FLN_MIXED_ACC == 2
          accd += (double)term;
#else
          accf += term;
#endif
        }
#if FLN_MIXED_ACC == 3
        if ((k & 31) == 31) {
          acc += (double)accf;
          accf = 0.f;
        }
#endif
        q = qn;
        ax = dx; ay = dy; az = dz;
        bx_ = cx; by = cy; bz = cz;
        la = ld; lb = lc; ab = cd;
      }
#if FLN_MIXED_ACC == 1
      acc += (double)accf - (double)comp;
#elif FLN_MIXED_ACC == 2
      acc += accd;
#else
      acc += (double)accf;
#endif
    }
    const double v = active ? acc * kInvTwoPi + (double)turns + near_turns : 0.0;
    const double s = block_sum<kB>(v, s_red);
    if (threadIdx.x == 0) A.partial[item] = s;
    if (near_count) atomicAdd(A.counter + 1, (unsigned long long)near_count);
  }
}

// Sums the item partials of each slot in item order and scatters the result
// to the caller's pair index.
__global__ void reduce_items_kernel(const double *partial, const int64_t *item_start, const int32_t *order,
                                    int32_t nslots, double *lk_out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  double acc = 0.0;
  for (int64_t it = item_start[s]; it < item_start[s + 1]; ++it) acc += partial[it];
  lk_out[order[s]] = acc;
}

// The tile shapes the direct sum can run with (fln_params.direct_tile), the
// default first: (curve-1 segments per item = threads per CTA, curve-2
// vertices per shared-memory tile).
struct TileShape {
  int block, tile;
};
constexpr TileShape kShapes[kDirectTileShapes] = {{128, 256}, {128, 128}, {128, 512},
                                                  {256, 256}, {256, 512}, {64, 256}};
static_assert(kShapes[0].block == kBlockSegs && kShapes[0].tile == kTile, "the default shape comes first");

template <int kB, int kT>
void launch_direct_t(cudaStream_t st, int sms, int precision, const DirectArgs &A) {
  if (precision == FLN_PREC_FP64) {
    const int per_sm = occupancy_of((const void *)direct_fp64_kernel<kB, kT>, kB);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(A.items, (int64_t)sms * per_sm));
    direct_fp64_kernel<kB, kT><<<grid, kB, 0, st>>>(A);
  } else {
    const int per_sm = occupancy_of((const void *)direct_mixed_kernel<kB, kT>, kB);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(A.items, (int64_t)sms * per_sm));
    direct_mixed_kernel<kB, kT><<<grid, kB, 0, st>>>(A);
  }
}

void launch_direct(int shape, cudaStream_t st, int sms, int precision, const DirectArgs &A) {
  switch (shape) {
    case 1: launch_direct_t<128, 128>(st, sms, precision, A); break;
    case 2: launch_direct_t<128, 512>(st, sms, precision, A); break;
    case 3: launch_direct_t<256, 256>(st, sms, precision, A); break;
    case 4: launch_direct_t<256, 512>(st, sms, precision, A); break;
    case 5: launch_direct_t<64, 256>(st, sms, precision, A); break;
    default: launch_direct_t<kBlockSegs, kTile>(st, sms, precision, A); break;
  }
}

}  // namespace

int direct_sum_device(Context &ctx, const double *d_xyz, const int64_t *d_off, const std::vector<int64_t> &h_off,
                      const std::vector<int32_t> &h_pairs, int precision, double near_factor, double *d_lk_out,
                      double *near_terms_out, int tile_shape) {
  if (tile_shape < 0 || tile_shape >= kDirectTileShapes)
    throw Error(FLN_ERR_INVALID_ARGUMENT, "direct_tile in [0, " + std::to_string(kDirectTileShapes - 1) + "]");
  const int kB = kShapes[tile_shape].block;
  const int64_t np = (int64_t)h_pairs.size() / 2;
  if (np == 0) return 0;
  // Plan: orient each pair so its longer loop is curve 1, and order slots by
  // decreasing work so the queue hands out the largest pairs first.
  std::vector<int32_t> order(np);
  std::iota(order.begin(), order.end(), 0);
  auto nseg = [&](int l) { return h_off[l + 1] - h_off[l]; };
  std::vector<double> cost(np);
  for (int64_t p = 0; p < np; ++p) cost[p] = (double)nseg(h_pairs[2 * p]) * (double)nseg(h_pairs[2 * p + 1]);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<int32_t> loops(2 * np);
  std::vector<int64_t> start(np + 1);
  start[0] = 0;
  for (int64_t s = 0; s < np; ++s) {
    int a = h_pairs[2 * order[s]], b = h_pairs[2 * order[s] + 1];
    if (nseg(b) > nseg(a)) std::swap(a, b);
    loops[2 * s] = a;
    loops[2 * s + 1] = b;
    start[s + 1] = start[s] + (nseg(a) + kB - 1) / kB;
  }
  const int64_t items = start[np];
  int32_t *d_loops = ctx.d_loops.as<int32_t>(2 * np + np);
  int32_t *d_order = d_loops + 2 * np;
  int64_t *d_start = ctx.d_items.as<int64_t>(np + 1);
  double *d_partial = ctx.d_partial.as<double>(items);
  unsigned long long *d_counter = ctx.d_counter.as<unsigned long long>(2);
  FLN_CUDA(cudaMemcpyAsync(d_loops, loops.data(), 2 * np * sizeof(int32_t), cudaMemcpyHostToDevice, ctx.stream));
  FLN_CUDA(cudaMemcpyAsync(d_order, order.data(), np * sizeof(int32_t), cudaMemcpyHostToDevice, ctx.stream));
  FLN_CUDA(cudaMemcpyAsync(d_start, start.data(), (np + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, ctx.stream));
  FLN_CUDA(cudaMemsetAsync(d_counter, 0, 2 * sizeof(unsigned long long), ctx.stream));
  DirectArgs A{d_xyz, d_off, d_loops, d_start, (int32_t)np, items, d_partial, d_counter, (float)near_factor};
  FLN_CUDA(cudaEventRecord(ctx.ev2, ctx.stream));
  launch_direct(tile_shape, ctx.stream, ctx.num_sms, precision, A);
  FLN_CUDA(cudaGetLastError());
  FLN_CUDA(cudaEventRecord(ctx.ev3, ctx.stream));
  reduce_items_kernel<<<(int)((np + 255) / 256), 256, 0, ctx.stream>>>(d_partial, d_start, d_order, (int32_t)np,
                                                                      d_lk_out);
  FLN_CUDA(cudaGetLastError());
  if (near_terms_out) {
    unsigned long long h = 0;
    FLN_CUDA(cudaMemcpyAsync(&h, d_counter + 1, sizeof h, cudaMemcpyDeviceToHost, ctx.stream));
    FLN_CUDA(cudaStreamSynchronize(ctx.stream));
    *near_terms_out = (double)h;
  }
  ctx.stats.ms_main_kernel += ctx.elapsed(ctx.ev2, ctx.ev3);
  return 2;
}

}  // namespace fln

// ---------------------------------------------------------------------------
// Direct sum that allocates nothing (fln_linking_numbers_direct_noalloc).
//
// Some callers cannot call cudaMalloc: code that runs while another framework
// owns the device's memory pool (a renderer or simulator with its own
// allocator and a fixed budget), code that must not add allocator
// synchronisation or fragmentation to a latency-critical loop, and code on
// paths where an allocation failure cannot be handled. For them the direct
// sum runs entirely in the caller's input and output buffers plus one
// file-scope device array, g_noalloc_scratch, of kNoAllocScratchBytes
// (about 9.3 MB). Every GPU that loads libfln.so holds that array until the
// process exits. Limits: at most kNoAllocMaxPairs loop pairs per call and
// kNoAllocMaxItems work items (one item = 128 segments of the longer loop of
// a pair, summed over the pairs); larger calls are rejected with
// FLN_ERR_INVALID_ARGUMENT before any kernel runs on them. The mixed
// precision uses the default near factor (kDefaultNearFactor), so results
// equal the allocating entry point's with fln_default_params.
//
// Every call copies the plan's header (item count, status) back to the host
// and waits for it: the call blocks until the work queued earlier on the
// stream and the planning kernel have run.
//
// In host code the name g_noalloc_scratch only stands for the array: its
// device address is obtained once per device with cudaGetSymbolAddress, on
// the first call made with that device current, and cached. That first call
// therefore does the set-up and should come before any stream capture.
// All calls share the array and it keeps the previous call's contents: the
// planning kernel clears the work-queue counters at the start of every call.
// Calls whose work overlaps on the GPU (different streams, or host threads
// racing) race on the array; issue them one after another.
namespace fln {
namespace {

constexpr int64_t kNoAllocMaxPairs = 65536;
constexpr int64_t kNoAllocMaxItems = int64_t(1) << 20;
constexpr size_t kNaHeader = 256;  // counters[2], total items, status
constexpr size_t kNaLoops = kNaHeader;                                       // int32 x 2 per pair
constexpr size_t kNaOrder = kNaLoops + 2 * kNoAllocMaxPairs * 4;             // int32 per pair
constexpr size_t kNaStart = kNaOrder + kNoAllocMaxPairs * 4;                 // int64 per pair + 1
constexpr size_t kNaPartial = (kNaStart + (kNoAllocMaxPairs + 1) * 8 + 255) / 256 * 256;  // double per item
constexpr size_t kNoAllocScratchBytes = kNaPartial + kNoAllocMaxItems * 8;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NaHeader {
  unsigned long long counter[2];  // work queue head, near-singular term count
  long long total_items;
  int status;                     // bit 0: bad pair index, bit 1: loop with < 2 vertices
};

// One CTA plans the call inside the scratch array: orients each pair (longer
// loop first), counts its items, scans them into item_start and clears the
// counters the direct-sum kernels start from.
__global__ void __launch_bounds__(1024) noalloc_plan(const int64_t *off, int32_t nloops, const int32_t *pairs,
                                                     int64_t npairs, unsigned char *scratch) {
  NaHeader *h = reinterpret_cast<NaHeader *>(scratch);
  int32_t *loops = reinterpret_cast<int32_t *>(scratch + kNaLoops);
  int32_t *order = reinterpret_cast<int32_t *>(scratch + kNaOrder);
  int64_t *start = reinterpret_cast<int64_t *>(scratch + kNaStart);
  __shared__ long long s_warp[32];
  __shared__ long long s_carry;
  __shared__ int s_status;
  if (threadIdx.x == 0) {
    s_carry = 0;
    s_status = 0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = 0; base < npairs; base += 1024) {
    const int64_t p = base + threadIdx.x;
    long long items = 0;
    if (p < npairs) {
      int a = pairs[2 * p], b = pairs[2 * p + 1];
      if (a < 0 || a >= nloops || b < 0 || b >= nloops || a == b) {
        atomicOr(&s_status, 1);
      } else {
        int64_t na = off[a + 1] - off[a], nb = off[b + 1] - off[b];
        if (na < 2 || nb < 2) {
          atomicOr(&s_status, 2);
        } else {
          if (nb > na) {
            const int t = a;
            a = b;
            b = t;
            const int64_t tn = na;
            na = nb;
            nb = tn;
          }
          items = (na + kBlockSegs - 1) / kBlockSegs;
        }
      }
      loops[2 * p] = a;
      loops[2 * p + 1] = b;
      order[p] = (int32_t)p;
    }
    // Exclusive block scan of `items`.
    long long incl = items;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      long long v = s_warp[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
      }
      s_warp[lane] = v;  // inclusive over warps
    }
    __syncthreads();
    const long long warp_base = warp ? s_warp[warp - 1] : 0;
    if (p < npairs) start[p] = s_carry + warp_base + incl - items;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += s_warp[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    start[npairs] = s_carry;
    h->counter[0] = 0;
    h->counter[1] = 0;
    h->total_items = s_carry;
    h->status = s_status;
  }
}

// Device address of g_noalloc_scratch per device, set up on first use.
void *noalloc_scratch_for_current_device(fln_status &st, std::string &msg) {
  static void *addr[64] = {nullptr};
  static std::mutex mu;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    st = e == cudaSuccess ? FLN_ERR_INVALID_ARGUMENT : FLN_ERR_NO_DEVICE;
    msg = std::string("cudaGetDevice: ") + (e == cudaSuccess ? "device index >= 64" : cudaGetErrorString(e));
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      st = FLN_ERR_CUDA;
      msg = std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e);
      return nullptr;
    }
    addr[dev] = p;
  }
  return addr[dev];
}

}  // namespace

// Records the message behind a non-OK status for fln_last_error() (capi.cpp).
void set_last_error(const std::string &msg);

}  // namespace fln

extern "C" fln_status fln_linking_numbers_direct_noalloc(const double *d_xyz, const int64_t *d_loop_offsets,
                                                         int32_t nloops, const int32_t *d_pairs, int64_t npairs,
                                                         int32_t precision, double *d_lk_out, void *stream) {
  using namespace fln;
  auto fail = [](fln_status s, const std::string &m) {
    set_last_error(m);
    return s;
  };
  if (npairs < 0 || npairs > kNoAllocMaxPairs)
    return fail(FLN_ERR_INVALID_ARGUMENT, "fln_linking_numbers_direct_noalloc: npairs must be in [0, " +
                                              std::to_string(kNoAllocMaxPairs) + "], got " + std::to_string(npairs));
  if (nloops < 0 || (npairs > 0 && (!d_xyz || !d_loop_offsets || !d_pairs || !d_lk_out)))
    return fail(FLN_ERR_INVALID_ARGUMENT, "fln_linking_numbers_direct_noalloc: NULL or negative argument");
  if (precision != FLN_PREC_FP64 && precision != FLN_PREC_MIXED)
    return fail(FLN_ERR_INVALID_ARGUMENT, "fln_linking_numbers_direct_noalloc: unknown precision");
  if (npairs == 0) return FLN_OK;
  fln_status st = FLN_OK;
  std::string msg;
  unsigned char *scratch = static_cast<unsigned char *>(noalloc_scratch_for_current_device(st, msg));
  if (!scratch) return fail(st, msg);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  noalloc_plan<<<1, 1024, 0, s>>>(d_loop_offsets, nloops, d_pairs, npairs, scratch);
  NaHeader h;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, scratch, sizeof h, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(FLN_ERR_CUDA, std::string("fln_linking_numbers_direct_noalloc: ") + cudaGetErrorString(e));
  if (h.status & 1) return fail(FLN_ERR_INVALID_ARGUMENT, "fln_linking_numbers_direct_noalloc: pair index out of range or a pair names one loop twice");
  if (h.status & 2) return fail(FLN_ERR_INVALID_ARGUMENT, "fln_linking_numbers_direct_noalloc: every loop in a pair needs at least two vertices");
  if (h.total_items > kNoAllocMaxItems)
    return fail(FLN_ERR_INVALID_ARGUMENT, "fln_linking_numbers_direct_noalloc: " + std::to_string(h.total_items) +
                                              " work items exceed the limit of " + std::to_string(kNoAllocMaxItems) +
                                              " (one item = 128 segments of the longer loop of a pair)");
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // The default tile shape (the planning kernel cuts items of kBlockSegs).
  DirectArgs A{d_xyz, d_loop_offsets, reinterpret_cast<const int32_t *>(scratch + kNaLoops),
               reinterpret_cast<const int64_t *>(scratch + kNaStart), (int32_t)npairs, h.total_items,
               reinterpret_cast<double *>(scratch + kNaPartial), reinterpret_cast<unsigned long long *>(scratch),
               (float)kDefaultNearFactor};
  if (precision == FLN_PREC_FP64) {
    per_sm = occupancy_of((const void *)direct_fp64_kernel<kBlockSegs, kTile>, kBlockSegs);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(h.total_items, (int64_t)sms * std::max(per_sm, 1)));
    direct_fp64_kernel<kBlockSegs, kTile><<<grid, kBlockSegs, 0, s>>>(A);
  } else {
    per_sm = occupancy_of((const void *)direct_mixed_kernel<kBlockSegs, kTile>, kBlockSegs);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(h.total_items, (int64_t)sms * std::max(per_sm, 1)));
    direct_mixed_kernel<kBlockSegs, kTile><<<grid, kBlockSegs, 0, s>>>(A);
  }
  reduce_items_kernel<<<(int)((npairs + 255) / 256), 256, 0, s>>>(
      reinterpret_cast<const double *>(scratch + kNaPartial), reinterpret_cast<const int64_t *>(scratch + kNaStart),
      reinterpret_cast<const int32_t *>(scratch + kNaOrder), (int32_t)npairs, d_lk_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(FLN_ERR_CUDA, std::string("fln_linking_numbers_direct_noalloc: ") + cudaGetErrorString(e));
  return FLN_OK;
}
