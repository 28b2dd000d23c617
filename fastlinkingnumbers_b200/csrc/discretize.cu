// Discretize on the GPU: the adaptive refinement of discretize.cpp:103-281
// with the potential-link searches around it (potential_link_search.cpp:
// 88-165), producing the same closed polylines and pairs as the host path
// (host.cpp) bit for bit.
//
// Each round, every live piece whose closed box meets a live piece box of
// another, potentially linked curve is halved in t; the others become final.
// The refined set depends only on the piece boxes and the closed-interval
// predicate, so any exact broad phase gives the same result. Here:
//
// - All pieces of all curves live in one array sorted by (curve, segment,
//   t0). A round rewrites it through a scan (a hit piece emits its two
//   halves, every other piece itself), so it stays sorted and the output
//   polyline of a curve is the start point of each of its pieces in order.
// - The live pieces of a curve form a curve-order box tree (node = range of
//   live pieces, split at the middle; internal node id = split - 1, leaf id =
//   m - 1 + position), built bottom-up with acquire-release arrival counters.
// - A two-tree walk per potential pair marks the pieces of overlapping leaf
//   pairs. Warps take batches of up to 32 node pairs from a queue and work a
//   batch for at most kBudget steps; what is left (or what overflows the
//   shared stack) is handed on as new batches of the next launch.
//
// Piece boxes come from seg_box (geometry.hpp), the host's own code. This
// file is compiled with --fmad=false and CUDA's correctly rounded division
// and square root, so the boxes are the host's bit for bit.
#include <cub/cub.cuh>
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

#include "engine.hpp"
#include "geometry.hpp"

namespace fln {

namespace {

constexpr int kDWarps = 4;
constexpr int kDStack = 256;  // shared stack entries per warp
constexpr int kBudget = 256;  // steps per batch and launch

struct DNode {
  double lo[3], hi[3];
  int32_t a, b;  // range [a, b) of the curve's live pieces
};

struct DBatch {
  int32_t slot;
  int32_t count;
  int2 pairs[32];
};

struct CurveSet {
  const double *cp;       // control points, 3 doubles each
  const int64_t *cp_off;  // curve -> first control point; nc + 1
  const int32_t *kind;    // SegKind per curve
};

struct Pieces {
  int32_t *c, *s;
  double *t0, *t1;
  uint8_t *live;
};

__device__ __forceinline__ int find_curve(const int64_t *start, int n, int64_t x) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (start[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Order-preserving key of a non-negative double (NaN above +inf).
__device__ __forceinline__ unsigned long long dkey(double v) { return (unsigned long long)__double_as_longlong(v); }

// count[key] += 1 for the calling lane, one atomic per distinct key of the
// warp (neighbouring pieces mostly belong to the same curve).
__device__ __forceinline__ void add_one(int32_t *count, int32_t key, bool active) {
  const unsigned act = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const unsigned peers = __match_any_sync(act, key);
  if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&count[key], __popc(peers));
}

__global__ void init_pieces(const int64_t *seg_off, int nc, int64_t total, Pieces P) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int c = find_curve(seg_off, nc, g);
  P.c[g] = c;
  P.s[g] = (int32_t)(g - seg_off[c]);
  P.t0[g] = 0.0;
  P.t1[g] = 1.0;
  P.live[g] = 1;
}

__global__ void flag_live(const uint8_t *live, int64_t n, int32_t *flag) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) flag[k] = live[k];
}

__global__ void compact_live(const uint8_t *live, const int32_t *pos, const int32_t *curve, int64_t n, int32_t *lidx,
                             int32_t *count_per_curve) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool on = k < n && live[k];
  if (on) lidx[pos[k]] = (int32_t)k;
  add_one(count_per_curve, on ? curve[k] : 0, on);
}

// Leaf records of the live pieces: the piece box and its range; the minimum
// box diagonal (Discretize's "segment too small" test) by an atomic on the
// order-preserving bit pattern.
__global__ void leaf_records(CurveSet C, Pieces P, const int32_t *lidx, const int64_t *loff, int64_t L, DNode *nodes,
                             unsigned long long *min_diag) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double d = INFINITY;
  if (q < L) {
    const int32_t k = lidx[q];
    const int c = P.c[k];
    const int64_t m = loff[c + 1] - loff[c], pos = q - loff[c];
    DNode nd;
    const int64_t o = C.cp_off[c], ncp = C.cp_off[c + 1] - o;
    seg_box(C.kind[c], C.cp + 3 * o, ncp, P.s[k], P.t0[k], P.t1[k], nd.lo, nd.hi);
    nd.a = (int32_t)pos;
    nd.b = (int32_t)pos + 1;
    nodes[2 * loff[c] + (m - 1) + pos] = nd;
    const double dx = nd.hi[0] - nd.lo[0], dy = nd.hi[1] - nd.lo[1], dz = nd.hi[2] - nd.lo[2];
    d = sqrt(dx * dx + dy * dy + dz * dz);
  }
  for (int o = 16; o; o >>= 1) d = fmin(d, __shfl_xor_sync(0xffffffffu, d, o));
  if ((threadIdx.x & 31) == 0 && d < INFINITY) atomicMin(min_diag, dkey(d));
}

// Internal nodes: range by descent from the root, children and parents.
// Thread per internal node; int_off[c] = sum over earlier curves of (m - 1).
__global__ void internal_topology(const int64_t *loff, const int64_t *int_off, int nc, int64_t total_int,
                                  DNode *nodes, int32_t *child, int32_t *parent, int32_t *arrive) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total_int) return;
  const int c = find_curve(int_off, nc, g);
  const int64_t m = loff[c + 1] - loff[c], base = 2 * loff[c];
  const int32_t node = (int32_t)(g - int_off[c]);
  const int64_t s = node + 1;
  int64_t lo = 0, hi = m;
  int32_t par = -1;
  for (int depth = 0; depth < 64; ++depth) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (mid == s) break;
    par = (int32_t)(mid - 1);
    if (s < mid) hi = mid;
    else lo = mid;
  }
  const int32_t leaf0 = (int32_t)(m - 1);
  const int32_t left = (s - lo == 1) ? leaf0 + (int32_t)lo : (int32_t)(lo + (s - lo) / 2 - 1);
  const int32_t right = (hi - s == 1) ? leaf0 + (int32_t)s : (int32_t)(s + (hi - s) / 2 - 1);
  nodes[base + node].a = (int32_t)lo;
  nodes[base + node].b = (int32_t)hi;
  child[2 * (base + node)] = left;
  child[2 * (base + node) + 1] = right;
  parent[base + node] = par;
  parent[base + left] = node;
  parent[base + right] = node;
  arrive[base + node] = 0;
}

// Boxes of internal nodes: thread per leaf walks up; the second child to
// arrive forms the parent's box (the union, as grow() does on the host).
__global__ void internal_boxes(const int32_t *curve_of_live, const int64_t *loff, int64_t L, DNode *nodes,
                               const int32_t *child, const int32_t *parent, int32_t *arrive) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= L) return;
  const int c = curve_of_live[q];
  const int64_t m = loff[c + 1] - loff[c], base = 2 * loff[c];
  int32_t node = (int32_t)((m - 1) + (q - loff[c]));
  for (int guard = 0; guard < 80; ++guard) {
    const int32_t par = parent[base + node];
    if (par < 0) break;
    cuda::atomic_ref<int32_t, cuda::thread_scope_device> arr(arrive[base + par]);
    if (arr.fetch_add(1, cuda::memory_order_acq_rel) == 0) break;  // first arrival stops
    const int32_t cl = child[2 * (base + par)], cr = child[2 * (base + par) + 1];
    const DNode *L_ = nodes + base + cl, *R_ = nodes + base + cr;
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      lo[d] = min_of(__ldcg(&L_->lo[d]), __ldcg(&R_->lo[d]));
      hi[d] = max_of(__ldcg(&L_->hi[d]), __ldcg(&R_->hi[d]));
    }
    DNode *P_ = nodes + base + par;
    for (int d = 0; d < 3; ++d) {
      P_->lo[d] = lo[d];
      P_->hi[d] = hi[d];
    }
    node = par;
  }
}

__global__ void curve_of_live_kernel(const int32_t *lidx, const int32_t *pc, int64_t L, int32_t *out) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < L) out[q] = pc[lidx[q]];
}

// Root node pair of every slot (potential pair with live pieces on both sides).
__global__ void root_batches_d(const int32_t *slot_curves, int64_t nslots, const int64_t *loff, DBatch *out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  const int ci = slot_curves[2 * s], cj = slot_curves[2 * s + 1];
  const int64_t mi = loff[ci + 1] - loff[ci], mj = loff[cj + 1] - loff[cj];
  out[s].slot = (int32_t)s;
  out[s].count = 1;
  out[s].pairs[0] = make_int2(mi == 1 ? 0 : (int)(mi / 2 - 1), mj == 1 ? 0 : (int)(mj / 2 - 1));
}

struct DTravArgs {
  const DNode *nodes;
  const int64_t *loff;
  const int32_t *lidx;
  const int32_t *slot_curves;
  const DBatch *in;
  int64_t nin;
  DBatch *out;
  int64_t out_cap;
  unsigned long long *out_count;
  unsigned long long *queue;
  uint8_t *hit;
  unsigned long long *overlaps;
  int32_t *status;
};

// Writes entries [0, n) of stack as batches of slot `slot` to the next
// launch's list; false (and status bit 1) when the list is full.
__device__ bool hand_on(const DTravArgs &A, int slot, const int2 *stack, int n, int lane) {
  const int nb = (n + 31) / 32;
  unsigned long long at = 0;
  if (lane == 0) at = atomicAdd(A.out_count, (unsigned long long)nb);
  at = __shfl_sync(0xffffffffu, at, 0);
  if ((long long)(at + nb) > A.out_cap) {
    if (lane == 0) atomicOr(A.status, 1);
    return false;
  }
  for (int b = 0; b < nb; ++b) {
    const int e = 32 * b + lane;
    if (e < n) A.out[at + b].pairs[lane] = stack[e];
    if (lane == 0) {
      A.out[at + b].slot = slot;
      A.out[at + b].count = min(32, n - 32 * b);
    }
  }
  return true;
}

__device__ __forceinline__ int32_t child_id(int32_t a, int32_t b, int64_t m, bool right) {
  const int32_t mid = a + (b - a) / 2;
  const int32_t leaf0 = (int32_t)(m - 1);
  if (!right) return (mid - a == 1) ? leaf0 + a : a + (mid - a) / 2 - 1;
  return (b - mid == 1) ? leaf0 + mid : mid + (b - mid) / 2 - 1;
}

// stack[0, n) = stack[k, k + n) in passes of 32 that read before they write
// (the lanes of a warp need not run the passes in step).
__device__ __noinline__ void shift_down_d(int2 *stack, int k, int n, int lane) {
  for (int xb = 0; xb < n; xb += 32) {
    const int x = xb + lane;
    int2 v = make_int2(0, 0);
    if (x < n) v = stack[k + x];
    __syncwarp();
    if (x < n) stack[x] = v;
    __syncwarp();
  }
}

__global__ void __launch_bounds__(32 * kDWarps) disc_traverse(DTravArgs A) {
  __shared__ int2 s_stack[kDWarps][kDStack];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int2 *stack = s_stack[w];
  unsigned long long found = 0;
  for (;;) {
    long long b = 0;
    if (lane == 0) b = (long long)atomicAdd(A.queue, 1ULL);
    b = __shfl_sync(0xffffffffu, b, 0);
    if (b >= A.nin) break;
    const int slot = A.in[b].slot;
    const int cnt0 = A.in[b].count;
    const int ci = A.slot_curves[2 * slot], cj = A.slot_curves[2 * slot + 1];
    const int64_t li = A.loff[ci], lj = A.loff[cj];
    const int64_t mi = A.loff[ci + 1] - li, mj = A.loff[cj + 1] - lj;
    const DNode *NI = A.nodes + 2 * li, *NJ = A.nodes + 2 * lj;
    if (lane < cnt0) stack[lane] = A.in[b].pairs[lane];
    int top = cnt0;
    __syncwarp();
    for (int steps = 0; top > 0; ++steps) {
      if (steps >= kBudget) {  // hand the rest on
        hand_on(A, slot, stack, top, lane);
        top = 0;
        __syncwarp();
        break;
      }
      const int cnt = min(top, 32);
      const bool act = lane < cnt;
      int2 pr = make_int2(0, 0);
      if (act) pr = stack[top - cnt + lane];
      __syncwarp();
      top -= cnt;
      bool split = false;
      int2 c0 = make_int2(0, 0), c1 = make_int2(0, 0);
      if (act) {
        const DNode &X = NI[pr.x], &Y = NJ[pr.y];
        const bool meet = X.lo[0] <= Y.hi[0] && X.lo[1] <= Y.hi[1] && X.lo[2] <= Y.hi[2] && Y.lo[0] <= X.hi[0] &&
                          Y.lo[1] <= X.hi[1] && Y.lo[2] <= X.hi[2];
        if (meet) {
          const int32_t sx = X.b - X.a, sy = Y.b - Y.a;
          if (sx == 1 && sy == 1) {
            A.hit[A.lidx[li + X.a]] = 1;
            A.hit[A.lidx[lj + Y.a]] = 1;
            ++found;
          } else if (sy == 1 || (sx > 1 && sx >= sy)) {
            split = true;
            c0 = make_int2(child_id(X.a, X.b, mi, false), pr.y);
            c1 = make_int2(child_id(X.a, X.b, mi, true), pr.y);
          } else {
            split = true;
            c0 = make_int2(pr.x, child_id(Y.a, Y.b, mj, false));
            c1 = make_int2(pr.x, child_id(Y.a, Y.b, mj, true));
          }
        }
      }
      const unsigned sm = __ballot_sync(0xffffffffu, split);
      const int ns = __popc(sm);
      if (top + 2 * ns > kDStack) {  // hand the older half on
        const int k = top / 2;
        if (!hand_on(A, slot, stack, k, lane)) {
          top = 0;
          break;
        }
        __syncwarp();
        shift_down_d(stack, k, top - k, lane);
        top -= k;
      }
      if (split) {
        const int rank = __popc(sm & ((1u << lane) - 1));
        stack[top + 2 * rank] = c0;
        stack[top + 2 * rank + 1] = c1;
      }
      top += 2 * ns;
      __syncwarp();
    }
  }
  for (int o = 16; o; o >>= 1) found += __shfl_xor_sync(0xffffffffu, found, o);
  if (lane == 0 && found) atomicAdd(A.overlaps, found);
}

__global__ void emit_counts(const uint8_t *live, const uint8_t *hit, int64_t n, int32_t *cnt) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) cnt[k] = (live[k] && hit[k]) ? 2 : 1;
}

// One refinement round: a hit piece is replaced by its two halves (live),
// a live piece that was not hit becomes final, final pieces stay.
__global__ void refine(Pieces S, const uint8_t *hit, const int32_t *pos, int64_t n, Pieces D) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int64_t p = pos[k];
  const int32_t c = S.c[k], s = S.s[k];
  const double t0 = S.t0[k], t1 = S.t1[k];
  if (S.live[k] && hit[k]) {
    const double tm = 0.5 * (t0 + t1);
    D.c[p] = c;
    D.s[p] = s;
    D.t0[p] = t0;
    D.t1[p] = tm;
    D.live[p] = 1;
    D.c[p + 1] = c;
    D.s[p + 1] = s;
    D.t0[p + 1] = tm;
    D.t1[p + 1] = t1;
    D.live[p + 1] = 1;
  } else {
    D.c[p] = c;
    D.s[p] = s;
    D.t0[p] = t0;
    D.t1[p] = t1;
    D.live[p] = 0;
  }
}

__global__ void count_per_curve(const int32_t *pc, int64_t n, int32_t *cnt) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  add_one(cnt, k < n ? pc[k] : 0, k < n);
}

// Output vertex of every piece (its start point).
__global__ void emit_points(CurveSet C, Pieces P, int64_t n, const int64_t *pstart, const int64_t *out_off,
                            double *xyz) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = P.c[k];
  const int64_t o = C.cp_off[c], ncp = C.cp_off[c + 1] - o;
  double v[3];
  seg_point(C.kind[c], C.cp + 3 * o, ncp, P.s[k], P.t0[k], v);
  const int64_t at = out_off[c] + (k - pstart[c]);
  for (int d = 0; d < 3; ++d) xyz[3 * at + d] = v[d];
}

// The end point of the last piece of each open curve.
__global__ void emit_end_points(CurveSet C, Pieces P, const int32_t *open_curves, int n_open, const int64_t *pstart,
                                const int64_t *out_off, double *xyz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_open) return;
  const int c = open_curves[i];
  const int64_t k = pstart[c + 1] - 1;
  const int64_t o = C.cp_off[c], ncp = C.cp_off[c + 1] - o;
  double v[3];
  seg_point(C.kind[c], C.cp + 3 * o, ncp, P.s[k], P.t1[k], v);
  const int64_t at = out_off[c + 1] - 1;
  for (int d = 0; d < 3; ++d) xyz[3 * at + d] = v[d];
}

// Box of each output polyline for the potential-link search of the result:
// one CTA per curve, min and max over its vertices (every vertex starts a
// segment of the closed polyline, so this is the union of the segment
// boxes; min and max are exact, so the grouping does not matter).
__global__ void polyline_boxes(const double *xyz, const int64_t *off, double *box) {
  const int c = blockIdx.x;
  const int64_t a = off[c], n = off[c + 1] - a;
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int64_t k = threadIdx.x; k < n; k += blockDim.x)
    for (int d = 0; d < 3; ++d) {
      const double v = xyz[3 * (a + k) + d];
      lo[d] = min_of(lo[d], v);
      hi[d] = max_of(hi[d], v);
    }
  __shared__ double s_lo[3][32], s_hi[3][32];
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o; o >>= 1) {
      lo[d] = min_of(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = max_of(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
    if ((threadIdx.x & 31) == 0) {
      s_lo[d][threadIdx.x >> 5] = lo[d];
      s_hi[d][threadIdx.x >> 5] = hi[d];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) {
      double l = s_lo[d][0], h = s_hi[d][0];
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
        l = min_of(l, s_lo[d][w]);
        h = max_of(h, s_hi[d][w]);
      }
      box[6 * c + d] = l;
      box[6 * c + 3 + d] = h;
    }
}

// Root boxes of the curve trees of round 0: the boxes of the whole curves.
__global__ void root_boxes(const DNode *nodes, const int64_t *loff, int nc, double *box) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int64_t m = loff[c + 1] - loff[c];
  if (m == 0) {
    for (int d = 0; d < 3; ++d) {
      box[6 * c + d] = DBL_MAX;
      box[6 * c + 3 + d] = -DBL_MAX;
    }
    return;
  }
  const DNode &r = nodes[2 * loff[c] + (m == 1 ? 0 : m / 2 - 1)];
  for (int d = 0; d < 3; ++d) {
    box[6 * c + d] = r.lo[d];
    box[6 * c + 3 + d] = r.hi[d];
  }
}

// float32 control points (as a BCC file stores them) -> FP64, exactly.
__global__ void widen_f32(const float *src, int64_t n, double *dst) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    dst[k] = (double)src[k];
}

template <class T>
T *buf(DevBuf &b, int64_t n) {
  return b.as<T>((size_t)std::max<int64_t>(n, 1));
}

void exclusive_scan_i32(Context &ctx, DevBuf &tmp, const int32_t *in, int32_t *out, int64_t n) {
  size_t bytes = 0;
  FLN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, ctx.stream));
  void *t = tmp.need(bytes + 16);
  FLN_CUDA(cub::DeviceScan::ExclusiveSum(t, bytes, in, out, (int)n, ctx.stream));
}

// Potential-link search on the device (potential_link_search.cpp:88-127):
// every pair i < j of curves whose closed boxes meet (box[6c..6c+2] low
// corner, [6c+3..6c+5] high corner; a box with lo.x > hi.x is empty and meets
// nothing), in (i, j) order, as the host sweep (box_pairs) returns it. Tiled
// all-pairs test: a CTA takes kJoinTile curves i and walks the tiles of j from
// its own, staged in shared memory. The first pass counts each i's partners,
// a scan turns the counts into offsets, the second pass writes each i's
// partners in increasing j. Same comparisons as the host, so the same set.
constexpr int kJoinTile = 256;

template <bool kWrite>
__global__ void __launch_bounds__(kJoinTile) box_join(const double *box, int nc, const int64_t *offs, int32_t *counts,
                                                      int2 *out) {
  __shared__ double s_b[6][kJoinTile];
  const int i0 = blockIdx.x * kJoinTile, i = i0 + threadIdx.x;
  double a[6];
  bool va = false;
  if (i < nc) {
    for (int d = 0; d < 6; ++d) a[d] = box[6 * (int64_t)i + d];
    va = a[0] <= a[3];
  }
  int64_t at = (kWrite && i < nc) ? offs[i] : 0;
  int cnt = 0;
  for (int j0 = i0; j0 < nc; j0 += kJoinTile) {
    __syncthreads();
    for (int x = threadIdx.x; x < 6 * kJoinTile; x += kJoinTile) {
      const int jj = x / 6, d = x - 6 * jj;
      s_b[d][jj] = j0 + jj < nc ? box[6 * (int64_t)(j0 + jj) + d] : 1.0;
    }
    __syncthreads();
    if (!va) continue;
    const int jn = min(kJoinTile, nc - j0);
    for (int jj = 0; jj < jn; ++jj) {
      const int j = j0 + jj;
      if (j <= i) continue;
      const double l0 = s_b[0][jj], l1 = s_b[1][jj], l2 = s_b[2][jj];
      const double h0 = s_b[3][jj], h1 = s_b[4][jj], h2 = s_b[5][jj];
      const bool hit = l0 <= h0 && a[0] <= h0 && a[1] <= h1 && a[2] <= h2 && l0 <= a[3] && l1 <= a[4] &&
                       l2 <= a[5];
      if (hit) {
        if (kWrite) out[at++] = make_int2(i, j);
        else ++cnt;
      }
    }
  }
  if (!kWrite && i < nc) counts[i] = cnt;
}

// The sorted pairs of the boxes in d_box (nc curves) on the host; curves
// with empty[c] set get an empty box first. Beyond kJoinMaxCurves curves the
// all-pairs test costs more than the host sweep, which then runs instead.
constexpr int kJoinMaxCurves = 1 << 17;
constexpr int kJoinBufs = 34;  // d_disc[34], [35]: the join's own; [36] the float32 upload (0..33: Discretize)
std::vector<Box3> boxes_to_host(Context &ctx, const double *d_box, int nc);
std::vector<std::pair<int, int>> device_box_pairs(Context &ctx, const double *d_box, int nc) {
  if (nc > kJoinMaxCurves) return box_pairs(boxes_to_host(ctx, d_box, nc));
  std::vector<std::pair<int, int>> pl;
  if (nc < 2) return pl;
  cudaStream_t st = ctx.stream;
  const int grid = (nc + kJoinTile - 1) / kJoinTile;
  int32_t *d_cnt = static_cast<int32_t *>(ctx.d_disc[kJoinBufs].need((size_t)nc * sizeof(int32_t) + 16));
  box_join<false><<<grid, kJoinTile, 0, st>>>(d_box, nc, nullptr, d_cnt, nullptr);
  FLN_CUDA(cudaGetLastError());
  std::vector<int32_t> cnt(nc);
  FLN_CUDA(cudaMemcpyAsync(cnt.data(), d_cnt, nc * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaStreamSynchronize(st));
  std::vector<int64_t> offs(nc);
  int64_t total = 0;
  for (int c = 0; c < nc; ++c) {
    offs[c] = total;
    total += cnt[c];
  }
  if (total == 0) return pl;
  int64_t *d_offs = static_cast<int64_t *>(ctx.d_disc[kJoinBufs + 1].need((size_t)nc * sizeof(int64_t) + (size_t)total * 8));
  int2 *d_out = reinterpret_cast<int2 *>(d_offs + nc);
  FLN_CUDA(cudaMemcpyAsync(d_offs, offs.data(), nc * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  box_join<true><<<grid, kJoinTile, 0, st>>>(d_box, nc, d_offs, nullptr, d_out);
  FLN_CUDA(cudaGetLastError());
  std::vector<int2> h((size_t)total);
  FLN_CUDA(cudaMemcpyAsync(h.data(), d_out, total * sizeof(int2), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaStreamSynchronize(st));
  pl.resize((size_t)total);
  for (int64_t k = 0; k < total; ++k) pl[k] = {h[k].x, h[k].y};
  return pl;
}

std::vector<Box3> boxes_to_host(Context &ctx, const double *d_box, int nc) {
  std::vector<double> h(6 * (size_t)nc);
  if (nc > 0)
    FLN_CUDA(cudaMemcpyAsync(h.data(), d_box, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
  FLN_CUDA(cudaStreamSynchronize(ctx.stream));
  std::vector<Box3> b(nc);
  for (int c = 0; c < nc; ++c)
    for (int d = 0; d < 3; ++d) {
      b[c].lo[d] = h[6 * c + d];
      b[c].hi[d] = h[6 * c + 3 + d];
    }
  return b;
}

}  // namespace

void discretize_device(Context &ctx, const std::vector<CurveData> &curves, const float *bcc_f32,
                       std::vector<int64_t> &offsets, DoubleArray &xyz, std::vector<int32_t> &pairs_out,
                       int32_t &rounds) {
  const int nc = (int)curves.size();
  cudaStream_t st = ctx.stream;
  DevBuf *B = ctx.d_disc;
  // Control points, kinds and segment counts.
  std::vector<int64_t> cp_off(nc + 1, 0), seg_off(nc + 1, 0);
  std::vector<int32_t> kind(std::max(nc, 1), 0);
  for (int c = 0; c < nc; ++c) {
    cp_off[c + 1] = cp_off[c] + (int64_t)curves[c].q.size();
    seg_off[c + 1] = seg_off[c] + std::max(curves[c].segments(), 0);
    kind[c] = curves[c].kind;
  }
  // The packed FP64 control points, unless the float32 ones of the BCC file
  // are uploaded and widened on the device.
  DoubleArray cp(bcc_f32 ? 0 : 3 * (size_t)std::max<int64_t>(cp_off[nc], 1));
  const int64_t nseg = seg_off[nc];
  DoubleArray norms((size_t)std::max<int64_t>(nseg, 1));
#pragma omp parallel for schedule(dynamic, 16)
  for (int c = 0; c < nc; ++c) {
    if (!bcc_f32 && !curves[c].q.empty())
      std::memcpy(&cp[3 * cp_off[c]], &curves[c].q[0].x, curves[c].q.size() * sizeof(Vec3));
    for (int s = 0; s < curves[c].segments(); ++s) {
      const Vec3 &p = curves[c].q[s];
      norms[seg_off[c] + s] = std::sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    }
  }
  // Input sanity (discretize.cpp:126-160): mean |control point| over the
  // segment-indexed points, summed in the host's order.
  double norm_sum = 0;
  for (int64_t k = 0; k < nseg; ++k) norm_sum += norms[k];
  const double avg = norm_sum / ((double)nseg * 1.73205080757);
  const double thresh = std::numeric_limits<double>::epsilon() * avg;
  if (nseg > INT32_MAX) throw Error(FLN_ERR_OUT_OF_MEMORY, "Discretize: more than 2^31 segments");

  double *d_cp = buf<double>(B[0], 3 * std::max<int64_t>(cp_off[nc], 1));
  int64_t *d_cpoff = buf<int64_t>(B[1], nc + 1);
  int32_t *d_kind = buf<int32_t>(B[2], nc);
  int64_t *d_segoff = buf<int64_t>(B[3], nc + 1);
  if (bcc_f32) {
    const int64_t nf = 3 * cp_off[nc];
    float *d_f = buf<float>(B[kJoinBufs + 2], std::max<int64_t>(nf, 1));
    copy_h2d(ctx, d_f, bcc_f32, nf * sizeof(float));
    if (nf > 0) widen_f32<<<(int)std::min<int64_t>((nf + 255) / 256, 1 << 20), 256, 0, st>>>(d_f, nf, d_cp);
    FLN_CUDA(cudaGetLastError());
  } else {
    copy_h2d(ctx, d_cp, cp.data(), 3 * cp_off[nc] * sizeof(double));
  }
  FLN_CUDA(cudaMemcpyAsync(d_cpoff, cp_off.data(), (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemcpyAsync(d_kind, kind.data(), std::max(nc, 1) * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemcpyAsync(d_segoff, seg_off.data(), (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  const CurveSet C{d_cp, d_cpoff, d_kind};

  // Piece arrays (ping-pong sets 0 and 1).
  auto pieces = [&](int which, int64_t n) {
    DevBuf *b = B + 4 + 5 * which;
    return Pieces{buf<int32_t>(b[0], n), buf<int32_t>(b[1], n), buf<double>(b[2], n), buf<double>(b[3], n),
                  buf<uint8_t>(b[4], n)};
  };
  // Per-piece arrays with room for growth: refinement usually adds a few
  // tens of percent, and each reallocation would cost a device-wide free.
  const int64_t reserve = nseg + nseg / 2 + 1024;
  pieces(0, reserve);
  pieces(1, reserve);
  for (int k : {14, 15}) buf<int32_t>(B[k], reserve);
  buf<uint8_t>(B[28], reserve);
  int cur = 0;
  int64_t n = nseg;
  Pieces P = pieces(cur, n);
  if (n > 0) {
    init_pieces<<<(int)((n + 255) / 256), 256, 0, st>>>(d_segoff, nc, n, P);
    FLN_CUDA(cudaGetLastError());
  }
  const int kMaxRounds = 55;  // MAX_RECURSION (discretize.cpp:174)
  unsigned long long overlaps = 0;
  rounds = 0;
  std::vector<int32_t> slot_curves;
  std::vector<int32_t> counts(std::max(nc, 1));
  std::vector<int64_t> loff(nc + 1), int_off(nc + 1);
  int64_t L = 0;
  // Live compaction, leaf records and the curve trees of the live pieces;
  // returns the minimum leaf box diagonal.
  auto build_live = [&]() -> double {
    int32_t *d_flag = buf<int32_t>(B[14], n), *d_pos = buf<int32_t>(B[15], n);
    int32_t *d_cnt = buf<int32_t>(B[16], nc);
    FLN_CUDA(cudaMemsetAsync(d_cnt, 0, std::max(nc, 1) * sizeof(int32_t), st));
    int32_t last_pos = 0, last_flag = 0;
    if (n > 0) {
      flag_live<<<(int)((n + 255) / 256), 256, 0, st>>>(P.live, n, d_flag);
      exclusive_scan_i32(ctx, B[17], d_flag, d_pos, n);
      FLN_CUDA(cudaMemcpyAsync(&last_pos, d_pos + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      FLN_CUDA(cudaMemcpyAsync(&last_flag, d_flag + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    }
    FLN_CUDA(cudaStreamSynchronize(st));
    L = (int64_t)last_pos + last_flag;
    int32_t *d_lidx = buf<int32_t>(B[18], L);
    if (n > 0) compact_live<<<(int)((n + 255) / 256), 256, 0, st>>>(P.live, d_pos, P.c, n, d_lidx, d_cnt);
    FLN_CUDA(cudaGetLastError());
    if (nc > 0) FLN_CUDA(cudaMemcpyAsync(counts.data(), d_cnt, nc * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaStreamSynchronize(st));
    loff[0] = 0;
    int_off[0] = 0;
    for (int c = 0; c < nc; ++c) {
      loff[c + 1] = loff[c] + counts[c];
      int_off[c + 1] = int_off[c] + std::max<int64_t>(counts[c] - 1, 0);
    }
    int64_t *d_loff = buf<int64_t>(B[19], nc + 1), *d_intoff = buf<int64_t>(B[20], nc + 1);
    FLN_CUDA(cudaMemcpyAsync(d_loff, loff.data(), (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    FLN_CUDA(cudaMemcpyAsync(d_intoff, int_off.data(), (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    DNode *d_nodes = buf<DNode>(B[21], 2 * L);
    int32_t *d_child = buf<int32_t>(B[22], 4 * L), *d_parent = buf<int32_t>(B[23], 2 * L);
    int32_t *d_arrive = buf<int32_t>(B[24], 2 * L), *d_cl = buf<int32_t>(B[25], L);
    unsigned long long *d_md = buf<unsigned long long>(B[26], 1);
    const unsigned long long inf_key = 0x7FF0000000000000ULL;
    FLN_CUDA(cudaMemcpyAsync(d_md, &inf_key, sizeof inf_key, cudaMemcpyHostToDevice, st));
    if (L > 0) {
      leaf_records<<<(int)((L + 255) / 256), 256, 0, st>>>(C, P, d_lidx, d_loff, L, d_nodes, d_md);
      curve_of_live_kernel<<<(int)((L + 255) / 256), 256, 0, st>>>(d_lidx, P.c, L, d_cl);
      const int64_t ti = int_off[nc];
      if (ti > 0) {
        internal_topology<<<(int)((ti + 255) / 256), 256, 0, st>>>(d_loff, d_intoff, nc, ti, d_nodes, d_child,
                                                                     d_parent, d_arrive);
        internal_boxes<<<(int)((L + 255) / 256), 256, 0, st>>>(d_cl, d_loff, L, d_nodes, d_child, d_parent,
                                                                d_arrive);
      }
      FLN_CUDA(cudaGetLastError());
    }
    unsigned long long md = inf_key;
    FLN_CUDA(cudaMemcpyAsync(&md, d_md, sizeof md, cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaStreamSynchronize(st));
    double v;
    std::memcpy(&v, &md, sizeof v);
    return v;
  };
  const int grid = ctx.num_sms * occupancy_of((const void *)disc_traverse, 32 * kDWarps);
  const int64_t nwarps = (int64_t)grid * kDWarps;
  int64_t out_cap = 0;
  for (int it = 0; it < kMaxRounds; ++it) {
    ++rounds;
    const double md = build_live();
    if (it == 0 && !(md >= thresh))
      throw Error(FLN_ERR_SEGMENT_TOO_SMALL,
                  "Discretize: Smallest input segment is smaller than eps * avg coordinate. Consider combining.");
    if (it > 0 && !(md >= thresh))
      throw Error(FLN_ERR_SEGMENT_TOO_SMALL,
                  "Discretize: Smallest segment is smaller than eps * avg coordinate. Perhaps curves are too close.");
    const int64_t *d_loff = static_cast<const int64_t *>(B[19].ptr);
    const DNode *d_nodes = static_cast<const DNode *>(B[21].ptr);
    if (it == 0) {
      // Potential pairs of the input curves (their whole boxes).
      double *d_box = buf<double>(B[27], 6 * (int64_t)nc);
      if (nc > 0) root_boxes<<<(nc + 127) / 128, 128, 0, st>>>(d_nodes, d_loff, nc, d_box);
      FLN_CUDA(cudaGetLastError());
      const auto pl = device_box_pairs(ctx, d_box, nc);
      for (auto &p : pl) {
        slot_curves.push_back(p.first);
        slot_curves.push_back(p.second);
      }
    }
    // Pairs with live pieces on both sides.
    std::vector<int32_t> sc;
    for (size_t k = 0; k + 1 < slot_curves.size(); k += 2)
      if (counts[slot_curves[k]] > 0 && counts[slot_curves[k + 1]] > 0) {
        sc.push_back(slot_curves[k]);
        sc.push_back(slot_curves[k + 1]);
      }
    const int64_t nslots = (int64_t)sc.size() / 2;
    uint8_t *d_hit = buf<uint8_t>(B[28], n);
    unsigned long long *d_ctr = buf<unsigned long long>(B[29], 4);  // overlaps, queue, next count
    int32_t *d_status = buf<int32_t>(B[30], 1);
    overlaps = 0;
    FLN_CUDA(cudaMemsetAsync(d_hit, 0, (size_t)std::max<int64_t>(n, 1), st));
    if (nslots > 0) {
      int32_t *d_sc = buf<int32_t>(B[31], 2 * nslots);
      FLN_CUDA(cudaMemcpyAsync(d_sc, sc.data(), sc.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
      for (int attempt = 0;; ++attempt) {
        if (attempt > 6) throw Error(FLN_ERR_INTERNAL, "Discretize: node-pair list capacity");
        out_cap = std::max<int64_t>(out_cap, std::max<int64_t>(nslots, nwarps * (kDStack / 32 + 2)) * 4);
        DBatch *d_b = reinterpret_cast<DBatch *>(B[32].need((size_t)(2 * out_cap) * sizeof(DBatch)));
        DBatch *bin = d_b, *bout = d_b + out_cap;
        FLN_CUDA(cudaMemsetAsync(d_hit, 0, (size_t)std::max<int64_t>(n, 1), st));
        FLN_CUDA(cudaMemsetAsync(d_ctr, 0, 4 * sizeof(unsigned long long), st));
        FLN_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int32_t), st));
        root_batches_d<<<(int)((nslots + 255) / 256), 256, 0, st>>>(d_sc, nslots, d_loff, bin);
        FLN_CUDA(cudaGetLastError());
        int64_t nin = nslots;
        int32_t status = 0;
        for (int r = 0; nin > 0 && r < 1000000; ++r) {
          FLN_CUDA(cudaMemsetAsync(d_ctr + 1, 0, 2 * sizeof(unsigned long long), st));
          DTravArgs A{d_nodes, d_loff, static_cast<const int32_t *>(B[18].ptr), d_sc, bin, nin, bout, out_cap,
                      d_ctr + 2, d_ctr + 1, d_hit, d_ctr, d_status};
          const int g = (int)std::max<int64_t>(1, std::min<int64_t>((nin + kDWarps - 1) / kDWarps, grid));
          disc_traverse<<<g, 32 * kDWarps, 0, st>>>(A);
          FLN_CUDA(cudaGetLastError());
          unsigned long long next = 0;
          FLN_CUDA(cudaMemcpyAsync(&next, d_ctr + 2, sizeof next, cudaMemcpyDeviceToHost, st));
          FLN_CUDA(cudaMemcpyAsync(&status, d_status, sizeof status, cudaMemcpyDeviceToHost, st));
          FLN_CUDA(cudaStreamSynchronize(st));
          if (status) break;
          nin = (int64_t)next;
          std::swap(bin, bout);
        }
        if (!status) break;
        out_cap *= 4;  // the list overflowed: redo this round with more room
      }
      FLN_CUDA(cudaMemcpyAsync(&overlaps, d_ctr, sizeof overlaps, cudaMemcpyDeviceToHost, st));
      FLN_CUDA(cudaStreamSynchronize(st));
    }
    // Refinement.
    if (n > 0) {
      int32_t *d_emit = buf<int32_t>(B[14], n), *d_pos = buf<int32_t>(B[15], n);
      emit_counts<<<(int)((n + 255) / 256), 256, 0, st>>>(P.live, d_hit, n, d_emit);
      exclusive_scan_i32(ctx, B[17], d_emit, d_pos, n);
      int32_t lp = 0, le = 0;
      FLN_CUDA(cudaMemcpyAsync(&lp, d_pos + n - 1, sizeof lp, cudaMemcpyDeviceToHost, st));
      FLN_CUDA(cudaMemcpyAsync(&le, d_emit + n - 1, sizeof le, cudaMemcpyDeviceToHost, st));
      FLN_CUDA(cudaStreamSynchronize(st));
      const int64_t n2 = (int64_t)lp + le;
      if (n2 > INT32_MAX) throw Error(FLN_ERR_OUT_OF_MEMORY, "Discretize: more than 2^31 pieces");
      Pieces Q = pieces(1 - cur, n2);
      refine<<<(int)((n + 255) / 256), 256, 0, st>>>(P, d_hit, d_pos, n, Q);
      FLN_CUDA(cudaGetLastError());
      cur = 1 - cur;
      P = Q;
      n = n2;
    }
    if (overlaps == 0) break;
  }
  if (overlaps > 0) {
    // The last round split pieces: the host checks their size first.
    const double md = build_live();
    if (!(md >= thresh))
      throw Error(FLN_ERR_SEGMENT_TOO_SMALL,
                  "Discretize: Smallest segment is smaller than eps * avg coordinate. Perhaps curves are too close.");
    throw Error(FLN_ERR_MAX_RECURSION, "Reached max recursion (curves are too close) in Discretize().");
  }
  // Output polylines: start point of every piece, plus the end point of an
  // open curve's last piece.
  int32_t *d_cnt = buf<int32_t>(B[16], nc);
  FLN_CUDA(cudaMemsetAsync(d_cnt, 0, std::max(nc, 1) * sizeof(int32_t), st));
  if (n > 0) count_per_curve<<<(int)((n + 255) / 256), 256, 0, st>>>(P.c, n, d_cnt);
  if (nc > 0) FLN_CUDA(cudaMemcpyAsync(counts.data(), d_cnt, nc * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaStreamSynchronize(st));
  std::vector<int64_t> pstart(nc + 1, 0);
  offsets.assign(nc + 1, 0);
  std::vector<int32_t> open_curves;
  for (int c = 0; c < nc; ++c) {
    pstart[c + 1] = pstart[c] + counts[c];
    const bool extra = !curves[c].closed && counts[c] > 0;
    offsets[c + 1] = offsets[c] + counts[c] + (extra ? 1 : 0);
    if (extra) open_curves.push_back(c);
  }
  const int64_t nv = offsets[nc];
  int64_t *d_pstart = buf<int64_t>(B[19], nc + 1), *d_out = buf<int64_t>(B[20], nc + 1);
  double *d_xyz = buf<double>(B[33], 3 * nv);
  FLN_CUDA(cudaMemcpyAsync(d_pstart, pstart.data(), (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemcpyAsync(d_out, offsets.data(), (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  if (n > 0) emit_points<<<(int)((n + 255) / 256), 256, 0, st>>>(C, P, n, d_pstart, d_out, d_xyz);
  if (!open_curves.empty()) {
    int32_t *d_open = buf<int32_t>(B[31], (int64_t)open_curves.size());
    FLN_CUDA(cudaMemcpyAsync(d_open, open_curves.data(), open_curves.size() * sizeof(int32_t),
                             cudaMemcpyHostToDevice, st));
    emit_end_points<<<(int)((open_curves.size() + 127) / 128), 128, 0, st>>>(C, P, d_open, (int)open_curves.size(),
                                                                            d_pstart, d_out, d_xyz);
  }
  FLN_CUDA(cudaGetLastError());
  FLN_CUDA(cudaStreamSynchronize(st));
  xyz.resize(3 * nv);
  copy_d2h(ctx, xyz.data(), d_xyz, 3 * nv * sizeof(double));
  // Potential pairs of the polylines.
  double *d_box = buf<double>(B[27], 6 * (int64_t)nc);
  if (nc > 0) polyline_boxes<<<nc, 256, 0, st>>>(d_xyz, d_out, d_box);
  FLN_CUDA(cudaGetLastError());
  // (A curve without vertices gets the empty box from polyline_boxes.)
  const auto pl = device_box_pairs(ctx, d_box, nc);
  pairs_out.resize(2 * pl.size());
  for (size_t k = 0; k < pl.size(); ++k) {
    pairs_out[2 * k] = pl[k].first;
    pairs_out[2 * k + 1] = pl[k].second;
  }
  // The working buffers (tens of GB for 10^8 segments) are not kept for the
  // linking-number stage that follows.
  FLN_CUDA(cudaStreamSynchronize(st));
  for (int k = 0; k < 37; ++k) B[k].release();
}

}  // namespace fln
