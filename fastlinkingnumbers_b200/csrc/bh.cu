// Two-tree Barnes–Hut linking numbers on B200 (sm_100a).
//
// Trees. One binary tree per loop over its segments, leaves = single
// segments. Default ("curve-order"): node = contiguous segment range
// [lo, hi), split at lo + (hi - lo) / 2; a polyline is continuous, so these
// ranges are spatially compact and the tree needs no sort. Its topology is
// implicit: the internal node splitting at s has local id s - 1, found by a
// root-to-node descent per node. Optionally the reference's kd-median tree
// (ModifiedKdBVH.h:207-237) is built on the host and uploaded (bh_tree = 1).
// Local ids: internal nodes 0..n-2, leaf of object position p = n-1+p.
//
// Moments (compute_link.h:95-114, compute_link.cpp:333-389) are built in
// FP64 bottom-up: each leaf thread walks to the root; at every parent the
// second arriving child computes the parent (box union, centre, the Eq. 21-23
// shift of monopole c_M, dipole C_D, quadrupole C_Q) and continues. They are
// then stored for traversal in FP32 relative to the node centre; the centre
// itself stays FP64 so node separations are formed in FP64. Each C_Q[k] is
// symmetric in its last two indices (leaf c_k c c^T / 12; the shift adds
// c_k r r^T + (r D_k) + (r D_k)^T), so 6 of its 9 entries are stored.
//
// Traversal (compute_link.cpp:547-666, :695-841). One warp per loop pair,
// pairs taken from a device queue. The warp keeps a LIFO of node pairs in
// shared memory (spilling its oldest half to a global buffer when full) and
// classifies up to 32 pairs per step, one per lane:
//   leaf-leaf        -> exact one-arctan term (compute_link.cpp:576-606);
//   far (|dr|^2 + eps^2 > (r1 + r2)^2 beta^2 + eps^2)
//                    -> monopole + dipole + quadrupole (Eq. 29-30) and the
//                       Eq. 14 error estimate (compute_link.cpp:411-524);
//   otherwise        -> push the two children of the larger node (the
//                       internal one if the other is a leaf).
// Far and leaf pairs go to two per-warp queues and are evaluated 32 at a
// time, so the expensive branches run with full warps. Leaf-leaf pairs
// closer than one segment length are evaluated in FP64 from the vertices.
// Sums are FP64 per lane, reduced per pair in a fixed order.
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <type_traits>

#include "engine.hpp"
#include "learned.cuh"

namespace fln {

namespace {

constexpr double kInvTwoPi = 0.15915494309189533576888376337251436;
constexpr double kInvFourPi = 0.079577471545947667884441881686257181;
constexpr double kInvRt3 = 0.57735026918962576450914878050195746;
constexpr int kWarps = 4;          // warps per traversal CTA
// Shared-memory stack entries per warp (> 128). 224 keeps a traversal CTA at
// 11 KB of shared memory, so five CTAs fit a 64 KB carveout and leave the
// rest of the SM's 256 KB to L1, which holds the node records the warps
// re-read: 182.9 ms against 188.8 ms with 512 entries (14M-segment polymer
// step, B200).
#ifndef FLN_BH_STACK
#define FLN_BH_STACK 224
#endif
// Preferred shared-memory carveout of the traversal kernel, percent: room
// for five CTAs of up to 16 KB (stacks, far-pair queue with its separations,
// and in the first pass the pairs' ratios for the frontier), 1 KB each
// reserved by the system.
#ifndef FLN_BH_CARVEOUT
#define FLN_BH_CARVEOUT 44
#endif
// Six and seven CTAs per SM (fln_params.bh_occupancy).
#ifndef FLN_BH_CARVEOUT_6
#define FLN_BH_CARVEOUT_6 58
#endif
constexpr int kStack = FLN_BH_STACK;
constexpr int kSpill = 8192;       // global spill entries per warp
// Curve-order nodes of at most 2^kSmallHeight segments are built straight
// from their segments (build_small), the rest level by level (build_height).
#ifndef FLN_BUILD_SMALL_HEIGHT
#define FLN_BUILD_SMALL_HEIGHT 4
#endif
constexpr int kSmallHeight = FLN_BUILD_SMALL_HEIGHT;
#ifndef FLN_BUCKET_SOFT_LOG2
#define FLN_BUCKET_SOFT_LOG2 19  // exact-list chunks per round before it stops taking batches
#endif
#ifndef FLN_CHUNK_SOFT_LOG2
#define FLN_CHUNK_SOFT_LOG2 20  // chunks per list before a round stops taking batches
#endif

// FP64 build record.
struct __align__(16) BuildNode {
  double lo[3], hi[3];
  double mid[3];
  double t[3];
  double D[9];   // row-major
  double Q[18];  // Q_k symmetric: (xx, yy, zz, xy, xz, yz) for k = 0, 1, 2
  int32_t seg_lo, seg_cnt;  // leaves below: a curve-order node covers segments [seg_lo, seg_lo + seg_cnt)
};
static_assert(sizeof(BuildNode) == 320, "BuildNode layout");

// Record copies as 16-byte vectors (a thread's record is contiguous; with
// field-by-field stores every warp instruction would touch 32 lines).
template <class T>
__device__ __forceinline__ void put16(T *dst, const T &src) {
  static_assert(sizeof(T) % 16 == 0 && alignof(T) >= 16, "16-byte record");
  const int4 *s = reinterpret_cast<const int4 *>(&src);
  int4 *d = reinterpret_cast<int4 *>(dst);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 16); ++i) d[i] = s[i];
}
template <class T>
__device__ __forceinline__ void get16(const T *src, T &dst) {
  const int4 *s = reinterpret_cast<const int4 *>(src);
  int4 *d = reinterpret_cast<int4 *>(&dst);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 16); ++i) d[i] = s[i];
}

// Traversal records.
struct __align__(32) NodeHdr {
  double m[3];      // centre (leaves: segment midpoint)
  double r;         // half the box diagonal
  double rsq;       // its square, 0.25 |diag|^2, for the reference's split rule
  int32_t left;     // internal: local child ids; leaf: left = -1 - segment
  int32_t right;
  int32_t lo;       // leaf: its segment; curve-order node: first segment of its range
  int32_t cnt;      // leaves below (curve-order: the range is [lo, lo + cnt))
  float tn;         // |c_M| and ||C_D||_F / sqrt(3) of the node's moments: the
  float dn;         // Eq. 14 weights, formed when a pair is classified far
};                  // 64 B: two 32-byte loads (load_hdr), never across a 128 B line
static_assert(sizeof(NodeHdr) == 64, "NodeHdr layout");
struct __align__(32) NodeMom {
  float t[3];
  float D[9];
  float Q[18];
  float qn;         // (1/3) ||C_Q||_F
  float pad;        // 128 B: four 32-byte loads (load_mom), one 128 B line
};
static_assert(sizeof(NodeMom) == 128, "NodeMom layout");

// Traversal records through the read-only path in 32-byte loads: the
// traversal is bound by L1 wavefronts, and a scattered 32-byte load costs
// one per lane where two 16-byte loads cost two. Every kernel that
// classifies or evaluates node pairs loads them this way, so the compiled
// arithmetic, and with it every rounding, is the same in all schedules.
__device__ __forceinline__ void load32(const void *p, unsigned long long *w) {
  asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(w[0]), "=l"(w[1]), "=l"(w[2]), "=l"(w[3]) : "l"(p));
}
__device__ __forceinline__ NodeHdr load_hdr(const NodeHdr *p) {
  NodeHdr h;
  unsigned long long *w = reinterpret_cast<unsigned long long *>(&h);
  load32(p, w);
  load32(reinterpret_cast<const char *>(p) + 32, w + 4);
  return h;
}
__device__ __forceinline__ NodeMom load_mom(const NodeMom *p) {
  NodeMom m;
  unsigned long long *w = reinterpret_cast<unsigned long long *>(&m);
#pragma unroll
  for (int i = 0; i < 4; ++i) load32(reinterpret_cast<const char *>(p) + 32 * i, w + 4 * i);
  return m;
}

// Moment records of far pairs staged in shared memory by bulk copies (1) or
// loaded by the lanes (0). A scattered 32-byte load costs the L1 data pipe
// one wavefront per lane, and the moment records are about half of the
// traversal's loads; a bulk copy of a record (cp.async.bulk, 128 bytes,
// completion counted on an mbarrier) is done by the copy engine instead, and
// the lanes then read the staged records from shared memory at 128 bytes per
// wavefront. Slots are 144 bytes apart (16-byte aligned, as bulk copies
// require), so chunk k of slot s sits in bank group (s + k) mod 8 and 8 lanes
// reading the same chunk of 8 consecutive slots do not conflict.
#ifndef FLN_BH_TMA_MOM
#define FLN_BH_TMA_MOM 0
#endif
constexpr int kStagePairs = 16;            // far pairs per staged drain
constexpr int kSlotF4 = 9;                 // slot stride in float4 (144 bytes)
constexpr int kStageWaitPolls = 1 << 20;   // bounded wait on the staging barrier
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Waits for the barrier's phase of the given parity; false if it did not
// complete within kStageWaitPolls tries.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (int i = 0; i < kStageWaitPolls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// One 128-byte moment record into a shared-memory slot (both 16-byte aligned).
__device__ __forceinline__ void bulk_record(void *dst, const NodeMom *src, uint64_t *bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"((uint32_t)sizeof(NodeMom)), "r"(smem_u32(bar))
               : "memory");
}
// The record staged in slot s.
__device__ __forceinline__ NodeMom stage_read(const float4 *stage, int s) {
  NodeMom m;
  float4 *d = reinterpret_cast<float4 *>(&m);
#pragma unroll
  for (int k = 0; k < 8; ++k) d[k] = stage[kSlotF4 * s + k];
  return m;
}


struct TreeArgs {
  const double *xyz;
  const int64_t *off;        // loop vertex offsets
  const int64_t *node_base;  // loop -> first global node
  const int32_t *loops;      // loops that need a tree
  int32_t nloops;
  int32_t *children;         // 2 per global node (internal nodes only used)
  int32_t *parent;           // per global node
  int32_t *leaf_seg;         // per global node: segment of a leaf (kd trees permute)
  int32_t *arrive;           // per global node: arrival counter
  BuildNode *bn;              // per internal node: bn[int_start[k] + id] for the k-th listed loop
  NodeHdr *hdr;
  NodeMom *mom;
  const int64_t *int_start;   // listed loop -> first build record (sum of (n - 1) before it)
};

__device__ __forceinline__ int find_loop_of(const int64_t *start, int n, int64_t x) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (start[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// The listed loop of index x, for a block whose threads take the consecutive
// indices [first, last]: two threads search the whole list for the block's
// first and last index, and every thread then searches only between the two
// (a block crosses few loop boundaries). Every thread of the block must call
// it once (it synchronises the block).
__device__ __forceinline__ int block_loop_of(const int64_t *start, int n, int64_t first, int64_t last, int64_t x) {
  __shared__ int s_range[2];
  if (threadIdx.x == 0) s_range[0] = find_loop_of(start, n, first);
  if (threadIdx.x == (blockDim.x > 1 ? 1 : 0)) s_range[1] = find_loop_of(start, n, last);
  __syncthreads();
  int lo = s_range[0], hi = s_range[1] + 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (start[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// count[key] += 1 for the calling lane, one atomic per distinct key of the
// warp; returns the count before the warp's run plus the lane's rank among
// the lanes of the warp with its key.
__device__ __forceinline__ int32_t add_one_rank(int32_t *count, int32_t key, bool active) {
  const unsigned act = __ballot_sync(0xffffffffu, active);
  if (!active) return 0;
  const unsigned peers = __match_any_sync(act, key);
  const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
  int32_t base = 0;
  if (lane == leader) base = atomicAdd(&count[key], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane) - 1));
}

// Curve-order topology: thread per internal node (local id s - 1 splits at s).
// seg_start[k] = sum of (n - 1) over the first k listed loops. With height
// != nullptr it also records the node's height ceil(log2(range size)) (the
// children of a node are always lower) and counts the nodes per height.
__global__ void curve_tree_topology(TreeArgs A, const int64_t *seg_start, int64_t g0, int64_t total_internal,
                                    uint8_t *height, int32_t *height_count, int2 *range) {
  const int64_t first = g0 + (int64_t)blockIdx.x * blockDim.x, g = first + threadIdx.x;
  const int64_t last = min(first + (int64_t)blockDim.x, total_internal) - 1;
  const int k = block_loop_of(seg_start, A.nloops, first, last, min(g, last));
  if (height) {  // every lane of the warp takes part in the counting
    int32_t h = 0;
    if (g < total_internal) {
      const int l = A.loops[k];
      const int64_t n = A.off[l + 1] - A.off[l];
      const int64_t s = g - seg_start[k] + 1;
      int64_t lo = 0, hi = n;
      for (int depth = 0; depth < 64; ++depth) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (mid == s) break;
        if (s < mid) hi = mid;
        else lo = mid;
      }
      h = 64 - __clzll((unsigned long long)(hi - lo - 1));
      height[g] = (uint8_t)h;
    }
    add_one_rank(height_count, h, g < total_internal);
  }
  if (g >= total_internal) return;
  const int l = A.loops[k];
  const int64_t n = A.off[l + 1] - A.off[l];
  const int32_t node = (int32_t)(g - seg_start[k]);  // local internal id
  const int64_t s = node + 1;                        // split position
  const int64_t base = A.node_base[l];
  int64_t lo = 0, hi = n, psize = 0;
  int32_t par = -1;
  for (int depth = 0; depth < 64; ++depth) {
    const int64_t m = lo + (hi - lo) / 2;
    if (m == s) break;
    par = (int32_t)(m - 1);
    psize = hi - lo;
    if (s < m) hi = m;
    else lo = m;
  }
  if (range) {  // the node's segment range; bit 31 of .y: its parent is built by build_height
    const bool need = par >= 0 && psize > (int64_t(1) << kSmallHeight);
    range[g] = make_int2((int32_t)lo, (int32_t)hi | (need ? INT_MIN : 0));
  }
  const int32_t leaf0 = (int32_t)(n - 1);
  const int32_t left = (s - lo == 1) ? leaf0 + (int32_t)lo : (int32_t)(lo + (s - lo) / 2 - 1);
  const int32_t right = (hi - s == 1) ? leaf0 + (int32_t)s : (int32_t)(s + (hi - s) / 2 - 1);
  A.children[2 * (base + node)] = left;
  A.children[2 * (base + node) + 1] = right;
  A.parent[base + node] = par;
  A.parent[base + left] = node;
  A.parent[base + right] = node;
  A.arrive[base + node] = 0;
}

// Reads a record written by another thread of this launch: L2 loads (the
// writer fenced before its arrival count), never a stale L1 line.
__device__ __forceinline__ void load_cg(const BuildNode *src, BuildNode &dst) {
  const double *s = reinterpret_cast<const double *>(src);
  double *d = reinterpret_cast<double *>(&dst);
  for (int a = 0; a < (int)(sizeof(BuildNode) / sizeof(double)); ++a) d[a] = __ldcg(s + a);
}

// Shift child moments onto the parent centre (Eqs. 21-23 of Qu & James 2021,
// as compute_link.cpp:367-381): c += c_c; D += D_c + c_c r^T;
// Q_k += Q_c,k + r D_c,k^T-row terms + c_c,k r r^T, with r = m_c - m.
__device__ void accumulate_child(BuildNode &P, const BuildNode &C) {
  const double r[3] = {C.mid[0] - P.mid[0], C.mid[1] - P.mid[1], C.mid[2] - P.mid[2]};
  for (int a = 0; a < 3; ++a) P.t[a] += C.t[a];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) P.D[3 * a + b] += C.D[3 * a + b] + C.t[a] * r[b];
  const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
  for (int k = 0; k < 3; ++k)
    for (int e = 0; e < 6; ++e) {
      const int i = ii[e], j = jj[e];
      P.Q[6 * k + e] += C.Q[6 * k + e] + r[j] * C.D[3 * k + i] + r[i] * C.D[3 * k + j] + C.t[k] * (r[i] * r[j]);
    }
}

__device__ void finish_record_regs(const BuildNode &B, NodeHdr &H, NodeMom &M, bool leaf, int32_t seg, int32_t l,
                                   int32_t r) {
  const double dx = B.hi[0] - B.lo[0], dy = B.hi[1] - B.lo[1], dz = B.hi[2] - B.lo[2];
  H.m[0] = B.mid[0];
  H.m[1] = B.mid[1];
  H.m[2] = B.mid[2];
  H.rsq = 0.25 * (dx * dx + dy * dy + dz * dz);
  H.r = sqrt(H.rsq);
  H.left = leaf ? -1 - seg : l;
  H.right = leaf ? -1 : r;
  H.lo = B.seg_lo;
  H.cnt = B.seg_cnt;
  const double tn = sqrt(B.t[0] * B.t[0] + B.t[1] * B.t[1] + B.t[2] * B.t[2]);
  double dd = 0, qq = 0;
  for (int a = 0; a < 9; ++a) dd += B.D[a] * B.D[a];
  for (int k = 0; k < 3; ++k)
    for (int e = 0; e < 6; ++e) qq += (e < 3 ? 1.0 : 2.0) * B.Q[6 * k + e] * B.Q[6 * k + e];
  for (int a = 0; a < 3; ++a) M.t[a] = (float)B.t[a];
  for (int a = 0; a < 9; ++a) M.D[a] = (float)B.D[a];
  for (int a = 0; a < 18; ++a) M.Q[a] = (float)B.Q[a];
  H.tn = (float)tn;
  H.dn = (float)(sqrt(dd) * kInvRt3);
  // Leaf: |c|^3 / 36, which is also (1/3) ||C_Q||_F for c c c^T / 12.
  M.qn = (float)(leaf ? tn * tn * tn / 36.0 : sqrt(qq) / 3.0);
  M.pad = 0.f;
}

// Traversal records of a node, formed in registers and stored as vectors.
__device__ __forceinline__ void finish_record(const BuildNode &B, NodeHdr &H, NodeMom &M, bool leaf, int32_t seg,
                                              int32_t l, int32_t r) {
  NodeHdr h;
  NodeMom m;
  finish_record_regs(B, h, m, leaf, seg, l, r);
  put16(&H, h);
  put16(&M, m);
}

// Leaf record of segment `seg` of a loop at vertex offset o with n segments
// (compute_link.cpp:351-363): box, midpoint, tangent c, C_D = 0, and
// C_Q,k = c_k c c^T / 12.
__device__ void leaf_build(const double *xyz, int64_t o, int64_t n, int32_t seg, BuildNode &B) {
  const int64_t v0 = o + seg, v1 = o + (seg + 1 == n ? 0 : seg + 1);
  double p0[3], p1[3];
  for (int a = 0; a < 3; ++a) {
    p0[a] = xyz[3 * v0 + a];
    p1[a] = xyz[3 * v1 + a];
    B.lo[a] = fmin(p0[a], p1[a]);
    B.hi[a] = fmax(p0[a], p1[a]);
    B.mid[a] = 0.5 * p0[a] + 0.5 * p1[a];
    B.t[a] = p1[a] - p0[a];
  }
  B.seg_lo = seg;
  B.seg_cnt = 1;
  for (int a = 0; a < 9; ++a) B.D[a] = 0.0;
  const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
  for (int kk = 0; kk < 3; ++kk)
    for (int e = 0; e < 6; ++e) B.Q[6 * kk + e] = ((1.0 / 12.0) * B.t[kk]) * (B.t[ii[e]] * B.t[jj[e]]);
}

// Leaf records of the curve-order trees (thread per leaf), straight from the
// segment's two vertices: the values finish_record forms from leaf_build's
// record (box, midpoint, tangent c, C_D = 0, C_Q,k = c_k c c^T / 12), without
// an FP64 build record in registers, so the kernel runs at full occupancy.
__global__ void __launch_bounds__(256) build_leaves(TreeArgs A, const int64_t *seg_start2, int64_t g0,
                                                    int64_t total) {
  const int64_t first = g0 + (int64_t)blockIdx.x * blockDim.x, g = first + threadIdx.x;
  const int64_t last = min(first + (int64_t)blockDim.x, total) - 1;
  const int k = block_loop_of(seg_start2, A.nloops, first, last, min(g, last));
  if (g >= total) return;
  const int l = A.loops[k];
  const int64_t o = A.off[l], n = A.off[l + 1] - o;
  const int64_t base = A.node_base[l];
  // Curve order: leaf position p holds segment p (the identity leaf map,
  // written here for build_height).
  const int32_t seg = (int32_t)(g - seg_start2[k]);
  const int32_t node = (int32_t)(n - 1 + seg);
  A.leaf_seg[base + node] = seg;
  const int64_t v0 = o + seg, v1 = o + (seg + 1 == n ? 0 : seg + 1);
  double t[3], d[3];
  NodeHdr h;
  NodeMom m;
  for (int a = 0; a < 3; ++a) {
    const double p0 = A.xyz[3 * v0 + a], p1 = A.xyz[3 * v1 + a];
    t[a] = p1 - p0;
    h.m[a] = 0.5 * p0 + 0.5 * p1;
    d[a] = fmax(p0, p1) - fmin(p0, p1);
  }
  h.rsq = 0.25 * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  h.r = sqrt(h.rsq);
  h.left = -1 - seg;
  h.right = -1;
  h.lo = seg;
  h.cnt = 1;
  const double tn = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  h.tn = (float)tn;
  h.dn = 0.f;
  for (int a = 0; a < 3; ++a) m.t[a] = (float)t[a];
  for (int a = 0; a < 9; ++a) m.D[a] = 0.f;
  const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
  for (int kk = 0; kk < 3; ++kk)
    for (int e = 0; e < 6; ++e) m.Q[6 * kk + e] = (float)(((1.0 / 12.0) * t[kk]) * (t[ii[e]] * t[jj[e]]));
  m.qn = (float)(tn * tn * tn / 36.0);
  m.pad = 0.f;
  put16(&A.hdr[base + node], h);
  put16(&A.mom[base + node], m);
}

// Thread per leaf: write the leaf's traversal record and walk up; the second
// child to arrive at a parent builds it. Leaf build records are never
// stored: a parent rebuilds a leaf child from its two vertices (48 B read
// instead of a 320 B record written and read back). The arrival counter is
// an acquire-release atomic, which orders the first child's record before
// the second child's reads.
__global__ void build_moments(TreeArgs A, const int64_t *seg_start2, int64_t total, bool walk_up) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int k = find_loop_of(seg_start2, A.nloops, g);
  const int l = A.loops[k];
  const int64_t o = A.off[l], n = A.off[l + 1] - o;
  const int64_t base = A.node_base[l];
  int32_t node = (int32_t)(n - 1 + (g - seg_start2[k]));
  {
    const int32_t seg = A.leaf_seg[base + node];
    BuildNode B;
    leaf_build(A.xyz, o, n, seg, B);
    finish_record(B, A.hdr[base + node], A.mom[base + node], true, seg, 0, 0);
  }
  const int32_t first_leaf = (int32_t)(n - 1);
  if (!walk_up) return;
  for (int guard = 0; guard < 128; ++guard) {
    const int32_t par = A.parent[base + node];
    if (par < 0) break;
    cuda::atomic_ref<int32_t, cuda::thread_scope_device> arrive(A.arrive[base + par]);
    if (arrive.fetch_add(1, cuda::memory_order_acq_rel) == 0) break;  // first arrival stops
    const int32_t cl = A.children[2 * (base + par)], cr = A.children[2 * (base + par) + 1];
    BuildNode L, R;
    if (cl >= first_leaf) leaf_build(A.xyz, o, n, A.leaf_seg[base + cl], L);
    else load_cg(A.bn + A.int_start[k] + cl, L);
    if (cr >= first_leaf) leaf_build(A.xyz, o, n, A.leaf_seg[base + cr], R);
    else load_cg(A.bn + A.int_start[k] + cr, R);
    BuildNode P;
    for (int a = 0; a < 3; ++a) {
      P.lo[a] = fmin(L.lo[a], R.lo[a]);
      P.hi[a] = fmax(L.hi[a], R.hi[a]);
      P.mid[a] = 0.5 * (P.hi[a] + P.lo[a]);
      P.t[a] = 0.0;
    }
    for (int a = 0; a < 9; ++a) P.D[a] = 0.0;
    for (int a = 0; a < 18; ++a) P.Q[a] = 0.0;
    accumulate_child(P, L);
    accumulate_child(P, R);
    P.seg_lo = L.seg_lo;
    P.seg_cnt = L.seg_cnt + R.seg_cnt;
    A.bn[A.int_start[k] + par] = P;
    finish_record(P, A.hdr[base + par], A.mom[base + par], false, 0, cl, cr);
    node = par;
  }
}

// Level-synchronous build of curve-order trees: the internal nodes of one
// height, listed in bucket[0, count), each from its two children, which
// earlier launches finished (leaves: rebuilt from their vertices). Same
// arithmetic as the walk-up of build_moments, so the same records.
__global__ void bucket_heights(const uint8_t *height, int64_t g0, int64_t total_internal, const int32_t *height_off,
                               int32_t *cursor, int32_t *bucket) {
  const int64_t g = g0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t h = g < total_internal ? height[g] : 0;
  const int32_t r = add_one_rank(cursor, h, g < total_internal);
  const int64_t pos = (int64_t)height_off[h] + r;
  if (g < total_internal && pos < total_internal) bucket[pos] = (int32_t)g;  // a count mismatch is caught on the host
}

// Nodes of height 1..kSmallHeight (at most 2^kSmallHeight segments), one
// thread each, built straight from their segments: box = the range's
// vertices; c_M, C_D and C_Q = the leaves' moments shifted to the node centre
// (for a leaf, C_D = 0 and C_Q,k = c_k c c^T / 12, so the shift adds c r^T and
// c_k r r^T with r = leaf midpoint - node centre). Algebraically the pairwise
// build of build_height; it writes no build record except for nodes whose
// parent build_height builds. Most internal nodes are this low, so this
// skips most of the 320-byte build records.
__global__ void build_small(TreeArgs A, const int64_t *seg_start, const int32_t *bucket, int64_t count,
                            const int2 *range) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const int64_t g = bucket[e];
  if (g < 0 || g >= seg_start[A.nloops]) return;  // only after a height-count mismatch, which the host reports
  const int k = find_loop_of(seg_start, A.nloops, g);
  const int l = A.loops[k];
  const int64_t o = A.off[l], n = A.off[l + 1] - o;
  const int64_t base = A.node_base[l];
  const int32_t node = (int32_t)(g - seg_start[k]);
  const int2 rg = range[g];
  const int32_t lo = rg.x, hi = rg.y & INT_MAX;
  const bool need = rg.y < 0;
  const double *V = A.xyz + 3 * o;
  BuildNode P;
  for (int a = 0; a < 3; ++a) {
    P.lo[a] = V[3 * lo + a];
    P.hi[a] = P.lo[a];
  }
  for (int32_t v = lo + 1; v <= hi; ++v) {
    const int64_t w = v == n ? 0 : v;
    for (int a = 0; a < 3; ++a) {
      const double x = V[3 * w + a];
      P.lo[a] = fmin(P.lo[a], x);
      P.hi[a] = fmax(P.hi[a], x);
    }
  }
  for (int a = 0; a < 3; ++a) {
    P.mid[a] = 0.5 * (P.hi[a] + P.lo[a]);
    P.t[a] = 0.0;
  }
  for (int a = 0; a < 9; ++a) P.D[a] = 0.0;
  for (int a = 0; a < 18; ++a) P.Q[a] = 0.0;
  const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
  for (int32_t sg = lo; sg < hi; ++sg) {
    const int64_t w0 = sg, w1 = sg + 1 == n ? 0 : sg + 1;
    double t[3], r[3];
    for (int a = 0; a < 3; ++a) {
      const double p0 = V[3 * w0 + a], p1 = V[3 * w1 + a];
      t[a] = p1 - p0;
      r[a] = (0.5 * p0 + 0.5 * p1) - P.mid[a];
    }
    for (int a = 0; a < 3; ++a) P.t[a] += t[a];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) P.D[3 * a + b] += t[a] * r[b];
    for (int kk = 0; kk < 3; ++kk)
      for (int q = 0; q < 6; ++q) {
        const int i = ii[q], j = jj[q];
        P.Q[6 * kk + q] += ((1.0 / 12.0) * t[kk]) * (t[i] * t[j]) + t[kk] * (r[i] * r[j]);
      }
  }
  P.seg_lo = lo;
  P.seg_cnt = hi - lo;
  if (need) put16(A.bn + g, P);
  const int32_t cl = A.children[2 * (base + node)], cr = A.children[2 * (base + node) + 1];
  finish_record(P, A.hdr[base + node], A.mom[base + node], false, 0, cl, cr);
}

__global__ void build_height(TreeArgs A, const int64_t *seg_start, const int32_t *bucket, int64_t count) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const int64_t g = bucket[e];
  if (g < 0 || g >= seg_start[A.nloops]) return;  // only after a height-count mismatch, which the host reports
  const int k = find_loop_of(seg_start, A.nloops, g);
  const int l = A.loops[k];
  const int64_t o = A.off[l], n = A.off[l + 1] - o;
  const int64_t base = A.node_base[l];
  const int32_t par = (int32_t)(g - seg_start[k]);
  const int32_t first_leaf = (int32_t)(n - 1);
  const int32_t cl = A.children[2 * (base + par)], cr = A.children[2 * (base + par) + 1];
  BuildNode L, R;
  if (cl >= first_leaf) leaf_build(A.xyz, o, n, A.leaf_seg[base + cl], L);
  else get16(A.bn + seg_start[k] + cl, L);
  if (cr >= first_leaf) leaf_build(A.xyz, o, n, A.leaf_seg[base + cr], R);
  else get16(A.bn + seg_start[k] + cr, R);
  BuildNode P;
  for (int a = 0; a < 3; ++a) {
    P.lo[a] = fmin(L.lo[a], R.lo[a]);
    P.hi[a] = fmax(L.hi[a], R.hi[a]);
    P.mid[a] = 0.5 * (P.hi[a] + P.lo[a]);
    P.t[a] = 0.0;
  }
  for (int a = 0; a < 9; ++a) P.D[a] = 0.0;
  for (int a = 0; a < 18; ++a) P.Q[a] = 0.0;
  accumulate_child(P, L);
  accumulate_child(P, R);
  P.seg_lo = L.seg_lo;
  P.seg_cnt = L.seg_cnt + R.seg_cnt;
  put16(A.bn + g, P);
  finish_record(P, A.hdr[base + par], A.mom[base + par], false, 0, cl, cr);
}

// ------------------------------------------------------------------ traversal
// Node pairs summed exactly, segment pair by segment pair: leaf pairs, and
// pairs that are neither far nor larger than `bucket` segments a side.
// Entry: first segment and segment count of each node (curve-order ranges;
// a leaf is its own segment, count 1). All entries of a chunk belong to one
// loop pair (slot).
struct BucketChunk {
  int32_t slot;
  int32_t count;
  int32_t pad[2];
  int4 e[32];  // lo1, lo2, cnt1, cnt2
};

// A unit of traversal work: up to 32 node pairs of one loop pair (slot).
struct Batch {
  int32_t slot;
  int32_t count;
  int2 pairs[32];
};

// Frontier of a Barnes–Hut pass: the far node pairs of one loop pair (slot),
// up to kFrontPairs per record, recorded so that the beta retry can continue
// from them instead of from the roots. Beside each pair, its separation
// ratio (|dr|^2 + eps^2 - eps^2) / (r1 + r2)^2 in FP32 (front_ratio): a pair
// whose ratio clears the retry's beta^2 by a margin far above the FP32
// rounding is far at that beta without loading its headers.
constexpr int kFrontPairs = 128;
struct FrontRec {
  int32_t slot;
  int32_t count;
  int2 pairs[kFrontPairs];
  float ratio[kFrontPairs];
};
// The ratio in FP32 from the FP64 quantities of the far test: three roundings
// (two conversions, one __fdividef of at most 2 ulp), so it lies within
// 4e-7 of the FP64 ratio. 0 (never clear) when (r1 + r2)^2 is below 1e-30,
// where the FP32 quotient is not trusted.
__device__ __forceinline__ float front_ratio(double dsq, double eps, double rs) {
  const double den = rs * rs;
  return den >= 1e-30 ? __fdividef((float)(dsq - eps), (float)den) : 0.f;
}
// A frontier pair is left to the full test unless ratio > beta^2 (1 + 1e-5):
// then |dr|^2 + eps^2 > (r1 + r2)^2 beta^2 + eps^2 holds in FP64 as well.
__device__ __forceinline__ float front_clear(double itolsq) { return (float)(itolsq * (1.0 + 1e-5)); }

struct TravArgs {
  const double *xyz;
  const int64_t *off;
  const int64_t *node_base;
  const NodeHdr *hdr;
  const NodeMom *mom;
  const int32_t *slot_loops;   // 2 per slot
  const double *itolsq;        // per slot beta^2
  double epssq;
  const Batch *in;             // this round's batches
  int64_t nin;
  Batch *out;                  // batches left over for the next round
  int64_t out_cap;
  unsigned long long *out_count;
  int32_t budget;              // iterations per batch before its stack is handed on
  int32_t bucket;              // node pairs of at most this many segments a side are summed exactly
  BucketChunk *bkt;            // exact node pairs, handed to bh_buckets
  unsigned long long *bkt_count;
  int64_t bkt_soft, bkt_cap;   // no new batch past soft; hard capacity
  unsigned long long *acc_lk;  // per slot, fixed point (2^-40 turns)
  unsigned long long *acc_err; // per slot, fixed point (2^-40)
  double *counts;              // [0] far evals, [1] leaf evals
  int2 *spill;                 // kSpill per warp
  unsigned long long *queue;   // batch queue head
  int32_t *status;             // nonzero on overflow
  // Second input source, taken after in[0, nin): frontier records of an
  // earlier pass (the beta retry's continuation); records of slots with
  // skip[slot] != 0 are passed over.
  const FrontRec *in1;
  int64_t nin1;
  const uint8_t *skip;
  // Frontier recording (the kFront instantiations): every far node pair
  // evaluated goes into a record of its slot; a slot whose records do not
  // fit gets front_lost[slot] = 1 (its retry then starts from the roots).
  FrontRec *front;
  unsigned long long *front_count;
  int64_t front_cap;
  uint8_t *front_lost;
  int32_t spill_cap;           // global spill entries per warp used (<= kSpill)
  // Learned opening criterion (frag == nullptr: off).
  LearnedCfg learned;
  double beta0;
  // Recording of training node pairs (rec == nullptr: off).
  int4 *rec;
  unsigned long long *rec_count;
  int64_t rec_cap;
  float rec_smin;
  uint32_t rec_keep;           // keep a candidate when its hash is below this
};

// Fixed-point (2^-40) accumulation: integer adds commute, so per-pair sums do
// not depend on which warp finished first.
constexpr double kFix = 1099511627776.0;  // 2^40
__device__ __forceinline__ void fix_add(unsigned long long *a, double v) {
  atomicAdd(a, (unsigned long long)__double2ll_rn(v * kFix));
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return ax * bx + ay * by + az * bz;
}

// One row of a symmetric Q (xx, yy, zz, xy, xz, yz) dotted with r.
__device__ __forceinline__ float qrow(const float *q, int i, float rx, float ry, float rz) {
  if (i == 0) return q[0] * rx + q[3] * ry + q[4] * rz;
  if (i == 1) return q[3] * rx + q[1] * ry + q[5] * rz;
  return q[4] * rx + q[5] * ry + q[2] * rz;
}

// Far-field scale factors in FP32 (1) or FP64 (0). FP32 drops the FP64
// square root and divisions from the far-field path: 96 instead of 128
// registers, five CTAs per SM instead of four, and 188.7 ms instead of
// 206.4 ms for the traversal of the 14M-segment polymer step.
#ifndef FLN_FAR_FP32_SCALE
#define FLN_FAR_FP32_SCALE 1
#endif
// The Eq. 14 weights of a node pair (compute_link.cpp:411-524), from the
// headers the classification loaded: the moment records of a far pair are
// then read once, at evaluation, and fill one 128-byte line each.
__device__ __forceinline__ float2 far_weights(const NodeHdr &h1, const NodeHdr &h2) {
  const float r1 = (float)h1.r, r2 = (float)h2.r;
  return make_float2(__fmaf_rn(r1, h2.tn, __fmul_rn(3.f, h2.dn)), __fmaf_rn(r2, h1.tn, __fmul_rn(3.f, h1.dn)));
}

// Far-field pair: monopole + Eq. 29 + Eq. 30 times 1/(4 pi |r|^3), and the
// Eq. 14 estimate with the same factor (compute_link.cpp:608-627, :411-524).
// Node 1 = u (moments m1 = "C" in the reference), node 2 = v ("D").
// ea1 = r_u |c_v| + 3 ||C_D,v|| / sqrt(3) and ea2 the same with u and v
// swapped (far_weights, from the two headers) weight the quadrupole norms.
__device__ void far_eval(const NodeMom &m1, const NodeMom &m2, float rx, float ry, float rz, double dsq, float ea1,
                         float ea2, double &sum, double &err) {
  const float *C3 = m1.D, *D3 = m2.D;
  const float C1x = m1.t[0], C1y = m1.t[1], C1z = m1.t[2];
  const float D1x = m2.t[0], D1y = m2.t[1], D1z = m2.t[2];
#if FLN_FAR_FP32_SCALE
  // 1/|r|^2 and 1/(4 pi |r|^3) in FP32 (|r| > beta (r1 + r2), far from 0).
  // Explicitly rounded operations: the error estimate (which decides the
  // beta retry) must not depend on how a kernel's compile contracts them.
  const float rinv = rsqrtf((float)dsq);
  const float rdist2 = __fmul_rn(rinv, rinv);
#else
  const float rdist2 = (float)(1.0 / dsq);
#endif
  // monopole r . (c2 x c1)
  float res = rx * (D1y * C1z - D1z * C1y) + ry * (D1z * C1x - D1x * C1z) + rz * (D1x * C1y - D1y * C1x);
  // dipole (Eq. 29)
  const float D2x = D3[5] - D3[7], D2y = D3[6] - D3[2], D2z = D3[1] - D3[3];
  const float C2x = C3[5] - C3[7], C2y = C3[6] - C3[2], C2z = C3[1] - C3[3];
  float ho = -(dot3(C1x, C1y, C1z, D2x, D2y, D2z) + dot3(C2x, C2y, C2z, D1x, D1y, D1z));
  const float Dr0 = D3[0] * rx + D3[1] * ry + D3[2] * rz, Dr1 = D3[3] * rx + D3[4] * ry + D3[5] * rz,
              Dr2 = D3[6] * rx + D3[7] * ry + D3[8] * rz;
  const float Cr0 = C3[0] * rx + C3[1] * ry + C3[2] * rz, Cr1 = C3[3] * rx + C3[4] * ry + C3[5] * rz,
              Cr2 = C3[6] * rx + C3[7] * ry + C3[8] * rz;
  // (D3 r) x C1 . r  and  (C3 r) x D1 . r
  const float t1 = rx * (Dr1 * C1z - Dr2 * C1y) + ry * (Dr2 * C1x - Dr0 * C1z) + rz * (Dr0 * C1y - Dr1 * C1x);
  const float t2 = rx * (Cr1 * D1z - Cr2 * D1y) + ry * (Cr2 * D1x - Cr0 * D1z) + rz * (Cr0 * D1y - Cr1 * D1x);
  ho -= 3.f * rdist2 * (t1 + t2);
  // quadrupole (Eq. 30)
  const float *P0 = m1.Q, *P1 = m1.Q + 6, *P2 = m1.Q + 12;
  const float *Q0 = m2.Q, *Q1 = m2.Q + 6, *Q2 = m2.Q + 12;
  const float ppx = P0[0] + P0[1] + P0[2], ppy = P1[0] + P1[1] + P1[2], ppz = P2[0] + P2[1] + P2[2];
  const float qqx = Q0[0] + Q0[1] + Q0[2], qqy = Q1[0] + Q1[1] + Q1[2], qqz = Q2[0] + Q2[1] + Q2[2];
  // -(r . (pp x D1 + C1 x qq))
  const float sx = (ppy * D1z - ppz * D1y) + (C1y * qqz - C1z * qqy);
  const float sy = (ppz * D1x - ppx * D1z) + (C1z * qqx - C1x * qqz);
  const float sz = (ppx * D1y - ppy * D1x) + (C1x * qqy - C1y * qqx);
  const float tqs1 = -(rx * sx + ry * sy + rz * sz);
  const float p01 = dot3(C3[0], C3[1], C3[2], D3[3], D3[4], D3[5]);
  const float p02 = dot3(C3[0], C3[1], C3[2], D3[6], D3[7], D3[8]);
  const float p10 = dot3(C3[3], C3[4], C3[5], D3[0], D3[1], D3[2]);
  const float p12 = dot3(C3[3], C3[4], C3[5], D3[6], D3[7], D3[8]);
  const float p20 = dot3(C3[6], C3[7], C3[8], D3[0], D3[1], D3[2]);
  const float p21 = dot3(C3[6], C3[7], C3[8], D3[3], D3[4], D3[5]);
  const float tqs2 = 2.f * (rx * (p12 - p21) + ry * (p20 - p02) + rz * (p01 - p10));
  const float tqs = tqs1 + tqs2;
  const float pXx = qrow(P1, 2, rx, ry, rz) - qrow(P2, 1, rx, ry, rz);
  const float pXy = qrow(P2, 0, rx, ry, rz) - qrow(P0, 2, rx, ry, rz);
  const float pXz = qrow(P0, 1, rx, ry, rz) - qrow(P1, 0, rx, ry, rz);
  float tqt = dot3(D1x, D1y, D1z, pXx, pXy, pXz);
  const float qXx = qrow(Q1, 2, rx, ry, rz) - qrow(Q2, 1, rx, ry, rz);
  const float qXy = qrow(Q2, 0, rx, ry, rz) - qrow(Q0, 2, rx, ry, rz);
  const float qXz = qrow(Q0, 1, rx, ry, rz) - qrow(Q1, 0, rx, ry, rz);
  tqt -= dot3(C1x, C1y, C1z, qXx, qXy, qXz);
  // r . (C3^T D2 - D3^T C2)
  const float ux = (C3[0] * D2x + C3[3] * D2y + C3[6] * D2z) - (D3[0] * C2x + D3[3] * C2y + D3[6] * C2z);
  const float uy = (C3[1] * D2x + C3[4] * D2y + C3[7] * D2z) - (D3[1] * C2x + D3[4] * C2y + D3[7] * C2z);
  const float uz = (C3[2] * D2x + C3[5] * D2y + C3[8] * D2z) - (D3[2] * C2x + D3[5] * C2y + D3[8] * C2z);
  tqt += rx * ux + ry * uy + rz * uz;
  // r^T Q r for each k
  const float a0 = rx * qrow(P0, 0, rx, ry, rz) + ry * qrow(P0, 1, rx, ry, rz) + rz * qrow(P0, 2, rx, ry, rz);
  const float a1 = rx * qrow(P1, 0, rx, ry, rz) + ry * qrow(P1, 1, rx, ry, rz) + rz * qrow(P1, 2, rx, ry, rz);
  const float a2 = rx * qrow(P2, 0, rx, ry, rz) + ry * qrow(P2, 1, rx, ry, rz) + rz * qrow(P2, 2, rx, ry, rz);
  const float b0 = rx * qrow(Q0, 0, rx, ry, rz) + ry * qrow(Q0, 1, rx, ry, rz) + rz * qrow(Q0, 2, rx, ry, rz);
  const float b1 = rx * qrow(Q1, 0, rx, ry, rz) + ry * qrow(Q1, 1, rx, ry, rz) + rz * qrow(Q1, 2, rx, ry, rz);
  const float b2 = rx * qrow(Q2, 0, rx, ry, rz) + ry * qrow(Q2, 1, rx, ry, rz) + rz * qrow(Q2, 2, rx, ry, rz);
  // -r . (D1 x a) ; r . (C1 x b)
  const float tfpp = -(rx * (D1y * a2 - D1z * a1) + ry * (D1z * a0 - D1x * a2) + rz * (D1x * a1 - D1y * a0));
  const float tfqq = rx * (C1y * b2 - C1z * b1) + ry * (C1z * b0 - C1x * b2) + rz * (C1x * b1 - C1y * b0);
  // 2 (C3 r) . (r x (D3 r))
  const float wx = ry * Dr2 - rz * Dr1, wy = rz * Dr0 - rx * Dr2, wz = rx * Dr1 - ry * Dr0;
  const float tfpq = 2.f * (Cr0 * wx + Cr1 * wy + Cr2 * wz);
  const float tf = tfpp + tfqq + tfpq;
  ho -= 1.5f * rdist2 * ((tqs + 2.f * tqt) + 5.f * rdist2 * tf);
#if FLN_FAR_FP32_SCALE
  const double mult = (double)__fmul_rn(__fmul_rn(rinv, rdist2), (float)kInvFourPi);
#else
  const double mult = 1.0 / (dsq * sqrt(dsq)) * kInvFourPi;
#endif
  sum += mult * ((double)res + (double)ho);
  const float e = __fmul_rn(rdist2, __fmaf_rn(m1.qn, ea1, __fmul_rn(m2.qn, ea2)));
  err = __fma_rn(mult, (double)e, err);
}

// Exact term of two segments in FP64 from their vertices (full turns).
__device__ __noinline__ double seg_term_fp64(const double *xyz, int64_t p0i, int64_t p1i, int64_t q0i, int64_t q1i) {
  double p0[3], p1[3], q0[3], q1[3];
  for (int a = 0; a < 3; ++a) {
    p0[a] = xyz[3 * p0i + a];
    p1[a] = xyz[3 * p1i + a];
    q0[a] = xyz[3 * q0i + a];
    q1[a] = xyz[3 * q1i + a];
  }
  // Midpoint/tangent form of compute_link.cpp:578-605.
  const double m1[3] = {0.5 * p0[0] + 0.5 * p1[0], 0.5 * p0[1] + 0.5 * p1[1], 0.5 * p0[2] + 0.5 * p1[2]};
  const double m2[3] = {0.5 * q0[0] + 0.5 * q1[0], 0.5 * q0[1] + 0.5 * q1[1], 0.5 * q0[2] + 0.5 * q1[2]};
  const double t1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
  const double t2[3] = {q1[0] - q0[0], q1[1] - q0[1], q1[2] - q0[2]};
  const double dr[3] = {m2[0] - m1[0], m2[1] - m1[1], m2[2] - m1[2]};
  const double det = dr[0] * (t2[1] * t1[2] - t2[2] * t1[1]) + dr[1] * (t2[2] * t1[0] - t2[0] * t1[2]) +
                     dr[2] * (t2[0] * t1[1] - t2[1] * t1[0]);
  double al[3], be[3], ga[3], de[3];
  for (int a = 0; a < 3; ++a) {
    al[a] = dr[a] + 0.5 * (t1[a] - t2[a]);
    be[a] = dr[a] + 0.5 * (-t2[a] - t1[a]);
    ga[a] = dr[a] + 0.5 * (t2[a] - t1[a]);
    de[a] = dr[a] + 0.5 * (t2[a] + t1[a]);
  }
  auto dt = [](const double *x, const double *y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
  const double la = sqrt(dt(al, al)), lb = sqrt(dt(be, be)), lc = sqrt(dt(ga, ga)), ld = sqrt(dt(de, de));
  const double ac = dt(al, ga);
  const double div1 = la * lb * lc + dt(al, be) * lc + ac * lb + dt(be, ga) * la;
  const double div2 = la * ld * lc + dt(al, de) * lc + ac * ld + dt(de, ga) * la;
  const double x = div1 * div2 - det * det;
  const double s = (det == 0) ? copysign(1.0, div1) + copysign(1.0, div2) : (div1 + div2);
  const double y = det * s;
  const double sg = (det == 0) ? -copysign(1.0, div1) : copysign(1.0, det);
  return kInvTwoPi * atan2(y, x) + (((s < 0) || ((s == 0) && (det < 0))) ? sg : 0.0);
}

// Exact segment-pair terms in FP32, in the vertex form of the reference's
// direct sum (compute_link.cpp:126-178): for segment p0 -> p1 of loop 1 and
// q0 -> q1 of loop 2, a = q0 - p0, b = q0 - p1, c = q1 - p1, d = q1 - p0,
// e = p1 - p0, f = q1 - q0, and
//   det  = a . (f x e)
//   div1 = |a||b||c| + (a.b)|c| + (c.a)|b| + (c.b)|a|
//   div2 = |a||d||c| + (a.d)|c| + (c.a)|d| + (c.d)|a|
//   term = atan2(det (div1 + div2), div1 div2 - det^2) / 2pi (+ the branch turn).
// The vertices are FP32 coordinates relative to an FP64 origin near the two
// segments (the exact-list kernel's entry origin); e = p1 - p0 is an FP64
// difference rounded once; b = a - e, c = d - e and f = d - a are FP32.
// Walking q along loop 2 for a fixed p, step k+1's a, b are step k's d, c,
// so a step forms two new vectors and two norms (walk_start_f, walk_step_f).
// Segments closer than the longer one's length (squared norms compared) are
// left to FP64 (seg_term_fp64).

// arctan(t) for |t| <= 1/4 from its Maclaurin series t - t^3/3 + t^5/5 - t^7/7
// + t^9/9; the first omitted term is below 2.2e-8 |t|, under FP32 rounding.
__device__ __forceinline__ float atan_quarter(float t) {
  const float u = t * t;
  float p = fmaf(u, 1.0f / 9.0f, -1.0f / 7.0f);
  p = fmaf(p, u, 1.0f / 5.0f);
  p = fmaf(p, u, -1.0f / 3.0f);
  p = fmaf(p, u, 1.0f);
  return p * t;
}

__device__ __forceinline__ float norm_of(float sq) { return sq * rsqrtf(sq); }

__device__ __forceinline__ void load3(const double *xyz, int64_t v, double *p) {
  p[0] = xyz[3 * v];
  p[1] = xyz[3 * v + 1];
  p[2] = xyz[3 * v + 2];
}

// Traversal steps a warp takes on one batch per round before it hands the
// rest of its stack on as new batches (fln_params.bh_budget 0: this).
// Traversal time of the 14M-segment polymer step on B200, leaf pairs only:
// 128 -> 208.2 ms, 256 -> 207.4 ms, 512 -> 222.5 ms, 1024 -> 240.2 ms; with
// the exact list, 128 -> 48.0 ms and 256 -> 49.6 ms.
#ifndef FLN_BH_BUDGET
#define FLN_BH_BUDGET kDefaultBhBudget
#endif
// Software prefetch of node records (generic addresses; the records are
// valid device memory). Bit 0: the next step's headers into L1; bit 1: the
// moment records of queued far-field and leaf pairs into L1. Same step:
// none 207.4 ms, bit 1 206.5 ms, bit 0 211.7 ms, both 212.2 ms.
// Node pairs (neither far nor split further) of at most this many segments
// a side are summed exactly, segment pair by segment pair.
#ifndef FLN_BH_BUCKET
#define FLN_BH_BUCKET 8
#endif
#ifndef FLN_BH_PREFETCH
#define FLN_BH_PREFETCH 2
#endif
__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.L1 [%0];" ::"l"(p)); }
template <class T>
__device__ __forceinline__ void prefetch_record(const T *p) {
  prefetch_l1(p);
  if constexpr (sizeof(T) > 128) prefetch_l1(reinterpret_cast<const char *>(p) + sizeof(T) - 1);
}

// stack[0, n) = stack[k, k + n), warp-wide, in passes of 32 that read before
// they write: the lanes of a warp need not run the passes in step
// (independent thread scheduling), so a lane ahead must not overwrite
// entries that a lagging lane has yet to read. Out of line: it runs only
// when a stack spills, and inlined it costs the traversal registers.
__device__ __noinline__ void shift_down(int2 *stack, int k, int n, int lane) {
  for (int xb = 0; xb < n; xb += 32) {
    const int x = xb + lane;
    int2 v = make_int2(0, 0);
    if (x < n) v = stack[k + x];
    __syncwarp();
    if (x < n) stack[x] = v;
    __syncwarp();
  }
}

// Appends n (<= 32) far node pairs and their separation ratios (front_ratio),
// one per lane (lanes < n), to the warp's
// open frontier record of `slot`, reserving records as they fill. The open
// record is (fr, ffill); fr < 0 means none. A record is closed (its header
// written) when it is full, when the warp moves to another batch, or when the
// warp finishes.
__device__ __forceinline__ void front_close(const TravArgs &A, int &fr, int &ffill, int slot, int lane) {
  if (fr >= 0 && lane == 0 && fr < A.front_cap) {
    A.front[fr].slot = slot;
    A.front[fr].count = ffill;
  }
  fr = -1;
  ffill = 0;
}
__device__ __forceinline__ void front_put(const TravArgs &A, int &fr, int &ffill, int slot, int2 q, float ratio,
                                          int n, int lane) {
  const int need = (fr < 0 ? 1 : 0) + (ffill + n > kFrontPairs ? 1 : 0);
  int c = 0;  // record index (clamped: past the capacity only "lost" matters)
  if (lane == 0 && need)
    c = (int)min(atomicAdd(A.front_count, (unsigned long long)need), (unsigned long long)(INT_MAX - 1));
  c = __shfl_sync(0xffffffffu, c, 0);
  const int cur = fr < 0 ? c : fr, nxt = fr < 0 ? c + 1 : c;
  const int pos = ffill + lane;
  const int dst = pos < kFrontPairs ? cur : nxt;
  if (lane < n && dst < A.front_cap) {
    const int at = pos < kFrontPairs ? pos : pos - kFrontPairs;
    A.front[dst].pairs[at] = q;
    A.front[dst].ratio[at] = ratio;
  }
  if (lane == 0 && (cur >= A.front_cap || (ffill + n > kFrontPairs && nxt >= A.front_cap))) A.front_lost[slot] = 1;
  if (ffill + n >= kFrontPairs) {
    int full = cur;
    int nfull = kFrontPairs;
    front_close(A, full, nfull, slot, lane);
    fr = ffill + n > kFrontPairs ? nxt : -1;
    ffill = ffill + n - kFrontPairs;
  } else {
    fr = cur;
    ffill += n;
  }
}

// One warp per batch. The warp runs the two-tree traversal of its batch's
// node pairs for at most `budget` steps; whatever is still on its stack then
// is written out as new batches for the next round, so a heavy loop pair
// spreads over many warps while light pairs finish in one go.
// kLearn: the learned opening criterion (A.learned); kRecord: sampling of
// training node pairs (A.rec). kMode: 0 plain; 1 the first pass, which
// records its frontier (A.front); 2 the beta retry continued from a frontier
// (A.in1 records).
// Input: the batches in[0, nin), then the frontier records in1[0, nin1)
// (up to kFrontPairs node pairs each), taken one at a time from A.queue.
//
// The continued retry (kMode 2) keeps the first pass's far-field and error
// sums of the slot. A node pair's far-field value and estimate do not depend
// on beta, so a frontier pair that is still far at the slot's beta is left
// alone: its value is already in the sums. Most such pairs are recognised at
// intake from the ratio recorded with them (front_clear); the rest go on the
// stack marked by bit 31 of their first node id and take the full test. A frontier pair that is opened now has its first-pass value and
// estimate subtracted (queued with a negative squared separation, evaluated
// at the one far-field call site, so the value is the one the first pass
// added) and is then exact or split like any pair.
constexpr int kFrontFlag = int(0x80000000u);
// Sum of a per-lane 32-bit count over the warp, in FP64 (no overflow).
__device__ __forceinline__ double warp_sum_u32(unsigned v) {
  unsigned long long s = v;
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return (double)s;
}
template <bool kLearn, bool kRecord, int kMode>
__device__ __forceinline__ void traverse(const TravArgs &A) {
  constexpr bool kFront = kMode == 1, kCont = kMode == 2;
  __shared__ int2 s_stack[kWarps][kStack];
  __shared__ int2 s_far[kWarps][64];
  __shared__ float4 s_farv[kWarps][64];  // separation (x, y, z) and its square (negative: subtract), per queued far pair
  __shared__ float2 s_farr[kWarps][64];  // the two Eq. 14 weights (far_weights)
  __shared__ float s_fart[kWarps][kFront ? 64 : 1];  // separation ratios for the frontier (front_ratio)
  __shared__ std::conditional_t<kLearn, MlpFrag, int> s_mlp;
  // Staged moment records (FLN_BH_TMA_MOM): node 1's in slots [0, 16), node
  // 2's in [16, 32), one barrier per warp.
  __shared__ __align__(128) float4 s_stage[kWarps][FLN_BH_TMA_MOM ? 2 * kStagePairs * kSlotF4 : 1];
  __shared__ __align__(8) uint64_t s_mbar[kWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int gw = blockIdx.x * kWarps + w;
  float4 *stage = s_stage[w];
  uint64_t *mbar = &s_mbar[w];
  uint32_t mphase = 0;
  const bool staged = FLN_BH_TMA_MOM != 0;
  bool sfail = false;  // a staging wait ran out (status 16)
  if (staged) {
    if (lane == 0) mbar_init(mbar, 1);
    __syncwarp();
  }
  int2 *stack = s_stack[w];
  int2 *farq = s_far[w];
  float4 *farv = s_farv[w];
  float2 *farr = s_farr[w];
  float *fart = s_fart[w];
  if constexpr (kLearn) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(A.learned.frag);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&s_mlp);
    for (int x = threadIdx.x; x < (int)(sizeof(MlpFrag) / 4); x += blockDim.x) dst[x] = src[x];
    __syncthreads();
  }
  int2 *spill = A.spill + (size_t)gw * kSpill;
  // Per-lane counts in 32 bits (a lane classifies at most one node pair per
  // step, and a launch's steps are bounded by its batches' budgets).
  unsigned nfar = 0, nent = 0;
  // kCont: frontier pairs kept far and opened, counted in shared memory (they
  // change once per frontier pair; registers are the traversal's limit).
  __shared__ unsigned s_fcount[kWarps][kCont ? 2 : 1];
  if constexpr (kCont) {
    if (lane == 0) {
      s_fcount[w][0] = 0;
      s_fcount[w][1] = 0;
    }
    __syncwarp();
  }
  // kFront: the warp's open frontier record, its fill and its slot, kept in
  // shared memory (read and written once per 32 far pairs) rather than in
  // registers across the traversal loop.
  __shared__ int s_fstate[kWarps][kFront ? 3 : 1];
  if constexpr (kFront) {
    if (lane == 0) {
      s_fstate[w][0] = -1;
      s_fstate[w][1] = 0;
      s_fstate[w][2] = -1;
    }
    __syncwarp();
  }
  const long long total = A.nin + A.nin1;
  for (;;) {
    if (sfail) break;
    long long b = 0;
    if (lane == 0) {
      // Past the soft limit of the exact list this round takes no new batch
      // (they carry over).
      const bool full = (int64_t)*(volatile unsigned long long *)A.bkt_count > A.bkt_soft;
      b = full ? total : (long long)atomicAdd(A.queue, 1ULL);
    }
    b = __shfl_sync(0xffffffffu, b, 0);
    if (b >= total) break;
    int slot, cnt0;
    const int2 *src;
    const bool from_front = b >= A.nin;
    if (!from_front) {
      slot = A.in[b].slot;
      cnt0 = A.in[b].count;
      src = A.in[b].pairs;
    } else {
      const FrontRec &r = A.in1[b - A.nin];
      slot = r.slot;
      cnt0 = r.count;
      src = r.pairs;
      if (cnt0 <= 0 || A.skip[slot]) continue;
    }
    if constexpr (kFront) {
      int frec = s_fstate[w][0], ffill = s_fstate[w][1];
      const int fslot = s_fstate[w][2];
      __syncwarp();
      // Every batch starts its own records: a record then holds the far
      // pairs of one batch, in that batch's traversal order, whichever warp
      // ran it and whatever it ran before. (A record shared by consecutive
      // batches of a slot would group the retry's far-field sums by the
      // warps' timing, and their last bits with it.)
      front_close(A, frec, ffill, fslot, lane);
      if (lane == 0) {
        s_fstate[w][0] = frec;
        s_fstate[w][1] = ffill;
        s_fstate[w][2] = slot;
      }
      __syncwarp();
    }
    const int l1 = A.slot_loops[2 * slot], l2 = A.slot_loops[2 * slot + 1];
    const NodeHdr *H1 = A.hdr + A.node_base[l1], *H2 = A.hdr + A.node_base[l2];
    const NodeMom *M1 = A.mom + A.node_base[l1], *M2 = A.mom + A.node_base[l2];
    const double itolsq = A.itolsq[slot], eps = A.epssq;
    // Threshold of the learned criterion: tau x (beta0 / beta)^4 in later passes.
    const float log10_tau = A.learned.log10_tau + 2.f * (float)log10(A.beta0 * A.beta0 / itolsq);
    int top = cnt0;
    if (kCont && from_front) {
      // Frontier pairs still clearly far at this slot's beta keep their
      // first-pass value and need no classification; the others go on the
      // stack, marked, for the full test.
      const float clear = front_clear(itolsq);
      const float *ratio = A.in1[b - A.nin].ratio;
      top = 0;
      for (int x0 = 0; x0 < cnt0; x0 += 32) {
        const int x = x0 + lane;
        int2 v = make_int2(0, 0);
        bool keep = false;
        if (x < cnt0) {
          v = src[x];
          keep = !(ratio[x] > clear);
        }
        const unsigned km = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_fcount[w][0] += (unsigned)(min(cnt0 - x0, 32) - __popc(km));
        v.x |= kFrontFlag;
        if (keep) stack[top + __popc(km & ((1u << lane) - 1))] = v;
        top += __popc(km);
      }
    } else {
      for (int x = lane; x < cnt0; x += 32) stack[x] = src[x];
    }
    int nspill = 0, nf = 0, steps = 0;
    int bc = -1;  // open chunk of the exact list
    int bfill = 0;      // entries in it
    bool overflow = false;
    double sum = 0.0, err = 0.0;
    __syncwarp();
    for (bool done = false; !done;) {
      if (top == 0 && nspill > 0) {  // refill from the spill buffer
        const int k = min(nspill, kStack / 2);
        for (int x = lane; x < k; x += 32) stack[x] = spill[nspill - k + x];
        nspill -= k;
        top = k;
        __syncwarp();
      }
      if (top == 0) done = true;
      if (!done && steps >= A.budget) {  // hand the rest on as new batches
        const int total_e = top + nspill;
        const int nb = (total_e + 31) / 32;
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(A.out_count, (unsigned long long)nb);
        at = __shfl_sync(0xffffffffu, at, 0);
        if ((long long)(at + nb) <= A.out_cap) {
          for (int q = 0; q < nb; ++q) {
            const int e = 32 * q + lane;
            if (e < total_e) A.out[at + q].pairs[lane] = e < nspill ? spill[e] : stack[e - nspill];
            if (lane == 0) {
              A.out[at + q].slot = slot;
              A.out[at + q].count = min(32, total_e - 32 * q);
            }
          }
          top = 0;
          nspill = 0;
          __syncwarp();
          done = true;
        } else {
          // No room left: mark the reserved batches below the capacity empty
          // and finish this batch here.
          if (lane == 0)
            for (int q = 0; q < nb && (long long)(at + q) < A.out_cap; ++q) {
              A.out[at + q].slot = slot;
              A.out[at + q].count = 0;
            }
          steps = INT_MIN;
        }
      }
      if (!done) {
        ++steps;
        const int cnt = min(top, 32);
        const bool act = lane < cnt;
        int2 pr = make_int2(0, 0);
        if (act) pr = stack[top - cnt + lane];
        __syncwarp();
        top -= cnt;
        bool fpair = false;  // a frontier pair of the continued retry
        if constexpr (kCont) {
          fpair = pr.x < 0;
          pr.x &= ~kFrontFlag;
        }
        int kind = 0;  // 0 none, 1 exact (leaf pair or bucket), 2 far, 3 split
        int4 ex = make_int4(0, 0, 1, 1);
        int2 c0 = make_int2(0, 0), c1 = make_int2(0, 0);
        float sep = 0.f;
        double dsq = 0.0;
        float4 fv = make_float4(0.f, 0.f, 0.f, 0.f);
        float2 fr = make_float2(0.f, 0.f);
        float fratio = 0.f;  // separation ratio for the frontier (kFront)
        int mincnt = 0;  // segments of the smaller node (learned criterion)
        if (act) {
          const NodeHdr h1 = load_hdr(H1 + pr.x), h2 = load_hdr(H2 + pr.y);
          const double dx = h2.m[0] - h1.m[0], dy = h2.m[1] - h1.m[1], dz = h2.m[2] - h1.m[2];
          const bool leaf1 = h1.left < 0, leaf2 = h2.left < 0;
          const double rs = h1.r + h2.r;
          dsq = dx * dx + dy * dy + dz * dz + eps;
          fv = make_float4((float)dx, (float)dy, (float)dz, (float)dsq);
          fr = far_weights(h1, h2);
          if constexpr (kFront) fratio = front_ratio(dsq, eps, rs);
          sep = (float)(sqrt(dsq) / rs);
          if constexpr (kLearn) mincnt = min(h1.cnt, h2.cnt);
          if (leaf1 && leaf2) {
            kind = 1;
            ex = make_int4(h1.lo, h2.lo, 1, 1);
          } else if (dsq > rs * rs * itolsq + eps) {
            kind = 2;
          } else if (h1.cnt <= A.bucket && h2.cnt <= A.bucket) {
            kind = 1;
            ex = make_int4(h1.lo, h2.lo, h1.cnt, h2.cnt);
          } else {
            kind = 3;
            const bool split2 = (!leaf1 && !leaf2) ? (h2.rsq > h1.rsq) : !leaf2;
            if (split2) {
              c0 = make_int2(pr.x, h2.left);
              c1 = make_int2(pr.x, h2.right);
            } else {
              c0 = make_int2(h1.left, pr.y);
              c1 = make_int2(h1.right, pr.y);
            }
          }
        }
        // Recording for training: opened pairs and far pairs near the threshold.
        if (kRecord && act && kind != 1 && sep >= A.rec_smin && sep * sep <= 1.5625f * (float)itolsq) {
          uint32_t hsh = (uint32_t)slot * 0x9E3779B1u ^ (uint32_t)pr.x * 0x85EBCA77u ^ (uint32_t)pr.y * 0xC2B2AE3Du;
          hsh ^= hsh >> 15;
          hsh *= 0x2C1B3C6Du;
          hsh ^= hsh >> 12;
          if (hsh < A.rec_keep) {
            const unsigned long long at = atomicAdd(A.rec_count, 1ULL);
            if ((int64_t)at < A.rec_cap) A.rec[at] = make_int4(slot, pr.x, pr.y, 0);
          }
        }
        // Learned criterion: a pair the beta test opens but whose separation is
        // at least s_min is accepted as far-field when the MLP predicts its
        // error below tau; it then adds its Eq. 14 estimate to err like any
        // far-field pair. The warp's candidates are evaluated at once, and only
        // when there are at least min_cand (>= 1) of them.
        if constexpr (kLearn) {
          const bool cand = kind == 3 && sep >= A.learned.s_min && mincnt >= A.learned.min_seg;
          if (__popc(__ballot_sync(0xffffffffu, cand)) >= A.learned.min_cand) {
            float f[kMlpIn];
            for (int k = 0; k < kMlpIn; ++k) f[k] = 0.f;
            if (cand) {
              const NodeHdr h1 = load_hdr(H1 + pr.x), h2 = load_hdr(H2 + pr.y);
              mlp_features(sep, (float)h1.r, (float)h2.r, dsq, h1.tn, h2.tn, h1.dn, h2.dn, M1[pr.x].qn, M2[pr.y].qn, f);
            }
            const float y = mlp_warp_predict(reinterpret_cast<const MlpFrag &>(s_mlp), f);
            if (cand && y < log10_tau) kind = 2;
          }
        }
        // Continued retry: a frontier pair still far keeps its first-pass
        // value; one that opens gives it back (subtract) and goes on.
        bool sub = false;
        if constexpr (kCont) {
          bool kept = false;
          if (fpair) {
            if (kind == 2) {
              kind = 0;
              kept = true;
            } else {
              sub = true;
              fv.w = -fv.w;
            }
          }
          const unsigned km = __ballot_sync(0xffffffffu, kept), um = __ballot_sync(0xffffffffu, sub);
          if (lane == 0) {
            s_fcount[w][0] += (unsigned)__popc(km);
            s_fcount[w][1] += (unsigned)__popc(um);
          }
        }
        const unsigned sm = __ballot_sync(0xffffffffu, kind == 3);
        const int ns = __popc(sm);
        if (top + 2 * ns > kStack) {  // spill the oldest half
          const int k = top / 2;
          if (nspill + k > A.spill_cap) {
            overflow = true;
            done = true;
          } else {
            for (int x = lane; x < k; x += 32) spill[nspill + x] = stack[x];
            __syncwarp();
            shift_down(stack, k, top - k, lane);
            nspill += k;
            top -= k;
            __syncwarp();
          }
        }
        if (!overflow) {
          if (kind == 3) {
            const int rank = __popc(sm & ((1u << lane) - 1));
            stack[top + 2 * rank] = c0;
            stack[top + 2 * rank + 1] = c1;
          }
          top += 2 * ns;
          const unsigned fm = __ballot_sync(0xffffffffu, kind == 2 || sub);
          const unsigned lm = __ballot_sync(0xffffffffu, kind == 1);
          if (kind == 2 || sub) {
            const int at = nf + __popc(fm & ((1u << lane) - 1));
            farq[at] = pr;
            farv[at] = fv;
            farr[at] = fr;
            if constexpr (kFront) fart[at] = fratio;
          }
#if FLN_BH_PREFETCH & 2
          if (kind == 2 || sub) {
            prefetch_record(M1 + pr.x);
            prefetch_record(M2 + pr.y);
          }
#endif
          nf += __popc(fm);
          if (lm) {  // append the exact pairs to the list, 32 entries per chunk
            const int ne = __popc(lm), pos = bfill + __popc(lm & ((1u << lane) - 1));
            nent += ne;
            const int need = (bc < 0 ? 1 : 0) + (bfill + ne > 32 ? 1 : 0);
            int c = 0;  // chunk index (clamped: past the capacity the status flags it)
            if (lane == 0 && need)
              c = (int)min(atomicAdd(A.bkt_count, (unsigned long long)need), (unsigned long long)(INT_MAX - 1));
            c = __shfl_sync(0xffffffffu, c, 0);
            const int cur = bc < 0 ? c : bc, nxt = bc < 0 ? c + 1 : c;
            const int dst = pos < 32 ? cur : nxt;
            if (kind == 1) {
              if (dst < A.bkt_cap) A.bkt[dst].e[pos & 31] = ex;
              else atomicOr(A.status, 4);
            }
            if (bfill + ne >= 32) {
              if (lane == 0 && cur < A.bkt_cap) {
                A.bkt[cur].slot = slot;
                A.bkt[cur].count = 32;
              }
              bc = bfill + ne > 32 ? nxt : -1;
              bfill = bfill + ne - 32;
            } else {
              bc = cur;
              bfill += ne;
            }
          }
          __syncwarp();
        }
      }
      // Far-field evaluation, 32 queued pairs at a time, and what is left
      // once the batch is done: the one far-field call site of the kernel
      // (a subtraction then gives back exactly what the first pass added).
      const int drain = staged ? kStagePairs : 32;
      while (nf >= drain || (done && nf > 0)) {
        const int m = min(nf, drain);
        int2 q = make_int2(0, 0);
        if (lane < m) q = farq[nf - m + lane];
        if constexpr (kFront) {
          int frec = s_fstate[w][0], ffill = s_fstate[w][1];
          __syncwarp();
          front_put(A, frec, ffill, slot, q, lane < m ? fart[nf - m + lane] : 0.f, m, lane);
          if (lane == 0) {
            s_fstate[w][0] = frec;
            s_fstate[w][1] = ffill;
          }
          __syncwarp();
        }
        if (staged) {
          if (lane == 0) mbar_expect(mbar, (uint32_t)(m * 2 * sizeof(NodeMom)));
          __syncwarp();
          if (lane < m) {
            bulk_record(stage + kSlotF4 * lane, M1 + q.x, mbar);
            bulk_record(stage + kSlotF4 * (kStagePairs + lane), M2 + q.y, mbar);
          }
          if (!__all_sync(0xffffffffu, mbar_wait(mbar, mphase))) {
            sfail = true;
            if (lane == 0) atomicOr(A.status, 16);
            done = true;
            break;
          }
          mphase ^= 1u;
        }
        if (lane < m) {
          const float4 v = farv[nf - m + lane];
          const float2 rr = farr[nf - m + lane];  // Eq. 14 weights
          double fs = 0.0, fe = 0.0;
          if (staged)
            far_eval(stage_read(stage, lane), stage_read(stage, kStagePairs + lane), v.x, v.y, v.z,
                     (double)fabsf(v.w), rr.x, rr.y, fs, fe);
          else
            far_eval(load_mom(M1 + q.x), load_mom(M2 + q.y), v.x, v.y, v.z, (double)fabsf(v.w), rr.x, rr.y, fs, fe);
          if (v.w < 0.f) {
            sum -= fs;
            err -= fe;
          } else {
            sum += fs;
            err += fe;
            nfar += 1;
          }
        }
        nf -= m;
        __syncwarp();
      }
    }
    if (bc >= 0 && lane == 0 && bc < A.bkt_cap) {
      A.bkt[bc].slot = slot;
      A.bkt[bc].count = bfill;
    }
    if (overflow && lane == 0) atomicExch(A.status, 1);
    for (int o = 16; o; o >>= 1) {
      sum += __shfl_xor_sync(0xffffffffu, sum, o);
      err += __shfl_xor_sync(0xffffffffu, err, o);
    }
    if (lane == 0) {
      fix_add(A.acc_lk + slot, sum);
      fix_add(A.acc_err + slot, err);
    }
  }
  if constexpr (kFront) {
    int frec = s_fstate[w][0], ffill = s_fstate[w][1];
    const int fslot = s_fstate[w][2];
    __syncwarp();
    front_close(A, frec, ffill, fslot, lane);
  }
  // A staging wait that ran out leaves copies in flight: give them another
  // bounded wait before the CTA's shared memory is released.
  if (sfail) mbar_wait(mbar, mphase);
  const double wfar = warp_sum_u32(nfar);
  if (lane == 0) {
    atomicAdd(A.counts, wfar);
    atomicAdd(A.counts + 5, (double)nent);
  }
  if constexpr (kCont) {
    __syncwarp();
    const double wreuse = (double)s_fcount[w][0], wsub = (double)s_fcount[w][1];
    if (lane == 0) {
      atomicAdd(A.counts + 6, wreuse);
      atomicAdd(A.counts + 7, wsub);
    }
  }
}

// Exact node pairs of a round: one warp per chunk (up to 32 entries of one
// loop pair). Entry j is a block of cnt1 x cnt2 segment pairs: segments
// [lo1, lo1 + cnt1) of loop 1 against [lo2, lo2 + cnt2) of loop 2.
//
// Per entry, an FP64 origin o_j (midway between vertex lo1 of loop 1 and
// vertex lo2 of loop 2) and the entry's cnt2 + 1 loop-2 vertices, relative to
// o_j and rounded to FP32, are staged in shared memory once (the lane of the
// entry writes them; .w holds the squared length of the loop-2 segment that
// starts there). The work is then cut into rows: one loop-1 segment against
// all cnt2 loop-2 segments of its entry. A lane takes a row, forms its two
// loop-1 vertices relative to o_j (FP64 difference, rounded once) and walks
// the staged loop-2 vertices in the vertex form of the reference's direct sum
// (walk_step_f). Rows are handed out in order of their length, so the lanes
// of a pass walk about as far. Segment pairs left to FP64 (closer than the
// longer segment's length) wait in a per-warp queue and are evaluated 32 at
// a time with full warps. Sums go to the chunk's loop pair in fixed point.
struct BucketArgs {
  const double *xyz;
  const int64_t *off;
  const int32_t *slot_loops;
  const BucketChunk *chunks;
  const unsigned long long *count;
  int64_t cap;
  unsigned long long *acc_lk;  // per slot: the exact sums
  double *counts;              // [1] segment pairs summed exactly
};

constexpr int kBkWarps = 4;     // warps per CTA
constexpr int kStageV = 320;    // staged loop-2 vertices per warp (32 entries of up to 9, or 16 of up to 17)

struct SegWalkF {        // the carried state of a walk along loop 2 (FP32)
  float ax, ay, az;      // a = q_k - p0
  float bx, by, bz;      // b = q_k - p1
  float aa, bb, ab;      // |a|^2, |b|^2, a.b
  float la, lb;          // |a|, |b|
  float mn;              // min(|a|^2, |b|^2)
};

__device__ __forceinline__ SegWalkF walk_start_f(float p0x, float p0y, float p0z, float4 q0, float ex, float ey,
                                                 float ez) {
  SegWalkF w;
  w.ax = q0.x - p0x;
  w.ay = q0.y - p0y;
  w.az = q0.z - p0z;
  w.bx = w.ax - ex;
  w.by = w.ay - ey;
  w.bz = w.az - ez;
  w.aa = dot3(w.ax, w.ay, w.az, w.ax, w.ay, w.az);
  w.bb = dot3(w.bx, w.by, w.bz, w.bx, w.by, w.bz);
  w.ab = dot3(w.ax, w.ay, w.az, w.bx, w.by, w.bz);
  w.la = norm_of(w.aa);
  w.lb = norm_of(w.bb);
  w.mn = fminf(w.aa, w.bb);
  return w;
}

// One step q0 -> q1 of the walk (q1.w unused; ff = |q1 - q0|^2 comes from
// the staged vertex q0), from FP32 coordinates relative to an origin: reads
// the state w at q0 and writes the state o at q1 (a walk alternates two
// states, so that no step copies one). The
// arctangent: when div1 + div2 > 0 and |y| < x / 4 the principal branch by
// the 5-term series (|angle| < 0.245), otherwise atan2f and the branch turn
// of the reference (compute_link.cpp:151-175). (A branch-free arctangent,
// range reduced by pi/6, measured slower on B200: the slow path is rare
// enough that the warps seldom diverge on it.)
__device__ __forceinline__ bool walk_step_f(const SegWalkF &w, SegWalkF &o, float p0x, float p0y, float p0z, float4 q1,
                                            float ff, float ex, float ey, float ez, float ee, float &acc, float &turns) {
  const float dx = q1.x - p0x, dy = q1.y - p0y, dz = q1.z - p0z;
  const float fx = dx - w.ax, fy = dy - w.ay, fz = dz - w.az;
  const float cx = dx - ex, cy = dy - ey, cz = dz - ez;
  const float cc = dot3(cx, cy, cz, cx, cy, cz), dd = dot3(dx, dy, dz, dx, dy, dz);
  const float cd = dot3(cx, cy, cz, dx, dy, dz);
  const float lc = norm_of(cc), ld = norm_of(dd);
  const float mn = fminf(cc, dd);
  const bool near = fminf(w.mn, mn) <= fmaxf(ee, ff);
  // Every step forms the term; a near step (left to FP64) drops it by a
  // select, so only the rare slow arctangent is a branch (0.6 % faster than
  // branching on the near test, which about 9 % of the steps take).
  {
    const float ca = dot3(cx, cy, cz, w.ax, w.ay, w.az), cb = dot3(cx, cy, cz, w.bx, w.by, w.bz);
    const float ad = dot3(w.ax, w.ay, w.az, dx, dy, dz);
    const float det = w.ax * (fy * ez - fz * ey) + w.ay * (fz * ex - fx * ez) + w.az * (fx * ey - fy * ex);
    const float t = w.la * lc;
    const float div1 = t * w.lb + w.ab * lc + ca * w.lb + cb * w.la;
    const float div2 = t * ld + ad * lc + ca * ld + cd * w.la;
    const float x = div1 * div2 - det * det;
    // s = div1 + div2 serves the fast path also when det = 0: y is then a
    // zero of det's sign under both forms of s, and the test below holds
    // under both exactly when div1 > 0 and div2 > 0. The other branch forms
    // the reference's s (compute_link.cpp:151-175).
    float s = div1 + div2;
    float y = det * s;
    const bool fast = s > 0.f && fabsf(y) < 0.25f * x;
    float term = atan_quarter(__fdividef(y, x));  // principal branch, |angle| < 0.245
    if (!fast && !near) {
      if (det == 0.f) {
        s = copysignf(1.f, div1) + copysignf(1.f, div2);
        y = det * s;
      }
      term = atan2f(y, x);
      const float sg = (det == 0.f) ? -copysignf(1.f, div1) : copysignf(1.f, det);
      if ((s < 0.f) || ((s == 0.f) && (det < 0.f))) turns += sg;
    }
    acc += near ? 0.f : term;
  }
  o.ax = dx; o.ay = dy; o.az = dz;
  o.bx = cx; o.by = cy; o.bz = cz;
  o.aa = dd; o.bb = cc; o.ab = cd;
  o.la = ld; o.lb = lc;
  o.mn = mn;
  return !near;
}

// Exact term of segment s1 of loop 1 (vertex offset o1, n1 segments) and
// segment s2 of loop 2 as the exact-list kernel forms it for a 1 x 1 entry:
// origin midway between the two segments' first vertices (FP64), vertices
// relative to it in FP32, one step of walk_step_f, FP64 for near segments.
// The persistent and split schedules sum their leaf pairs with it, so a leaf
// pair gets the same value in every schedule.
__device__ __forceinline__ double seg_pair_term(const double *xyz, int64_t o1, int64_t n1, int64_t s1, int64_t o2,
                                                int64_t n2, int64_t s2) {
  const int64_t a0 = o1 + s1, a1 = o1 + (s1 + 1 == n1 ? 0 : s1 + 1);
  const int64_t b0 = o2 + s2, b1 = o2 + (s2 + 1 == n2 ? 0 : s2 + 1);
  double p0[3], p1[3], q0[3], q1[3];
  load3(xyz, a0, p0);
  load3(xyz, a1, p1);
  load3(xyz, b0, q0);
  load3(xyz, b1, q1);
  const double ox = 0.5 * p0[0] + 0.5 * q0[0], oy = 0.5 * p0[1] + 0.5 * q0[1], oz = 0.5 * p0[2] + 0.5 * q0[2];
  float4 f0 = make_float4((float)(q0[0] - ox), (float)(q0[1] - oy), (float)(q0[2] - oz), 0.f);
  const float4 f1 = make_float4((float)(q1[0] - ox), (float)(q1[1] - oy), (float)(q1[2] - oz), 0.f);
  const float fx = f1.x - f0.x, fy = f1.y - f0.y, fz = f1.z - f0.z;
  f0.w = dot3(fx, fy, fz, fx, fy, fz);
  const float p0x = (float)(p0[0] - ox), p0y = (float)(p0[1] - oy), p0z = (float)(p0[2] - oz);
  const float ex = (float)(p1[0] - p0[0]), ey = (float)(p1[1] - p0[1]), ez = (float)(p1[2] - p0[2]);
  const float ee = dot3(ex, ey, ez, ex, ey, ez);
  const SegWalkF w = walk_start_f(p0x, p0y, p0z, f0, ex, ey, ez);
  SegWalkF o;
  float acc = 0.f, turns = 0.f;
  if (walk_step_f(w, o, p0x, p0y, p0z, f1, f0.w, ex, ey, ez, ee, acc, turns))
    return kInvTwoPi * (double)acc + (double)turns;
  return seg_term_fp64(xyz, a0, a1, b0, b1);
}

// Exact leaf-leaf term of the traversal schedules 1 and 2.
__device__ void leaf_eval(const double *xyz, const NodeHdr &h1, const NodeHdr &h2, const NodeMom &, const NodeMom &,
                          int64_t o1, int64_t n1, int64_t o2, int64_t n2, double &sum) {
  sum += seg_pair_term(xyz, o1, n1, -1 - h1.left, o2, n2, -1 - h2.left);
}

#ifndef FLN_BUCKET_MIN_CTAS
#define FLN_BUCKET_MIN_CTAS 6
#endif
__global__ void __launch_bounds__(32 * kBkWarps, FLN_BUCKET_MIN_CTAS) bh_buckets(BucketArgs A) {
  __shared__ float4 s_q[kBkWarps][kStageV];   // staged loop-2 vertices (x, y, z relative to o_j; |segment|^2)
  __shared__ double s_org[kBkWarps][3][32];   // per entry origin o_j (FP64)
  __shared__ int2 s_near[kBkWarps][64];       // (segment of loop 1, segment of loop 2) left to FP64
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  float4 *sq = s_q[wi];
  double(*org)[32] = s_org[wi];
  int2 *nq = s_near[wi];
  const int64_t nw = (int64_t)gridDim.x * kBkWarps;
  const int64_t n = min((int64_t)*A.count, A.cap);
  const unsigned lt = (1u << lane) - 1;
  double nexact = 0;
  for (int64_t c = (int64_t)blockIdx.x * kBkWarps + wi; c < n; c += nw) {
    const int slot = A.chunks[c].slot, cnt = A.chunks[c].count;
    const int l1 = A.slot_loops[2 * slot], l2 = A.slot_loops[2 * slot + 1];
    const int64_t o1 = A.off[l1], n1 = A.off[l1 + 1] - o1, o2 = A.off[l2], n2 = A.off[l2 + 1] - o2;
    const double *P1 = A.xyz + 3 * o1, *Q2 = A.xyz + 3 * o2;
    int4 e = make_int4(0, 0, 0, 0);
    if (lane < cnt) e = A.chunks[c].e[lane];
    nexact += (double)__reduce_add_sync(0xffffffffu, (unsigned)(e.z * e.w));
    // All entries fit the staging area unless bh_bucket > 8 makes them
    // longer; then the chunk goes in two halves of 16 entries.
    const int tot = __reduce_add_sync(0xffffffffu, lane < cnt ? e.w + 1 : 0);
    const int halves = tot > kStageV ? 2 : 1;
    double sum = 0.0;
    int nn = 0;  // queued FP64 pairs
    for (int h = 0; h < halves; ++h) {
      const bool mine = lane < cnt && (halves == 1 || (lane >> 4) == h);
      // Staging: lane j writes entry j's origin and loop-2 vertices.
      const int nv = mine ? e.w + 1 : 0;
      int vb = nv;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, vb, o);
        if (lane >= o) vb += y;
      }
      vb -= nv;
      if (mine) {
        double p[3], q[3];
        load3(P1, e.x, p);
        load3(Q2, e.y, q);
        const double ox = 0.5 * p[0] + 0.5 * q[0], oy = 0.5 * p[1] + 0.5 * q[1], oz = 0.5 * p[2] + 0.5 * q[2];
        org[0][lane] = ox;
        org[1][lane] = oy;
        org[2][lane] = oz;
        float4 prev = make_float4((float)(q[0] - ox), (float)(q[1] - oy), (float)(q[2] - oz), 0.f);
        for (int r = 1; r <= e.w; ++r) {
          const int t = e.y + r;
          load3(Q2, t >= n2 ? t - n2 : t, q);
          const float4 cur = make_float4((float)(q[0] - ox), (float)(q[1] - oy), (float)(q[2] - oz), 0.f);
          const float fx = cur.x - prev.x, fy = cur.y - prev.y, fz = cur.z - prev.z;
          prev.w = dot3(fx, fy, fz, fx, fy, fz);
          sq[vb + r - 1] = prev;
          prev = cur;
        }
        sq[vb + e.w] = prev;
      }
      // Rows in order of their length: rank the entries by cnt2 (counting
      // sort by ballots), then number the rows of the sorted entries.
      const int key = mine ? e.w : 0;
      int rank = 0, before = 0;
      for (int k = 1; k <= 16; ++k) {
        const unsigned m = __ballot_sync(0xffffffffu, key == k);
        if (key == k) rank = before + __popc(m & lt);
        before += __popc(m);
      }
      // Sorted position -> entry, and the row prefix in sorted order.
      __shared__ int s_perm[kBkWarps][32];
      if (mine) s_perm[wi][rank] = lane;
      __syncwarp();
      const int nact = before;  // active entries
      const int pj = lane < nact ? s_perm[wi][lane] : 0;
      // (Every lane takes part in the shuffle; the rows of lanes past nact
      // are dropped after it.)
      const int rows_pj = __shfl_sync(0xffffffffu, e.z, pj);
      const int rows_s = lane < nact ? rows_pj : 0;
      int rpre = rows_s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, rpre, o);
        if (lane >= o) rpre += y;
      }
      const int nrows = __shfl_sync(0xffffffffu, rpre, 31);
      rpre -= rows_s;  // exclusive
      for (int base = 0; base < nrows; base += 32) {
        const int g = base + lane;
        // the last sorted entry whose rows start at or before row g
        int i = 0;
#pragma unroll
        for (int st = 16; st; st >>= 1) {
          const int x = __shfl_sync(0xffffffffu, rpre, i + st);
          if (i + st < nact && x <= g) i += st;
        }
        const int j = __shfl_sync(0xffffffffu, pj, i);
        const int u = g - __shfl_sync(0xffffffffu, rpre, i);
        const int lo1 = __shfl_sync(0xffffffffu, e.x, j), lo2 = __shfl_sync(0xffffffffu, e.y, j);
        const int c2 = __shfl_sync(0xffffffffu, e.w, j), vbj = __shfl_sync(0xffffffffu, vb, j);
        const bool act = g < nrows;
        uint32_t nearmask = 0;  // steps of this lane's row left to FP64
        int s1 = 0;
        if (act) {
          s1 = lo1 + u;
          if (s1 >= n1) s1 -= (int)n1;
          const int s1n = s1 + 1 == n1 ? 0 : s1 + 1;
          double p0[3], p1[3];
          load3(P1, s1, p0);
          load3(P1, s1n, p1);
          const double ox = org[0][j], oy = org[1][j], oz = org[2][j];
          const float p0x = (float)(p0[0] - ox), p0y = (float)(p0[1] - oy), p0z = (float)(p0[2] - oz);
          const float ex = (float)(p1[0] - p0[0]), ey = (float)(p1[1] - p0[1]), ez = (float)(p1[2] - p0[2]);
          const float ee = dot3(ex, ey, ez, ex, ey, ez);
          const float4 q0 = sq[vbj];
          SegWalkF wa = walk_start_f(p0x, p0y, p0z, q0, ex, ey, ez), wb;
          float ff = q0.w, acc = 0.f, turns = 0.f;
          // Two steps per pass, the state going wa -> wb -> wa. Rows are
          // sorted, so the lanes of a warp mostly walk equally far.
          int k = 0;
          for (; k + 2 <= c2; k += 2) {
            const float4 q1 = sq[vbj + k + 1], q2 = sq[vbj + k + 2];
            if (!walk_step_f(wa, wb, p0x, p0y, p0z, q1, ff, ex, ey, ez, ee, acc, turns)) nearmask |= 1u << k;
            if (!walk_step_f(wb, wa, p0x, p0y, p0z, q2, q1.w, ex, ey, ez, ee, acc, turns)) nearmask |= 2u << k;
            ff = q2.w;
          }
          if (k < c2) {
            const float4 q1 = sq[vbj + k + 1];
            if (!walk_step_f(wa, wb, p0x, p0y, p0z, q1, ff, ex, ey, ez, ee, acc, turns)) nearmask |= 1u << k;
          }
          sum += kInvTwoPi * (double)acc + (double)turns;
        }
        // Queue this pass's FP64 pairs, one per lane per round; evaluate 32 at a time.
        while (__any_sync(0xffffffffu, nearmask != 0)) {
          const bool has = nearmask != 0;
          const unsigned bm = __ballot_sync(0xffffffffu, has);
          if (has) {
            const int k = __ffs(nearmask) - 1;
            nearmask &= nearmask - 1;
            int s2 = lo2 + k;
            if (s2 >= n2) s2 -= (int)n2;
            nq[nn + __popc(bm & lt)] = make_int2(s1, s2);
          }
          nn += __popc(bm);
          __syncwarp();
          if (nn >= 32) {
            const int2 q = nq[nn - 32 + lane];
            sum += seg_term_fp64(A.xyz, o1 + q.x, o1 + (q.x + 1 == n1 ? 0 : q.x + 1), o2 + q.y,
                                 o2 + (q.y + 1 == n2 ? 0 : q.y + 1));
            nn -= 32;
            __syncwarp();
          }
        }
      }
      __syncwarp();
    }
    if (lane < nn) {
      const int2 q = nq[lane];
      sum += seg_term_fp64(A.xyz, o1 + q.x, o1 + (q.x + 1 == n1 ? 0 : q.x + 1), o2 + q.y,
                           o2 + (q.y + 1 == n2 ? 0 : q.y + 1));
    }
    __syncwarp();
#pragma unroll
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) fix_add(A.acc_lk + slot, sum);
  }
  if (lane == 0 && nexact > 0) atomicAdd(A.counts + 1, nexact);
}

// The traversal kernels at N CTAs per SM (fln_params.bh_occupancy): 5 (96
// registers), 6 (80) or 7 (72, with some spills). The traversal is bound by
// dependent loads, so more resident warps can pay for the spills. (Without a
// minimum CTA count ptxas assumes one and took up to 138 registers.)
//   bh_traverse_oN        plain
//   bh_traverse_front_oN  the first pass, which records its frontier
//   bh_traverse_cont_oN   the beta retry continued from that frontier
#define FLN_TRAVERSE_KERNELS(N)                                                                              \
  __global__ void __launch_bounds__(32 * kWarps, N) bh_traverse_o##N(TravArgs A) { traverse<false, false, 0>(A); } \
  __global__ void __launch_bounds__(32 * kWarps, N) bh_traverse_front_o##N(TravArgs A) {                     \
    traverse<false, false, 1>(A);                                                                            \
  }                                                                                                          \
  __global__ void __launch_bounds__(32 * kWarps, N) bh_traverse_cont_o##N(TravArgs A) {                      \
    traverse<false, false, 2>(A);                                                                            \
  }
FLN_TRAVERSE_KERNELS(5)
FLN_TRAVERSE_KERNELS(6)
FLN_TRAVERSE_KERNELS(7)

// Internal nodes per height of the curve-order tree of an n-segment loop,
// added to hcnt[64]: the split of curve_tree_topology ([lo, hi) -> [lo, mid),
// [mid, hi), mid = lo + (hi - lo) / 2; a node of m >= 2 segments has height
// ceil(log2 m)). The ranges of one depth have at most two sizes, so this takes
// O(log n) steps. The host sizes the height launches from it without reading
// the device's counts back first; the device's counts are checked against it
// after the build.
void curve_height_counts(int64_t n, int64_t *hcnt) {
  std::vector<std::pair<int64_t, int64_t>> cur{{n, 1}}, next;
  while (!cur.empty()) {
    next.clear();
    for (const auto &mc : cur) {
      const int64_t m = mc.first, c = mc.second;
      if (m < 2) continue;
      hcnt[64 - __builtin_clzll((unsigned long long)(m - 1))] += c;
      for (const int64_t sz : {m / 2, m - m / 2}) {
        bool merged = false;
        for (auto &x : next)
          if (x.first == sz) {
            x.second += c;
            merged = true;
          }
        if (!merged) next.push_back({sz, c});
      }
    }
    cur.swap(next);
  }
}

struct TraverseSet {
  void (*plain)(TravArgs), (*front)(TravArgs), (*cont)(TravArgs);
  int ctas;       // CTAs per SM the set is built for
  int carveout;   // shared-memory carveout (percent) that fits that many CTAs of 16 KB
};
const TraverseSet kTraverseSets[] = {{bh_traverse_o5, bh_traverse_front_o5, bh_traverse_cont_o5, 5, FLN_BH_CARVEOUT},
                                     {bh_traverse_o6, bh_traverse_front_o6, bh_traverse_cont_o6, 6, FLN_BH_CARVEOUT_6},
                                     {bh_traverse_o7, bh_traverse_front_o7, bh_traverse_cont_o7, 7, 58}};
__global__ void __launch_bounds__(32 * kWarps) bh_traverse_record(TravArgs A) { traverse<false, true, 0>(A); }
// The learned kernels at FLN_LEARNED_MIN_CTAS CTAs per SM: their MLP code
// (BF16 warp MMA) takes 168 registers at three CTAs; held to five, the
// traversal keeps the plain kernel's occupancy and the inference, which runs
// only for some warp steps, spills.
#ifndef FLN_LEARNED_MIN_CTAS
#define FLN_LEARNED_MIN_CTAS 5
#endif
__global__ void __launch_bounds__(32 * kWarps, FLN_LEARNED_MIN_CTAS) bh_traverse_learned(TravArgs A) {
  traverse<true, false, 0>(A);
}
__global__ void __launch_bounds__(32 * kWarps, FLN_LEARNED_MIN_CTAS) bh_traverse_learned_front(TravArgs A) {
  traverse<true, false, 1>(A);
}
__global__ void __launch_bounds__(32 * kWarps, FLN_LEARNED_MIN_CTAS) bh_traverse_learned_cont(TravArgs A) {
  traverse<true, false, 2>(A);
}

// ------------------------------------------------------------------ split evaluation
// Rounds with the evaluation taken out of the traversal: bh_classify walks
// the trees and writes far-field and leaf node pairs as chunks of up to 32
// (one loop pair per chunk); bh_far_chunks and bh_leaf_chunks evaluate them.
// The traversal then needs few registers (more warps per SM to cover its
// dependent loads) and the evaluation runs as streaming kernels with full
// warps and one fixed-point atomic per chunk.
struct Chunk {
  int32_t slot;
  int32_t count;
  int2 pairs[32];
};

struct ClassifyArgs {
  const int64_t *off;
  const int64_t *node_base;
  const NodeHdr *hdr;
  const int32_t *slot_loops;
  const double *itolsq;
  double epssq;
  const Batch *in;
  int64_t nin;
  Batch *out;
  int64_t out_cap;
  unsigned long long *out_count;
  int32_t budget;
  Chunk *far_chunks, *leaf_chunks;
  unsigned long long *far_count, *leaf_count;  // chunks written
  int64_t chunk_soft, chunk_cap;                // stop taking batches past soft; hard capacity
  int2 *spill;
  unsigned long long *queue;
  int32_t *status;                              // bit 0 stack overflow, bit 2 chunk capacity
};

__device__ __forceinline__ void flush_chunk(Chunk *list, unsigned long long *count, int64_t cap, int slot,
                                            const int2 *q, int n, int lane, int32_t *status) {
  unsigned long long c = 0;
  if (lane == 0) c = atomicAdd(count, 1ULL);
  c = __shfl_sync(0xffffffffu, c, 0);
  if ((int64_t)c >= cap) {
    if (lane == 0) atomicOr(status, 4);
    return;
  }
  if (lane < n) list[c].pairs[lane] = q[lane];
  if (lane == 0) {
    list[c].slot = slot;
    list[c].count = n;
  }
}

__global__ void __launch_bounds__(32 * kWarps) bh_classify(ClassifyArgs A) {
  __shared__ int2 s_stack[kWarps][kStack];
  __shared__ int2 s_far[kWarps][64];
  __shared__ int2 s_leaf[kWarps][64];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int gw = blockIdx.x * kWarps + w;
  int2 *stack = s_stack[w];
  int2 *farq = s_far[w];
  int2 *leafq = s_leaf[w];
  int2 *spill = A.spill + (size_t)gw * kSpill;
  for (;;) {
    long long b = 0;
    if (lane == 0) {
      // Past the soft limit this round takes no new batch (they carry over).
      const bool full = (int64_t)*(volatile unsigned long long *)A.far_count > A.chunk_soft ||
                        (int64_t)*(volatile unsigned long long *)A.leaf_count > A.chunk_soft;
      b = full ? A.nin : (long long)atomicAdd(A.queue, 1ULL);
    }
    b = __shfl_sync(0xffffffffu, b, 0);
    if (b >= A.nin) break;
    const int slot = A.in[b].slot;
    const int cnt0 = A.in[b].count;
    const int l1 = A.slot_loops[2 * slot], l2 = A.slot_loops[2 * slot + 1];
    const NodeHdr *H1 = A.hdr + A.node_base[l1], *H2 = A.hdr + A.node_base[l2];
    const double itolsq = A.itolsq[slot], eps = A.epssq;
    if (lane < cnt0) stack[lane] = A.in[b].pairs[lane];
    int top = cnt0, nspill = 0, nf = 0, nl = 0, steps = 0;
    bool overflow = false;
    __syncwarp();
    while (true) {
      if (top == 0 && nspill > 0) {
        const int k = min(nspill, kStack / 2);
        for (int x = lane; x < k; x += 32) stack[x] = spill[nspill - k + x];
        nspill -= k;
        top = k;
        __syncwarp();
      }
      if (top == 0) break;
      if (steps >= A.budget) {
        const int total = top + nspill;
        const int nb = (total + 31) / 32;
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(A.out_count, (unsigned long long)nb);
        at = __shfl_sync(0xffffffffu, at, 0);
        if ((long long)(at + nb) <= A.out_cap) {
          for (int q = 0; q < nb; ++q) {
            const int e = 32 * q + lane;
            if (e < total) A.out[at + q].pairs[lane] = e < nspill ? spill[e] : stack[e - nspill];
            if (lane == 0) {
              A.out[at + q].slot = slot;
              A.out[at + q].count = min(32, total - 32 * q);
            }
          }
          top = 0;
          nspill = 0;
          __syncwarp();
          break;
        }
        if (lane == 0)
          for (int q = 0; q < nb && (long long)(at + q) < A.out_cap; ++q) {
            A.out[at + q].slot = slot;
            A.out[at + q].count = 0;
          }
        steps = INT_MIN;
      }
      ++steps;
      const int cnt = min(top, 32);
      const bool act = lane < cnt;
      int2 pr = make_int2(0, 0);
      if (act) pr = stack[top - cnt + lane];
      __syncwarp();
      top -= cnt;
      int kind = 0;
      int2 c0 = make_int2(0, 0), c1 = make_int2(0, 0);
      if (act) {
        const NodeHdr h1 = load_hdr(H1 + pr.x), h2 = load_hdr(H2 + pr.y);
        const double dx = h2.m[0] - h1.m[0], dy = h2.m[1] - h1.m[1], dz = h2.m[2] - h1.m[2];
        const bool leaf1 = h1.left < 0, leaf2 = h2.left < 0;
        const double rs = h1.r + h2.r;
        if (leaf1 && leaf2) {
          kind = 1;
        } else if (dx * dx + dy * dy + dz * dz + eps > rs * rs * itolsq + eps) {
          kind = 2;
        } else {
          kind = 3;
          const bool split2 = (!leaf1 && !leaf2) ? (h2.rsq > h1.rsq) : !leaf2;
          if (split2) {
            c0 = make_int2(pr.x, h2.left);
            c1 = make_int2(pr.x, h2.right);
          } else {
            c0 = make_int2(h1.left, pr.y);
            c1 = make_int2(h1.right, pr.y);
          }
        }
      }
      const unsigned sm = __ballot_sync(0xffffffffu, kind == 3);
      const int ns = __popc(sm);
      if (top + 2 * ns > kStack) {
        const int k = top / 2;
        if (nspill + k > kSpill) {
          overflow = true;
          break;
        }
        for (int x = lane; x < k; x += 32) spill[nspill + x] = stack[x];
        __syncwarp();
        shift_down(stack, k, top - k, lane);
        nspill += k;
        top -= k;
        __syncwarp();
      }
      if (kind == 3) {
        const int rank = __popc(sm & ((1u << lane) - 1));
        stack[top + 2 * rank] = c0;
        stack[top + 2 * rank + 1] = c1;
      }
      top += 2 * ns;
      const unsigned fm = __ballot_sync(0xffffffffu, kind == 2);
      const unsigned lm = __ballot_sync(0xffffffffu, kind == 1);
      if (kind == 2) farq[nf + __popc(fm & ((1u << lane) - 1))] = pr;
      if (kind == 1) leafq[nl + __popc(lm & ((1u << lane) - 1))] = pr;
      nf += __popc(fm);
      nl += __popc(lm);
      __syncwarp();
      if (nf >= 32) {
        flush_chunk(A.far_chunks, A.far_count, A.chunk_cap, slot, farq + nf - 32, 32, lane, A.status);
        nf -= 32;
        __syncwarp();
      }
      if (nl >= 32) {
        flush_chunk(A.leaf_chunks, A.leaf_count, A.chunk_cap, slot, leafq + nl - 32, 32, lane, A.status);
        nl -= 32;
        __syncwarp();
      }
    }
    if (nf > 0) flush_chunk(A.far_chunks, A.far_count, A.chunk_cap, slot, farq, nf, lane, A.status);
    if (nl > 0) flush_chunk(A.leaf_chunks, A.leaf_count, A.chunk_cap, slot, leafq, nl, lane, A.status);
    __syncwarp();
    if (overflow && lane == 0) atomicOr(A.status, 1);
  }
}

struct EvalArgs {
  const double *xyz;
  const int64_t *off;
  const int64_t *node_base;
  const NodeHdr *hdr;
  const NodeMom *mom;
  const int32_t *slot_loops;
  double epssq;
  const Chunk *chunks;
  int64_t nchunks;
  unsigned long long *acc_lk, *acc_err;
  double *count;  // evaluations
};

// One warp per chunk of far-field node pairs.
__global__ void __launch_bounds__(256) bh_far_chunks(EvalArgs A) {
  const int lane = threadIdx.x & 31;
  const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (c >= A.nchunks) return;
  const int slot = A.chunks[c].slot, n = A.chunks[c].count;
  const int l1 = A.slot_loops[2 * slot], l2 = A.slot_loops[2 * slot + 1];
  const int64_t b1 = A.node_base[l1], b2 = A.node_base[l2];
  double sum = 0.0, err = 0.0;
  if (lane < n) {
    const int2 q = A.chunks[c].pairs[lane];
    const NodeHdr h1 = load_hdr(A.hdr + b1 + q.x), h2 = load_hdr(A.hdr + b2 + q.y);
    const double dx = h2.m[0] - h1.m[0], dy = h2.m[1] - h1.m[1], dz = h2.m[2] - h1.m[2];
    const float2 w = far_weights(h1, h2);
    far_eval(load_mom(A.mom + b1 + q.x), load_mom(A.mom + b2 + q.y), (float)dx, (float)dy, (float)dz,
             dx * dx + dy * dy + dz * dz + A.epssq, w.x, w.y, sum, err);
  }
  for (int o = 16; o; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    err += __shfl_xor_sync(0xffffffffu, err, o);
  }
  if (lane == 0) {
    fix_add(A.acc_lk + slot, sum);
    fix_add(A.acc_err + slot, err);
    atomicAdd(A.count, (double)n);
  }
}

// One warp per chunk of leaf-leaf segment pairs.
__global__ void __launch_bounds__(256) bh_leaf_chunks(EvalArgs A) {
  const int lane = threadIdx.x & 31;
  const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (c >= A.nchunks) return;
  const int slot = A.chunks[c].slot, n = A.chunks[c].count;
  const int l1 = A.slot_loops[2 * slot], l2 = A.slot_loops[2 * slot + 1];
  const int64_t b1 = A.node_base[l1], b2 = A.node_base[l2];
  const int64_t o1 = A.off[l1], n1 = A.off[l1 + 1] - o1, o2 = A.off[l2], n2 = A.off[l2 + 1] - o2;
  double sum = 0.0;
  if (lane < n) {
    const int2 q = A.chunks[c].pairs[lane];
    leaf_eval(A.xyz, A.hdr[b1 + q.x], A.hdr[b2 + q.y], A.mom[b1 + q.x], A.mom[b2 + q.y], o1, n1, o2, n2, sum);
  }
  for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if (lane == 0) {
    fix_add(A.acc_lk + slot, sum);
    atomicAdd(A.count, (double)n);
  }
}

// Initial batches: the root pair of every slot in `slots`; clears their sums.
// The root pair of each listed slot as a batch; clears the slot's far,
// exact and error sums.
__global__ void root_batches(const int32_t *slots, int64_t n, const int32_t *slot_loops, const int64_t *off,
                             int32_t tree_kind, Batch *out, unsigned long long *acc_lk,
                             unsigned long long *acc_err, unsigned long long *acc_exact) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int s = slots[k];
  const int l1 = slot_loops[2 * s], l2 = slot_loops[2 * s + 1];
  const int64_t n1 = off[l1 + 1] - off[l1], n2 = off[l2 + 1] - off[l2];
  out[k].slot = s;
  out[k].count = 1;
  out[k].pairs[0] = tree_kind == 0 ? make_int2((int)(n1 / 2 - 1), (int)(n2 / 2 - 1))
                                   : make_int2((int)(n1 - 2), (int)(n2 - 2));
  acc_lk[s] = 0;
  acc_err[s] = 0;
  acc_exact[s] = 0;
}

// Fixed-point sums (far-field + exact) -> per caller pair doubles.
__global__ void finish_sums(const unsigned long long *acc_lk, const unsigned long long *acc_err,
                            const unsigned long long *acc_exact, const int32_t *slot_pair, int64_t nslots,
                            double *lk, double *err) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  const int p = slot_pair[s];
  lk[p] = (double)(long long)(acc_lk[s] + acc_exact[s]) / kFix;
  err[p] = (double)(long long)acc_err[s] / kFix;
}

// ------------------------------------------------------------------ persistent traversal
// One launch for the whole Barnes–Hut stage. Warps first take the root pair
// of each loop pair from a counter; later work comes from a ring of batches
// that busy warps fill when other warps are waiting (they hand over the
// older half of their stack). When the last batch of a pass of a loop pair
// finishes, the warp that finished it reads the pair's sums and either
// writes the result or queues the pair's next pass on the device: the
// reference's beta retry (lnc.cpp:165-184), then up to bh_escalations
// doublings of beta while the scaled estimate exceeds bh_err_limit. Every
// wait is bounded; a wait that runs out sets status bit 1 and the host reruns
// the stage with budgeted rounds.
constexpr int kRing = 1 << 16;                 // batches in the ring
// Queue counters on separate 128-byte lines (waiting warps poll kQLeft).
constexpr int kQRoot = 0, kQHead = 16, kQTail = 32, kQLeft = 48, kQWords = 64;
constexpr long long kWaitPolls = 1LL << 21;    // bounded wait (nanosleep backoff to 2 us: a few seconds)

struct PersistArgs {
  const double *xyz;
  const int64_t *off;
  const int64_t *node_base;
  const NodeHdr *hdr;
  const NodeMom *mom;
  const int32_t *slot_loops;   // 2 per slot
  const int32_t *slot_pair;    // slot -> caller pair
  int32_t nslots;
  int32_t tree_kind;
  double epssq, beta0, beta_limit, target_error, err_scale, err_limit;
  int32_t escalations;
  double *slot_itolsq;         // per slot, current pass
  int32_t *slot_pass;          // 0 first, 1 retry, >= 1 escalations
  int32_t *slot_left;          // unfinished batches of the current pass
  unsigned long long *acc_lk, *acc_err;
  Batch *ring;
  unsigned long long *ready;   // per ring entry: index + 1 once written
  unsigned long long *q;       // [kQRoot] root counter, [kQHead] head, [kQTail] tail, [kQLeft] outstanding
  double *lk, *err;            // per caller pair (err scaled)
  int32_t *flags;              // per caller pair
  double *counts;              // [0] far, [1] leaf, [2] retried, [3] escalated
  int2 *spill;
  int32_t *status;
  int32_t spill_cap;           // global spill entries per warp used (<= kSpill)
  long long wait_polls;        // polls before a wait gives up (status bit 1)
};

__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long *p) {
  return *(const volatile unsigned long long *)p;
}

// Publishes batches of slot `slot` built from the first `total` entries of
// (spill[0..nspill) ++ stack[0..top)); warp-wide. The ring slots are
// reserved with a compare-and-swap that refuses while more than half the ring
// is published but unclaimed, so entries are never overwritten before their
// claimant reads them. Returns false (nothing published) when refused.
__device__ bool publish(PersistArgs &A, int slot, int lane, const int2 *spill, const int2 *stack, int nspill,
                        int total) {
  const int nb = (total + 31) / 32;
  unsigned long long t = 0;
  int ok = 0;
  if (lane == 0) {
    for (int tries = 0; tries < 64; ++tries) {
      t = ld_volatile(&A.q[kQTail]);
      const long long unclaimed = (long long)(t + nb) - (long long)ld_volatile(&A.q[kQHead]);
      if (unclaimed > kRing / 2) break;
      if (atomicCAS(&A.q[kQTail], t, t + nb) == t) {
        ok = 1;
        break;
      }
    }
    if (ok) {
      atomicAdd(&A.slot_left[slot], nb);
      atomicAdd(&A.q[kQLeft], (unsigned long long)nb);
    }
  }
  ok = __shfl_sync(0xffffffffu, ok, 0);
  if (!ok) return false;
  t = __shfl_sync(0xffffffffu, t, 0);
  for (int b = 0; b < nb; ++b) {
    Batch &B = A.ring[(t + b) & (kRing - 1)];
    const int e = 32 * b + lane;
    if (e < total) B.pairs[lane] = e < nspill ? spill[e] : stack[e - nspill];
    if (lane == 0) {
      B.slot = slot;
      B.count = min(32, total - 32 * b);
    }
  }
  __threadfence();
  __syncwarp();
  for (int b = lane; b < nb; b += 32) atomicExch(&A.ready[(t + b) & (kRing - 1)], t + b + 1);
  return true;
}

// Called by the warp that finished the last batch of a pass of `slot`.
__device__ void finish_pass(PersistArgs &A, int slot, int lane) {
  if (lane != 0) return;
  __threadfence();
  const double lk = (double)(long long)atomicAdd(&A.acc_lk[slot], 0ULL) / kFix;
  const double e = (double)(long long)atomicAdd(&A.acc_err[slot], 0ULL) / kFix * A.err_scale;
  const int pass = A.slot_pass[slot];
  const double beta = sqrt(A.slot_itolsq[slot]);
  const int p = A.slot_pair[slot];
  const int escalated = pass - ((A.flags[p] & FLN_PAIR_BETA_RETRIED) ? 1 : 0);
  double next = 0.0;
  int flag = 0;
  if (pass == 0) {
    const double tb = fmin(pow(e / A.target_error, 0.25) * A.beta0, A.beta_limit);
    if (tb > A.beta0) {
      next = tb;
      flag = FLN_PAIR_BETA_RETRIED;
    }
  }
  if (next == 0.0 && !(e <= A.err_limit) && escalated < A.escalations && beta < 4.0 * A.beta_limit) {
    next = fmin(2.0 * beta, 4.0 * A.beta_limit);
    flag = FLN_PAIR_BETA_ESCALATED;
  }
  if (next == 0.0) {
    A.lk[p] = lk;
    A.err[p] = e;
    return;
  }
  // Queue the next pass of this pair.
  A.flags[p] |= flag;
  atomicAdd(A.counts + (flag == FLN_PAIR_BETA_RETRIED ? 2 : 3), 1.0);
  A.slot_itolsq[slot] = next * next;
  A.slot_pass[slot] = pass + 1;
  A.acc_lk[slot] = 0;
  A.acc_err[slot] = 0;
  A.slot_left[slot] = 1;
  atomicAdd(&A.q[kQLeft], 1ULL);
  const unsigned long long t = atomicAdd(&A.q[kQTail], 1ULL);
  Batch &B = A.ring[t & (kRing - 1)];
  const int l1 = A.slot_loops[2 * slot], l2 = A.slot_loops[2 * slot + 1];
  const int64_t n1 = A.off[l1 + 1] - A.off[l1], n2 = A.off[l2 + 1] - A.off[l2];
  B.slot = slot;
  B.count = 1;
  B.pairs[0] = A.tree_kind == 0 ? make_int2((int)(n1 / 2 - 1), (int)(n2 / 2 - 1))
                                : make_int2((int)(n1 - 2), (int)(n2 - 2));
  __threadfence();
  atomicExch(&A.ready[t & (kRing - 1)], t + 1);
}

__global__ void __launch_bounds__(32 * kWarps) bh_persistent(PersistArgs A) {
  __shared__ int2 s_stack[kWarps][kStack];
  __shared__ int2 s_far[kWarps][64];
  __shared__ int2 s_leaf[kWarps][64];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int gw = blockIdx.x * kWarps + w;
  const int nwarps = gridDim.x * kWarps;
  int2 *stack = s_stack[w];
  int2 *farq = s_far[w];
  int2 *leafq = s_leaf[w];
  int2 *spill = A.spill + (size_t)gw * kSpill;
  double nfar = 0, nleaf = 0;
  bool quit = false;
  while (!quit) {
    // ---- take a batch: a root, else the next ring entry (bounded wait)
    int slot = -1, cnt0 = 0;
    unsigned long long h = 0;
    bool from_ring = false;
    if (lane == 0) {
      if (ld_volatile(&A.q[kQRoot]) < (unsigned long long)A.nslots) {
        const unsigned long long r = atomicAdd(&A.q[kQRoot], 1ULL);
        if (r < (unsigned long long)A.nslots) slot = (int)r;
      }
      if (slot < 0) {
        from_ring = true;
        h = atomicAdd(&A.q[kQHead], 1ULL);
        unsigned ns = 256;
        long long polls = 0;
        while (true) {
          if (ld_volatile(&A.ready[h & (kRing - 1)]) == h + 1) break;
          if ((polls & 15) == 15 && ld_volatile(&A.q[kQLeft]) == 0) {
            slot = -2;  // all work done
            break;
          }
          if (++polls > A.wait_polls) {
            atomicOr(A.status, 2);
            slot = -2;
            break;
          }
          __nanosleep(ns);
          if (ns < 2048) ns *= 2;
        }
        if (slot != -2) {
          __threadfence();
          slot = __ldcg(&A.ring[h & (kRing - 1)].slot);
          cnt0 = __ldcg(&A.ring[h & (kRing - 1)].count);
        }
      } else {
        cnt0 = 1;
      }
    }
    slot = __shfl_sync(0xffffffffu, slot, 0);
    cnt0 = __shfl_sync(0xffffffffu, cnt0, 0);
    from_ring = __shfl_sync(0xffffffffu, from_ring, 0);
    h = __shfl_sync(0xffffffffu, h, 0);
    if (slot == -2) break;
    const int l1 = A.slot_loops[2 * slot], l2 = A.slot_loops[2 * slot + 1];
    const int64_t o1 = A.off[l1], n1 = A.off[l1 + 1] - o1, o2 = A.off[l2], n2 = A.off[l2 + 1] - o2;
    const NodeHdr *H1 = A.hdr + A.node_base[l1], *H2 = A.hdr + A.node_base[l2];
    const NodeMom *M1 = A.mom + A.node_base[l1], *M2 = A.mom + A.node_base[l2];
    const double itolsq = __ldcg(&A.slot_itolsq[slot]), eps = A.epssq;
    if (from_ring) {
      if (lane < cnt0) {
        const int2 *src = A.ring[h & (kRing - 1)].pairs;
        stack[lane] = make_int2(__ldcg(&src[lane].x), __ldcg(&src[lane].y));
      }
    } else if (lane == 0) {
      stack[0] = A.tree_kind == 0 ? make_int2((int)(n1 / 2 - 1), (int)(n2 / 2 - 1))
                                  : make_int2((int)(n1 - 2), (int)(n2 - 2));
    }
    int top = cnt0, nspill = 0, nf = 0, nl = 0, steps = 0;
    bool overflow = false;
    double sum = 0.0, err = 0.0;
    __syncwarp();
    while (true) {
      if (top == 0 && nspill > 0) {
        const int k = min(nspill, kStack / 2);
        for (int x = lane; x < k; x += 32) stack[x] = spill[nspill - k + x];
        nspill -= k;
        top = k;
        __syncwarp();
      }
      if (top == 0) break;
      // Hand the older half of the stack to waiting warps.
      if ((++steps & 7) == 0 && top + nspill >= 64) {
        long long waiting = 0;
        if (lane == 0) waiting = (long long)(ld_volatile(&A.q[kQHead]) - ld_volatile(&A.q[kQTail]));
        waiting = __shfl_sync(0xffffffffu, waiting, 0);
        if (waiting > 0 && waiting <= nwarps) {
          const int total = top + nspill;
          const long long want = waiting > 8 ? 8 : waiting;
          const int give = min(total / 2, 32 * (int)want);
          if (publish(A, slot, lane, spill, stack, nspill, give)) {
          // Drop the handed-over entries: they were the oldest (spill first).
          // Shifts read a pass of 32 before writing it; earlier passes only
          // wrote below what later passes read.
          const int from_spill = min(give, nspill);
          for (int base = 0; base < nspill - from_spill; base += 32) {
            const int x = base + lane;
            int2 v = make_int2(0, 0);
            if (x < nspill - from_spill) v = spill[from_spill + x];
            __syncwarp();
            if (x < nspill - from_spill) spill[x] = v;
            __syncwarp();
          }
          nspill -= from_spill;
          const int from_stack = give - from_spill;
          for (int base = 0; from_stack > 0 && base < top - from_stack; base += 32) {
            const int x = base + lane;
            int2 v = make_int2(0, 0);
            if (x < top - from_stack) v = stack[from_stack + x];
            __syncwarp();
            if (x < top - from_stack) stack[x] = v;
            __syncwarp();
          }
          top -= from_stack;
          __syncwarp();
          if (top == 0 && nspill == 0) break;
          if (top == 0) continue;
          }
        }
      }
      const int cnt = min(top, 32);
      const bool act = lane < cnt;
      int2 pr = make_int2(0, 0);
      if (act) pr = stack[top - cnt + lane];
      __syncwarp();
      top -= cnt;
      int kind = 0;
      int2 c0 = make_int2(0, 0), c1 = make_int2(0, 0);
      if (act) {
        const NodeHdr h1 = load_hdr(H1 + pr.x), h2 = load_hdr(H2 + pr.y);
        const double dx = h2.m[0] - h1.m[0], dy = h2.m[1] - h1.m[1], dz = h2.m[2] - h1.m[2];
        const bool leaf1 = h1.left < 0, leaf2 = h2.left < 0;
        const double rs = h1.r + h2.r;
        if (leaf1 && leaf2) {
          kind = 1;
        } else if (dx * dx + dy * dy + dz * dz + eps > rs * rs * itolsq + eps) {
          kind = 2;
        } else {
          kind = 3;
          const bool split2 = (!leaf1 && !leaf2) ? (h2.rsq > h1.rsq) : !leaf2;
          if (split2) {
            c0 = make_int2(pr.x, h2.left);
            c1 = make_int2(pr.x, h2.right);
          } else {
            c0 = make_int2(h1.left, pr.y);
            c1 = make_int2(h1.right, pr.y);
          }
        }
      }
      const unsigned sm = __ballot_sync(0xffffffffu, kind == 3);
      const int ns = __popc(sm);
      if (top + 2 * ns > kStack) {
        const int k = top / 2;
        if (nspill + k > A.spill_cap) {
          overflow = true;
          break;
        }
        for (int x = lane; x < k; x += 32) spill[nspill + x] = stack[x];
        __syncwarp();
        shift_down(stack, k, top - k, lane);
        nspill += k;
        top -= k;
        __syncwarp();
      }
      if (kind == 3) {
        const int rank = __popc(sm & ((1u << lane) - 1));
        stack[top + 2 * rank] = c0;
        stack[top + 2 * rank + 1] = c1;
      }
      top += 2 * ns;
      const unsigned fm = __ballot_sync(0xffffffffu, kind == 2);
      const unsigned lm = __ballot_sync(0xffffffffu, kind == 1);
      if (kind == 2) farq[nf + __popc(fm & ((1u << lane) - 1))] = pr;
      if (kind == 1) leafq[nl + __popc(lm & ((1u << lane) - 1))] = pr;
      nf += __popc(fm);
      nl += __popc(lm);
      __syncwarp();
      while (nf >= 32) {
        const int2 q = farq[nf - 32 + lane];
        const NodeHdr h1 = load_hdr(H1 + q.x), h2 = load_hdr(H2 + q.y);
        const double dx = h2.m[0] - h1.m[0], dy = h2.m[1] - h1.m[1], dz = h2.m[2] - h1.m[2];
        const float2 w = far_weights(h1, h2);
        far_eval(load_mom(M1 + q.x), load_mom(M2 + q.y), (float)dx, (float)dy, (float)dz, dx * dx + dy * dy + dz * dz + eps,
                 w.x, w.y, sum, err);
        nfar += 32;
        nf -= 32;
        __syncwarp();
      }
      while (nl >= 32) {
        const int2 q = leafq[nl - 32 + lane];
        leaf_eval(A.xyz, H1[q.x], H2[q.y], M1[q.x], M2[q.y], o1, n1, o2, n2, sum);
        nleaf += 32;
        nl -= 32;
        __syncwarp();
      }
    }
    if (lane < nf) {
      const int2 q = farq[lane];
      const NodeHdr h1 = load_hdr(H1 + q.x), h2 = load_hdr(H2 + q.y);
      const double dx = h2.m[0] - h1.m[0], dy = h2.m[1] - h1.m[1], dz = h2.m[2] - h1.m[2];
      const float2 w = far_weights(h1, h2);
      far_eval(load_mom(M1 + q.x), load_mom(M2 + q.y), (float)dx, (float)dy, (float)dz, dx * dx + dy * dy + dz * dz + eps, w.x,
               w.y, sum, err);
    }
    if (lane < nl) {
      const int2 q = leafq[lane];
      leaf_eval(A.xyz, H1[q.x], H2[q.y], M1[q.x], M2[q.y], o1, n1, o2, n2, sum);
    }
    nfar += nf;
    nleaf += nl;
    __syncwarp();
    if (overflow && lane == 0) atomicOr(A.status, 1);
    for (int o = 16; o; o >>= 1) {
      sum += __shfl_xor_sync(0xffffffffu, sum, o);
      err += __shfl_xor_sync(0xffffffffu, err, o);
    }
    int last = 0;
    if (lane == 0) {
      fix_add(A.acc_lk + slot, sum);
      fix_add(A.acc_err + slot, err);
      __threadfence();
      last = atomicSub(&A.slot_left[slot], 1) == 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) finish_pass(A, slot, lane);
    if (lane == 0) {
      __threadfence();
      atomicAdd(&A.q[kQLeft], ~0ULL);  // -1
    }
    __syncwarp();
  }
  if (lane == 0) {
    atomicAdd(A.counts, nfar);
    atomicAdd(A.counts + 1, nleaf);
  }
}

// Features and multipole value of recorded node pairs (thread per sample).
__global__ void sample_features(const int64_t *node_base, const NodeHdr *hdr, const NodeMom *mom,
                                const int32_t *slot_loops, const int4 *samples, int64_t n, double epssq, float *X,
                                double *approx, float *sep_out, float *est_out, double err_scale) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int4 sm = samples[k];
  const int l1 = slot_loops[2 * sm.x], l2 = slot_loops[2 * sm.x + 1];
  const int64_t b1 = node_base[l1], b2 = node_base[l2];
  const NodeHdr h1 = load_hdr(hdr + b1 + sm.y), h2 = load_hdr(hdr + b2 + sm.z);
  const NodeMom m1 = load_mom(mom + b1 + sm.y), m2 = load_mom(mom + b2 + sm.z);
  const double dx = h2.m[0] - h1.m[0], dy = h2.m[1] - h1.m[1], dz = h2.m[2] - h1.m[2];
  const double dsq = dx * dx + dy * dy + dz * dz + epssq;
  const float sep = (float)(sqrt(dsq) / (h1.r + h2.r));
  float f[kMlpIn];
  mlp_features(sep, (float)h1.r, (float)h2.r, dsq, h1.tn, h2.tn, h1.dn, h2.dn, m1.qn, m2.qn, f);
  for (int i = 0; i < kMlpIn; ++i) X[k * kMlpIn + i] = f[i];
  double v = 0.0, e = 0.0;
  const float2 w = far_weights(h1, h2);
  far_eval(m1, m2, (float)dx, (float)dy, (float)dz, dsq, w.x, w.y, v, e);
  approx[k] = v;
  sep_out[k] = sep;
  est_out[k] = (float)log10(e * err_scale + 1e-30);
}

// Segment range [lo, hi) of local node `node` of the curve-order tree over n
// segments (the topology of curve_tree_topology).
__device__ __forceinline__ void node_range(int64_t n, int32_t node, int64_t &lo, int64_t &hi) {
  if (node >= n - 1) {
    lo = node - (n - 1);
    hi = lo + 1;
    return;
  }
  const int64_t s = node + 1;
  lo = 0;
  hi = n;
  for (int d = 0; d < 64; ++d) {
    const int64_t m = lo + (hi - lo) / 2;
    if (m == s) return;
    if (s < m) hi = m;
    else lo = m;
  }
}

// One CTA per sample: the exact FP64 sum over the two nodes' segment ranges
// (the leaf term seg_term_fp64) and the log10 error of the multipole value.
__global__ void sample_exact(const double *xyz, const int64_t *off, const int32_t *slot_loops, const int4 *samples,
                             const double *approx, int64_t n, int64_t max_terms, float *target, int32_t *valid) {
  const int64_t k = blockIdx.x;
  if (k >= n) return;
  const int4 sm = samples[k];
  const int la = slot_loops[2 * sm.x], lb = slot_loops[2 * sm.x + 1];
  const int64_t oa = off[la], na = off[la + 1] - oa, ob = off[lb], nb = off[lb + 1] - ob;
  int64_t a0, a1, b0, b1;
  node_range(na, sm.y, a0, a1);
  node_range(nb, sm.z, b0, b1);
  if ((a1 - a0) * (b1 - b0) > max_terms) {
    if (threadIdx.x == 0) valid[k] = 0;
    return;
  }
  __shared__ double s_part[32];
  const int64_t nbr = b1 - b0, terms = (a1 - a0) * nbr;
  double acc = 0.0;
  for (int64_t t = threadIdx.x; t < terms; t += blockDim.x) {
    const int64_t i = a0 + t / nbr, j = b0 + t % nbr;
    acc += seg_term_fp64(xyz, oa + i, oa + (i + 1 == na ? 0 : i + 1), ob + j, ob + (j + 1 == nb ? 0 : j + 1));
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_part[w];
    target[k] = (float)log10(fabs(approx[k] - t) + 1e-14);
    valid[k] = 1;
  }
}

__global__ void scatter_kernel(const double *src, const int32_t *idx, int64_t n, double *dst) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) dst[idx[k]] = src[k];
}

// Host kd-median tree (ModifiedKdBVH.h:101-132, :207-237), for bh_tree = 1:
// children in local ids, leaf_seg per leaf position.
void host_kd_tree(const double *xyz, int64_t n, std::vector<int32_t> &children, std::vector<int32_t> &leaf_seg) {
  std::vector<double> lo(3 * n), hi(3 * n), cen(3 * n);
  for (int64_t s = 0; s < n; ++s) {
    const double *p = xyz + 3 * s, *q = xyz + 3 * ((s + 1) % n);
    for (int a = 0; a < 3; ++a) {
      lo[3 * s + a] = std::min(p[a], q[a]);
      hi[3 * s + a] = std::max(p[a], q[a]);
      cen[3 * s + a] = (lo[3 * s + a] + hi[3 * s + a]) / 2.0;
    }
  }
  std::vector<int32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  children.assign(2 * (n - 1), 0);
  int32_t next = 0;
  struct R {
    std::vector<int32_t> &idx, &ch;
    const std::vector<double> &cen;
    int32_t &next;
    int64_t n;
    int32_t go(int64_t from, int64_t to, int dim) {
      auto cmp = [&](int32_t a, int32_t b) { return cen[3 * a + dim] < cen[3 * b + dim]; };
      const int64_t size = to - from;
      int32_t l, r;
      if (size == 2) {
        l = (int32_t)(from + n - 1);
        r = (int32_t)(from + n);
      } else if (size == 3) {
        const int64_t mid = from + 2;
        std::nth_element(idx.begin() + from, idx.begin() + mid, idx.begin() + to, cmp);
        l = go(from, mid, (dim + 1) % 3);
        r = (int32_t)(mid + n - 1);
      } else {
        const int64_t mid = from + size / 2;
        std::nth_element(idx.begin() + from, idx.begin() + mid, idx.begin() + to, cmp);
        l = go(from, mid, (dim + 1) % 3);
        r = go(mid, to, (dim + 1) % 3);
      }
      const int32_t me = next++;
      ch[2 * me] = l;
      ch[2 * me + 1] = r;
      return me;
    }
  } rec{idx, children, cen, next, n};
  rec.go(0, n, 0);
  leaf_seg = idx;
}

__global__ void parents_from_children(const int32_t *children, const int64_t *node_base, const int64_t *off,
                                      const int32_t *loops, int32_t nloops, const int64_t *seg_start,
                                      int64_t total_internal, int32_t *parent, int32_t *arrive) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total_internal) return;
  const int k = find_loop_of(seg_start, nloops, g);
  const int l = loops[k];
  const int64_t base = node_base[l];
  const int32_t node = (int32_t)(g - seg_start[k]);
  const int64_t n = off[l + 1] - off[l];
  parent[base + children[2 * (base + node)]] = node;
  parent[base + children[2 * (base + node) + 1]] = node;
  arrive[base + node] = 0;
  if (node == n - 2) parent[base + node] = -1;
}

}  // namespace

void scatter_doubles(Context &ctx, const double *src, const int32_t *idx, int64_t n, double *dst) {
  if (n <= 0) return;
  scatter_kernel<<<(int)((n + 255) / 256), 256, 0, ctx.stream>>>(src, idx, n, dst);
  FLN_CUDA(cudaGetLastError());
}

int barnes_hut_device(Context &ctx, const double *d_xyz, const int64_t *d_off, const std::vector<int64_t> &h_off,
                      const std::vector<int32_t> &h_pairs, const fln_params &prm, double *d_lk_out,
                      double *d_err_out, int32_t *d_flags_out) {
  const int64_t np = (int64_t)h_pairs.size() / 2;
  if (np == 0) return 0;
  const int nl_all = (int)h_off.size() - 1;
  // Loops that need a tree, their node bases and build index ranges.
  std::vector<char> need(nl_all, 0);
  for (int32_t l : h_pairs) need[l] = 1;
  std::vector<int32_t> loops;
  std::vector<int64_t> node_base(nl_all, 0), seg_int(1, 0), seg_all(1, 0);
  int64_t nodes = 0;
  int maxdepth = 0;
  for (int l = 0; l < nl_all; ++l) {
    if (!need[l]) continue;
    const int64_t n = h_off[l + 1] - h_off[l];
    loops.push_back(l);
    node_base[l] = nodes;
    nodes += 2 * n - 1;
    seg_int.push_back(seg_int.back() + (n - 1));
    seg_all.push_back(seg_all.back() + n);
    int d = 0;
    while ((int64_t(1) << d) < n) ++d;
    maxdepth = std::max(maxdepth, d);
  }
  const int32_t nloops = (int32_t)loops.size();
  const int64_t tot_int = seg_int.back(), tot_leaf = seg_all.back();
  // Device buffers (grow-only).
  int32_t *d_loops = ctx.d_bh[0].as<int32_t>(nloops);
  int64_t *d_base = ctx.d_bh[1].as<int64_t>(nl_all);
  int64_t *d_segint = ctx.d_bh[2].as<int64_t>(nloops + 1);
  int64_t *d_segall = ctx.d_bh[3].as<int64_t>(nloops + 1);
  int32_t *d_children = ctx.d_bh[4].as<int32_t>(2 * nodes);
  int32_t *d_parent = ctx.d_bh[5].as<int32_t>(nodes);
  int32_t *d_leafseg = ctx.d_bh[6].as<int32_t>(nodes);
  int32_t *d_arrive = ctx.d_bh[7].as<int32_t>(nodes);
  BuildNode *d_bn = ctx.d_bh[8].as<BuildNode>(std::max<int64_t>(tot_int, 1));  // internal nodes only
  NodeHdr *d_hdr = ctx.d_bh[9].as<NodeHdr>(nodes);
  NodeMom *d_mom = ctx.d_bh[10].as<NodeMom>(nodes);
  cudaStream_t st = ctx.stream;
  FLN_CUDA(cudaMemcpyAsync(d_loops, loops.data(), nloops * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemcpyAsync(d_base, node_base.data(), nl_all * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemcpyAsync(d_segint, seg_int.data(), (nloops + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemcpyAsync(d_segall, seg_all.data(), (nloops + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  TreeArgs T{d_xyz, d_off, d_base, d_loops, nloops, d_children, d_parent, d_leafseg, d_arrive, d_bn, d_hdr, d_mom,
             d_segint};
  // Slots: pairs ordered by decreasing estimated work. Host work, done once
  // the tree build is queued (while the GPU runs it, before the host waits
  // for its counts).
  std::vector<int32_t> order(np), slot_loops(2 * np);
  bool slots_ordered = false;
  auto order_slots = [&]() {
    std::iota(order.begin(), order.end(), 0);
    std::vector<double> cost(np);
    for (int64_t p = 0; p < np; ++p) {
      const double a = (double)(h_off[h_pairs[2 * p] + 1] - h_off[h_pairs[2 * p]]);
      const double b = (double)(h_off[h_pairs[2 * p + 1] + 1] - h_off[h_pairs[2 * p + 1]]);
      cost[p] = (a + b) * std::log2(a + b + 2.0);
    }
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    for (int64_t s = 0; s < np; ++s) {
      slot_loops[2 * s] = h_pairs[2 * order[s]];
      slot_loops[2 * s + 1] = h_pairs[2 * order[s] + 1];
    }
    slots_ordered = true;
  };
  int launches = 0;
  FLN_CUDA(cudaEventRecord(ctx.ev2, st));
  if (prm.bh_tree == 1) {
    // The reference's kd-median tree, built on the host from a copy of the loops.
    wait_xyz_pieces(ctx);
    std::vector<int32_t> ch_all(2 * nodes, 0), ls_all(nodes, 0);
    std::vector<double> xyz_host(3 * h_off.back());
    FLN_CUDA(cudaMemcpyAsync(xyz_host.data(), d_xyz, xyz_host.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaStreamSynchronize(st));
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < nloops; ++k) {
      const int l = loops[k];
      const int64_t n = h_off[l + 1] - h_off[l];
      std::vector<int32_t> ch, ls;
      host_kd_tree(xyz_host.data() + 3 * h_off[l], n, ch, ls);
      std::copy(ch.begin(), ch.end(), ch_all.begin() + 2 * node_base[l]);
      for (int64_t p = 0; p < n; ++p) ls_all[node_base[l] + n - 1 + p] = ls[p];
    }
    FLN_CUDA(cudaMemcpyAsync(d_children, ch_all.data(), ch_all.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    FLN_CUDA(cudaMemcpyAsync(d_leafseg, ls_all.data(), ls_all.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    parents_from_children<<<(int)((tot_int + 255) / 256), 256, 0, st>>>(d_children, d_base, d_off, d_loops, nloops,
                                                                        d_segint, tot_int, d_parent, d_arrive);
    FLN_CUDA(cudaStreamSynchronize(st));  // host vectors go out of scope
    ++launches;
    build_moments<<<(int)((tot_leaf + 127) / 128), 128, 0, st>>>(T, d_segall, tot_leaf, true);
    FLN_CUDA(cudaGetLastError());
    ++launches;
  } else {
    // Curve-order trees: topology with node heights, leaf records, then one
    // launch per height (no arrival counters, no serial walk-up chains).
    uint8_t *d_height = ctx.d_bh[20].as<uint8_t>(std::max<int64_t>(tot_int, 1));
    // Per group: the device's height counts (checked after the build), then
    // the height offsets and cursors of bucket_heights.
    const int max_groups = std::max(ctx.xyz_pieces, 1);
    int32_t *d_hcnt = ctx.d_bh[18].as<int32_t>((size_t)64 * max_groups + 128);
    int32_t *d_hoff = d_hcnt + 64 * max_groups, *d_hcur = d_hoff + 64;
    int32_t *d_bucket = ctx.d_bh[19].as<int32_t>(std::max<int64_t>(tot_int, 1));
    int2 *d_range = ctx.d_bh[22].as<int2>(std::max<int64_t>(tot_int, 1));
    // The loops in groups: one per piece of the vertices still arriving from
    // the host (each group's build waits only for its piece), else one.
    std::vector<int32_t> group_end;  // loop index (into `loops`) where each group ends
    std::vector<int> group_piece;
    if (ctx.xyz_pieces > 0) {
      int32_t k = 0;
      for (int i = 0; i < ctx.xyz_pieces; ++i) {
        while (k < nloops && h_off[loops[k] + 1] <= ctx.xyz_piece_end[i]) ++k;
        group_end.push_back(k);
        group_piece.push_back(i);
      }
      group_end.back() = nloops;
    } else {
      group_end.push_back(nloops);
      group_piece.push_back(-1);
    }
    FLN_CUDA(cudaMemsetAsync(d_hcnt, 0, (size_t)64 * max_groups * sizeof(int32_t), st));
    std::vector<int64_t> host_counts((size_t)64 * group_end.size(), 0);
    std::vector<int32_t> hoff_all((size_t)64 * group_end.size(), 0);  // lives until the stream has read it
    int32_t k0 = 0;
    for (size_t gi = 0; gi < group_end.size(); ++gi) {
      const int32_t k1 = group_end[gi];
      if (group_piece[gi] >= 0) FLN_CUDA(cudaStreamWaitEvent(st, ctx.ev_piece[group_piece[gi]], 0));
      if (k1 <= k0) continue;
      const int64_t i0 = seg_int[k0], i1 = seg_int[k1], f0 = seg_all[k0], f1 = seg_all[k1];
      int64_t *hc = host_counts.data() + 64 * gi;
      for (int32_t k = k0; k < k1; ++k) curve_height_counts(h_off[loops[k] + 1] - h_off[loops[k]], hc);
      if (i1 > i0)
        curve_tree_topology<<<(int)((i1 - i0 + 255) / 256), 256, 0, st>>>(T, d_segint, i0, i1, d_height,
                                                                          d_hcnt + 64 * gi, d_range);
      build_leaves<<<(int)((f1 - f0 + 255) / 256), 256, 0, st>>>(T, d_segall, f0, f1);
      FLN_CUDA(cudaGetLastError());
      launches += 2;
      int32_t hcnt[64];
      int32_t *hoff = hoff_all.data() + 64 * gi;
      int64_t acc = i0;  // this group's nodes fill bucket[i0, i1)
      for (int h = 0; h < 64; ++h) {
        hcnt[h] = (int32_t)hc[h];
        hoff[h] = (int32_t)acc;
        acc += hc[h];
      }
      if (i1 > i0) {
        FLN_CUDA(cudaMemsetAsync(d_hcur, 0, 64 * sizeof(int32_t), st));
        FLN_CUDA(cudaMemcpyAsync(d_hoff, hoff, 64 * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        bucket_heights<<<(int)((i1 - i0 + 255) / 256), 256, 0, st>>>(d_height, i0, i1, d_hoff, d_hcur, d_bucket);
        ++launches;
        const int64_t nsmall = (int64_t)hoff[kSmallHeight + 1] - hoff[1];  // heights 1..kSmallHeight
        if (nsmall > 0) {
          build_small<<<(int)((nsmall + 127) / 128), 128, 0, st>>>(T, d_segint, d_bucket + hoff[1], nsmall, d_range);
          ++launches;
        }
        for (int h = kSmallHeight + 1; h < 64; ++h) {
          if (!hcnt[h]) continue;
          build_height<<<(hcnt[h] + 127) / 128, 128, 0, st>>>(T, d_segint, d_bucket + hoff[h], hcnt[h]);
          ++launches;
        }
        FLN_CUDA(cudaGetLastError());
      }
      k0 = k1;
    }
    order_slots();
    // The device's height counts against the host's, which sized the launches.
    std::vector<int32_t> dev_counts((size_t)64 * group_end.size());
    FLN_CUDA(cudaMemcpyAsync(dev_counts.data(), d_hcnt, dev_counts.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                             st));
    FLN_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < dev_counts.size(); ++i)
      if (dev_counts[i] != host_counts[i])
        throw Error(FLN_ERR_INTERNAL, "curve-order tree: node heights disagree with their count");
  }
  wait_xyz_pieces(ctx);  // the traversal reads every loop's vertices
  FLN_CUDA(cudaEventRecord(ctx.ev3, st));
  ctx.stats.ms_tree_build = ctx.elapsed(ctx.ev2, ctx.ev3);

  if (!slots_ordered) order_slots();
  int32_t *d_slots = ctx.d_bh[11].as<int32_t>(4 * np);
  int32_t *d_slot_pair = d_slots + 2 * np;
  int32_t *d_active = d_slots + 3 * np;
  double *d_itol = ctx.d_bh[12].as<double>(np);
  double *d_counts = ctx.d_bh[13].as<double>(8);  // far, leaf, retried, escalated, status words
  int32_t *d_status = reinterpret_cast<int32_t *>(d_counts + 2);
  // Per slot, fixed point: far-field sum, error estimate, exact sum.
  unsigned long long *d_acc = ctx.d_bh[15].as<unsigned long long>(3 * np + 16);
  unsigned long long *d_acc_err = d_acc + np;
  unsigned long long *d_acc_exact = d_acc + 2 * np;
  // [0] queue, [1] next-round count, [2] exact (or far) chunks, [3] leaf chunks, [4] frontier records;
  // [8, 12) the copy of [0, 4) for the odd rounds of the fused schedule.
  unsigned long long *d_ctr = d_acc + 3 * np;
  unsigned long long *const d_ctrs[2] = {d_ctr, d_ctr + 8};
  const TraverseSet &TS = kTraverseSets[prm.bh_occupancy == 6 ? 1 : prm.bh_occupancy == 7 ? 2 : 0];
  static const bool round_log = std::getenv("FLN_BH_ROUND_LOG") != nullptr;
  // Carveouts and occupancies are set and queried once per context: driver
  // queries on every call cost host time while the GPU waits.
  const int ts_index = (int)(&TS - kTraverseSets);
  if (ctx.bh_per_sm[ts_index] == 0) {
    int m = 64;
    for (auto k : {TS.plain, TS.front, TS.cont}) {
      FLN_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, TS.carveout));
      int n = 0;
      FLN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, 32 * kWarps, 0));
      m = std::min(m, n);
    }
    ctx.bh_per_sm[ts_index] = std::max(m, 1);
  }
  if (ctx.bh_per_sm_learned == 0) {
    int n = 0;
    FLN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bh_traverse_learned, 32 * kWarps, 0));
    ctx.bh_per_sm_learned = std::max(n, 1);
    FLN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bh_classify, 32 * kWarps, 0));
    ctx.bh_per_sm_classify = std::max(n, 1);
  }
  const int per_sm = ctx.bh_per_sm[ts_index];
  const int grid = ctx.num_sms * per_sm;
  const int grid_f = grid;
  const int64_t nwarps = (int64_t)grid * kWarps;
  const int spill_cap = prm.bh_spill_cap > 0 ? std::min(prm.bh_spill_cap, kSpill) : kSpill;
  const int grid_l = ctx.num_sms * ctx.bh_per_sm_learned;  // <= grid: the learned kernel uses more registers
  const int grid_c = ctx.num_sms * ctx.bh_per_sm_classify;
  const int64_t nwarps_c = (int64_t)grid_c * kWarps;
  int2 *d_spill = ctx.d_bh[14].as<int2>((size_t)std::max(nwarps, nwarps_c) * kSpill);
  // Round buffers: a warp hands on at most (kStack + kSpill) / 32 + 1 batches.
  const int64_t cap = std::max<int64_t>(np, nwarps * ((kStack + kSpill) / 32 + 1));
  Batch *d_batch[2] = {reinterpret_cast<Batch *>(ctx.d_partial.need(2 * cap * sizeof(Batch))), nullptr};
  d_batch[1] = d_batch[0] + cap;
  FLN_CUDA(cudaMemcpyAsync(d_slots, slot_loops.data(), 2 * np * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemcpyAsync(d_slot_pair, order.data(), np * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaMemsetAsync(d_counts, 0, 2 * sizeof(double) + sizeof(int32_t), st));
  FLN_CUDA(cudaMemsetAsync(d_counts + 5, 0, 3 * sizeof(double), st));  // exact entries, reused, subtracted
  const double b0 = prm.barnes_hut_init_beta;
  const int budget = prm.bh_budget > 0 ? prm.bh_budget : FLN_BH_BUDGET;
  // Buckets need contiguous segment ranges: curve-order trees only.
  const int bucket = prm.bh_tree == 1 ? 1 : (prm.bh_bucket > 0 ? prm.bh_bucket : FLN_BH_BUCKET);
  if ((ctx.learned.frag || ctx.recording.rec) && prm.bh_schedule != 0)
    throw Error(FLN_ERR_INVALID_ARGUMENT, "The learned opening criterion runs with bh_schedule 0 only.");
  // Chunk lists of the split evaluation: a warp can write at most budget + 2
  // chunks per list after the soft limit stops new batches.
  const int64_t chunk_soft = int64_t(1) << FLN_CHUNK_SOFT_LOG2;
  const int64_t chunk_cap = chunk_soft + std::max(nwarps, nwarps_c) * (budget + 2);
  Chunk *d_far = nullptr, *d_leaf = nullptr;
  // Exact list of the fused rounds: past the soft limit a round takes no new
  // batch; a warp writes at most budget + 2 chunks after that.
  const int64_t bkt_soft = int64_t(1) << FLN_BUCKET_SOFT_LOG2;
  const int64_t bkt_cap = bkt_soft + nwarps * (budget + 2);
  // Two lists: round r writes list r & 1 while the exact-list kernel of
  // round r - 1 reads the other.
  BucketChunk *d_bkt = nullptr;
  if (prm.bh_schedule == 0)
    d_bkt = reinterpret_cast<BucketChunk *>(ctx.d_bh[21].need((size_t)(2 * bkt_cap) * sizeof(BucketChunk)));
  if (prm.bh_schedule == 2) {
    d_far = reinterpret_cast<Chunk *>(ctx.d_bh[16].need((size_t)chunk_cap * sizeof(Chunk)));
    d_leaf = reinterpret_cast<Chunk *>(ctx.d_bh[17].need((size_t)chunk_cap * sizeof(Chunk)));
  }
  ctx.stats.bh_rounds = 0;
  // Frontier of the first pass (bh_schedule 0): its far node pairs, so that
  // the beta retry continues from them. Sized from the previous call's
  // frontier (grow-only); slots whose records do not fit retry from the roots.
  const bool use_front = prm.bh_schedule == 0 && !prm.bh_retry_from_roots && !ctx.recording.rec;
  FrontRec *d_front = nullptr;
  uint8_t *d_lost = nullptr, *d_skip = nullptr;
  int64_t front_cap = 0;
  if (use_front) {
    const size_t have = ctx.d_bh[23].bytes / sizeof(FrontRec);
    const size_t want_hint = ctx.bh_front_hint > 0 ? (size_t)(1.25 * (double)ctx.bh_front_hint) + 1024 : 0;
    size_t want = have;
    if (want_hint == 0 || want_hint > have) {  // the buffer must grow: ask how much memory is free
      size_t free_b = 0, total_b = 0;
      FLN_CUDA(cudaMemGetInfo(&free_b, &total_b));
      want = want_hint > 0 ? want_hint : std::min<size_t>((size_t)16 << 30, free_b / 5) / sizeof(FrontRec);
      want = std::max(want, have);
      if (want > have && (want - have) * sizeof(FrontRec) > free_b / 2) want = have + free_b / 2 / sizeof(FrontRec);
    }
    front_cap = (int64_t)std::max<size_t>(want, 1024);
    d_front = reinterpret_cast<FrontRec *>(ctx.d_bh[23].need((size_t)front_cap * sizeof(FrontRec)));
    d_lost = ctx.d_bh[25].as<uint8_t>(2 * np);
    d_skip = d_lost + np;
    FLN_CUDA(cudaMemsetAsync(d_lost, 0, np, st));
  }
  int64_t front_n = 0;  // records the first pass wrote (<= front_cap)
  // One Barnes–Hut pass with per-slot beta^2: the root pairs of the slots in
  // `roots`, then (the retry's continuation) the frontier records of the
  // slots whose skip byte is 0. `front` records this pass's frontier.
  auto pass = [&](const std::vector<int32_t> &roots, const std::vector<double> &itol_slots, bool record, bool front,
                  int64_t nstream) {
    const bool cont = nstream > 0;  // the retry continued from the frontier
    const int64_t na = (int64_t)roots.size();
    FLN_CUDA(cudaMemcpyAsync(d_active, roots.data(), na * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    FLN_CUDA(cudaMemcpyAsync(d_itol, itol_slots.data(), np * sizeof(double), cudaMemcpyHostToDevice, st));
    if (na > 0) {
      root_batches<<<(int)((na + 255) / 256), 256, 0, st>>>(d_active, na, d_slots, d_off, prm.bh_tree == 1 ? 1 : 0,
                                                            d_batch[0], d_acc, d_acc_err, d_acc_exact);
      FLN_CUDA(cudaGetLastError());
      ++launches;
    }
    if (front) FLN_CUDA(cudaMemsetAsync(d_ctr + 4, 0, sizeof(unsigned long long), st));
    int64_t nin = na, pos = 0;
    int cur = 0;
    // Fused rounds: round r's exact-list kernel runs on the exact stream
    // beside round r + 1's traversal. Round r fills list and counters r & 1;
    // before it clears them it waits for the exact-list kernel of round r - 2
    // (which read them). Per round four events: the traversal's end (on st),
    // the exact-list kernel's start and end (on the exact stream), the
    // traversal's start (on st).
    bool pend[2] = {false, false};
    cudaEvent_t done[2] = {nullptr, nullptr};
    int nev = 0;
    auto event_at = [&](int x) {
      while ((int)ctx.ev_round.size() <= x) {
        cudaEvent_t e = nullptr;
        FLN_CUDA(cudaEventCreate(&e));
        ctx.ev_round.push_back(e);
      }
      return ctx.ev_round[x];
    };
    // The context's stream waits for every exact-list launch of the pass
    // (also when the pass throws, so that later work stays ordered).
    auto join = [&]() {
      if (nev == 0) return;
      cudaEvent_t e = event_at(4 * nev);
      FLN_CUDA(cudaEventRecord(e, ctx.exact_stream));
      FLN_CUDA(cudaStreamWaitEvent(st, e, 0));
    };
    if (prm.bh_schedule != 2 && !ctx.exact_stream)
      FLN_CUDA(cudaStreamCreateWithFlags(&ctx.exact_stream, cudaStreamNonBlocking));
    try {
      for (int round = 0; (nin > 0 || pos < nstream) && round < 65536; ++round) {
        const int par = round & 1;
        if (prm.bh_schedule != 2 && pend[par]) FLN_CUDA(cudaStreamWaitEvent(st, done[par], 0));
        FLN_CUDA(cudaMemsetAsync(prm.bh_schedule == 2 ? d_ctr : d_ctrs[par], 0, 4 * sizeof(unsigned long long), st));
        if (prm.bh_schedule == 2) {
          // Classify, then evaluate this round's chunks.
          ClassifyArgs C{d_off, d_base, d_hdr, d_slots, d_itol, prm.epssq, d_batch[cur], nin, d_batch[1 - cur], cap,
                         d_ctr + 1, budget, d_far, d_leaf, d_ctr + 2, d_ctr + 3, chunk_soft, chunk_cap, d_spill,
                         d_ctr, d_status};
          const int g = (int)std::max<int64_t>(1, std::min<int64_t>((nin + kWarps - 1) / kWarps, grid_c));
          bh_classify<<<g, 32 * kWarps, 0, st>>>(C);
          FLN_CUDA(cudaGetLastError());
          unsigned long long c4[4];
          FLN_CUDA(cudaMemcpyAsync(c4, d_ctr, sizeof c4, cudaMemcpyDeviceToHost, st));
          FLN_CUDA(cudaStreamSynchronize(st));
          const int64_t nfar = (int64_t)std::min<unsigned long long>(c4[2], (unsigned long long)chunk_cap);
          const int64_t nleaf = (int64_t)std::min<unsigned long long>(c4[3], (unsigned long long)chunk_cap);
          EvalArgs E{d_xyz, d_off, d_base, d_hdr, d_mom, d_slots, prm.epssq, d_far, nfar, d_acc, d_acc_err, d_counts};
          if (nfar > 0) bh_far_chunks<<<(int)((nfar * 32 + 255) / 256), 256, 0, st>>>(E);
          E.chunks = d_leaf;
          E.nchunks = nleaf;
          E.count = d_counts + 1;
          if (nleaf > 0) bh_leaf_chunks<<<(int)((nleaf * 32 + 255) / 256), 256, 0, st>>>(E);
          FLN_CUDA(cudaGetLastError());
          launches += 3;
          ++ctx.stats.bh_rounds;
          // Batches not taken this round (past the chunk soft limit) carry over.
          int64_t next = (int64_t)std::min<unsigned long long>(c4[1], (unsigned long long)cap);
          const int64_t taken = (int64_t)std::min<unsigned long long>(c4[0], (unsigned long long)nin);
          if (taken < nin) {
            const int64_t keep = std::min<int64_t>(nin - taken, cap - next);
            FLN_CUDA(cudaMemcpyAsync(d_batch[1 - cur] + next, d_batch[cur] + taken, keep * sizeof(Batch),
                                     cudaMemcpyDeviceToDevice, st));
            if (keep < nin - taken) throw Error(FLN_ERR_INTERNAL, "Barnes-Hut round buffer too small");
            next += keep;
          }
          nin = next;
          cur = 1 - cur;
          continue;
        }
        if (!d_bkt) throw Error(FLN_ERR_INTERNAL, "Barnes-Hut rounds without an exact list");
        unsigned long long *const c = d_ctrs[par];
        BucketChunk *const bl = d_bkt + par * bkt_cap;
        TravArgs A{d_xyz, d_off, d_base, d_hdr, d_mom, d_slots, d_itol, prm.epssq, d_batch[cur], nin,
                   d_batch[1 - cur], cap, c + 1, budget, bucket, bl, c + 2, bkt_soft, bkt_cap, d_acc,
                   d_acc_err, d_counts, d_spill, c, d_status,
                   d_front + pos, nstream - pos, d_skip,
                   front ? d_front : nullptr, d_ctr + 4, front_cap, d_lost, spill_cap,
                   ctx.learned, b0, nullptr, nullptr, 0, 0.f, 0u};
        if (record) {
          A.rec = ctx.recording.rec;
          A.rec_count = ctx.recording.count;
          A.rec_cap = ctx.recording.cap;
          A.rec_smin = ctx.recording.s_min;
          A.rec_keep = ctx.recording.keep;
        }
        const int gmax = (A.learned.frag && !A.rec) ? grid_l : (front ? grid_f : grid);
        const int64_t work = nin + (nstream - pos);
        const int g = (int)std::max<int64_t>(1, std::min<int64_t>((work + kWarps - 1) / kWarps, gmax));
        FLN_CUDA(cudaEventRecord(event_at(4 * nev + 3), st));
        if (A.rec)
          bh_traverse_record<<<g, 32 * kWarps, 0, st>>>(A);
        else if (A.learned.frag)
          (front ? bh_traverse_learned_front : cont ? bh_traverse_learned_cont : bh_traverse_learned)
              <<<g, 32 * kWarps, 0, st>>>(A);
        else
          (front ? TS.front : cont ? TS.cont : TS.plain)<<<g, 32 * kWarps, 0, st>>>(A);
        FLN_CUDA(cudaGetLastError());
        BucketArgs BA{d_xyz, d_off, d_slots, bl, c + 2, bkt_cap, d_acc_exact, d_counts};
        {
          // bh_exact_serial: on the context's stream, after its traversal.
          cudaStream_t xs = prm.bh_exact_serial ? st : ctx.exact_stream;
          cudaEvent_t et = event_at(4 * nev), e0 = event_at(4 * nev + 1), e1 = event_at(4 * nev + 2);
          FLN_CUDA(cudaEventRecord(et, st));
          FLN_CUDA(cudaStreamWaitEvent(xs, et, 0));
          FLN_CUDA(cudaEventRecord(e0, xs));
          bh_buckets<<<ctx.num_sms * 2 * FLN_BUCKET_MIN_CTAS, 32 * kBkWarps, 0, xs>>>(BA);
          FLN_CUDA(cudaGetLastError());
          FLN_CUDA(cudaEventRecord(e1, xs));
          done[par] = e1;
          pend[par] = true;
          ++nev;
        }
        launches += 2;
        ++ctx.stats.bh_rounds;
        unsigned long long c2[2];
        FLN_CUDA(cudaMemcpyAsync(c2, c, sizeof c2, cudaMemcpyDeviceToHost, st));
        FLN_CUDA(cudaStreamSynchronize(st));
        if (round_log) {  // FLN_BH_ROUND_LOG: cumulative counts after each round, for profiling
          FLN_CUDA(cudaStreamSynchronize(ctx.exact_stream));
          double cnt[8];
          FLN_CUDA(cudaMemcpyAsync(cnt, d_counts, sizeof cnt, cudaMemcpyDeviceToHost, st));
          FLN_CUDA(cudaStreamSynchronize(st));
          std::fprintf(stderr,
                       "[fln] round %d (%s): far node pairs %.0f, exact node pairs %.0f, exact segment pairs %.0f\n",
                       ctx.stats.bh_rounds, front ? "first pass" : cont ? "continued retry" : "from roots", cnt[0],
                       cnt[5], cnt[1]);
        }
        // Input not taken this round (past the soft limit) carries over: the
        // batches by copy, the frontier records by position.
        int64_t next = (int64_t)std::min<unsigned long long>(c2[1], (unsigned long long)cap);
        const int64_t taken = (int64_t)std::min<unsigned long long>(c2[0], (unsigned long long)(nin + nstream - pos));
        if (taken < nin) {
          const int64_t keep = std::min<int64_t>(nin - taken, cap - next);
          FLN_CUDA(cudaMemcpyAsync(d_batch[1 - cur] + next, d_batch[cur] + taken, keep * sizeof(Batch),
                                   cudaMemcpyDeviceToDevice, st));
          if (keep < nin - taken) throw Error(FLN_ERR_INTERNAL, "Barnes-Hut round buffer too small");
          next += keep;
        } else {
          pos += taken - nin;
        }
        nin = next;
        cur = 1 - cur;
      }
    } catch (...) {
      join();
      throw;
    }
    join();
    for (int x = 0; x < nev; ++x) {
      ctx.stats.ms_exact += ctx.elapsed(ctx.ev_round[4 * x + 1], ctx.ev_round[4 * x + 2]);
      ctx.stats.ms_traverse += ctx.elapsed(ctx.ev_round[4 * x + 3], ctx.ev_round[4 * x]);
    }
    if (nin > 0 || pos < nstream) throw Error(FLN_ERR_INTERNAL, "Barnes-Hut pass did not finish in 65536 rounds");
    if (front) {
      unsigned long long nrec = 0;
      FLN_CUDA(cudaMemcpyAsync(&nrec, d_ctr + 4, sizeof nrec, cudaMemcpyDeviceToHost, st));
      FLN_CUDA(cudaStreamSynchronize(st));
      front_n = (int64_t)std::min<unsigned long long>(nrec, (unsigned long long)front_cap);
      ctx.bh_front_hint = std::max<int64_t>(ctx.bh_front_hint, (int64_t)nrec);
      ctx.stats.bh_front_records = (int64_t)nrec;
    }
  };
  // bh_schedule = 1: one persistent launch (retry and escalation on the
  // device). The budgeted rounds below are the default and the fallback when
  // a bounded wait of the persistent kernel runs out.
  if (prm.bh_schedule == 1) {
    double *d_sitol = ctx.d_bh[12].as<double>(np);
    int32_t *d_sint = reinterpret_cast<int32_t *>(ctx.d_near.need((size_t)np * 2 * sizeof(int32_t) + 64));
    int32_t *d_pass_arr = d_sint, *d_left = d_sint + np;
    unsigned long long *d_ready = reinterpret_cast<unsigned long long *>(
        ctx.d_items.need((size_t)(kRing + kQWords) * sizeof(unsigned long long)));
    unsigned long long *d_q = d_ready + kRing;
    Batch *d_ring = reinterpret_cast<Batch *>(ctx.d_partial.need((size_t)kRing * sizeof(Batch)));
    int32_t *d_fl = d_flags_out ? d_flags_out : reinterpret_cast<int32_t *>(ctx.d_flags.need(np * sizeof(int32_t)));
    double *d_cnt4 = d_counts;  // [0] far [1] leaf [2] retried [3] escalated [4] status
    d_status = reinterpret_cast<int32_t *>(d_cnt4 + 4);
    std::vector<double> itol0(np, b0 * b0);
    std::vector<int32_t> ones(np, 1);
    unsigned long long q0[kQWords] = {0};
    q0[kQLeft] = (unsigned long long)np;
    FLN_CUDA(cudaMemcpyAsync(d_sitol, itol0.data(), np * sizeof(double), cudaMemcpyHostToDevice, st));
    FLN_CUDA(cudaMemsetAsync(d_pass_arr, 0, np * sizeof(int32_t), st));
    FLN_CUDA(cudaMemcpyAsync(d_left, ones.data(), np * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    FLN_CUDA(cudaMemsetAsync(d_acc, 0, 2 * np * sizeof(unsigned long long), st));
    FLN_CUDA(cudaMemsetAsync(d_ready, 0, kRing * sizeof(unsigned long long), st));
    FLN_CUDA(cudaMemcpyAsync(d_q, q0, sizeof q0, cudaMemcpyHostToDevice, st));
    FLN_CUDA(cudaMemsetAsync(d_fl, 0, np * sizeof(int32_t), st));
    FLN_CUDA(cudaMemsetAsync(d_cnt4, 0, 4 * sizeof(double) + sizeof(int32_t), st));
    PersistArgs P{d_xyz, d_off, d_base, d_hdr, d_mom, d_slots, d_slot_pair, (int32_t)np, prm.bh_tree == 1 ? 1 : 0,
                  prm.epssq, b0, prm.barnes_hut_beta_limit, prm.target_error, prm.error_est_scale,
                  prm.bh_err_limit, prm.bh_escalations, d_sitol, d_pass_arr, d_left, d_acc, d_acc_err, d_ring,
                  d_ready, d_q, d_lk_out, d_err_out, d_fl, d_cnt4, d_spill, d_status, spill_cap,
                  prm.bh_wait_polls > 0 ? (long long)prm.bh_wait_polls : kWaitPolls};
    const int gp = std::min(grid, ctx.num_sms * occupancy_of((const void *)bh_persistent, 32 * kWarps));
    FLN_CUDA(cudaEventRecord(ctx.ev2, st));
    bh_persistent<<<gp, 32 * kWarps, 0, st>>>(P);
    FLN_CUDA(cudaGetLastError());
    FLN_CUDA(cudaEventRecord(ctx.ev3, st));
    ++launches;
    ctx.stats.bh_rounds = 1;
    double cnt[4];
    int32_t pst = 0;
    FLN_CUDA(cudaMemcpyAsync(cnt, d_cnt4, sizeof cnt, cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaMemcpyAsync(&pst, d_status, sizeof pst, cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaStreamSynchronize(st));
    ctx.stats.ms_main_kernel += ctx.elapsed(ctx.ev2, ctx.ev3);
    if (pst & 1)
      throw Error(FLN_ERR_STACK_OVERFLOW, "Barnes-Hut traversal stack exceeded its bound (depth " +
                                              std::to_string(maxdepth) + ").");
    if (!(pst & 2)) {
      ctx.stats.bh_far_evals = cnt[0];
      ctx.stats.bh_leaf_evals = cnt[1];
      ctx.stats.beta_retried = (int64_t)cnt[2];
      ctx.stats.bh_escalated = (int64_t)cnt[3];
      return launches;
    }
    // A bounded wait ran out: redo the stage with budgeted rounds, which
    // need the exact list the persistent schedule does not use.
    ctx.stats.bh_wait_timeouts += 1;
    d_bkt = reinterpret_cast<BucketChunk *>(ctx.d_bh[21].need((size_t)(2 * bkt_cap) * sizeof(BucketChunk)));
    d_status = reinterpret_cast<int32_t *>(d_counts + 2);
    FLN_CUDA(cudaMemsetAsync(d_counts, 0, 2 * sizeof(double) + sizeof(int32_t), st));
    FLN_CUDA(cudaMemsetAsync(d_counts + 5, 0, 3 * sizeof(double), st));
  }
  std::vector<int32_t> all(np);
  std::iota(all.begin(), all.end(), 0);
  std::vector<double> itol(np, b0 * b0);
  FLN_CUDA(cudaEventRecord(ctx.ev2, st));
  pass(all, itol, ctx.recording.rec != nullptr, use_front, 0);
  FLN_CUDA(cudaEventRecord(ctx.ev3, st));
  finish_sums<<<(int)((np + 255) / 256), 256, 0, st>>>(d_acc, d_acc_err, d_acc_exact, d_slot_pair, np, d_lk_out,
                                                       d_err_out);
  FLN_CUDA(cudaGetLastError());
  ++launches;
  // Error estimate and beta retry (lnc.cpp:165-184).
  std::vector<double> err(np);
  FLN_CUDA(cudaMemcpyAsync(err.data(), d_err_out, np * sizeof(double), cudaMemcpyDeviceToHost, st));
  int32_t status = 0;
  FLN_CUDA(cudaMemcpyAsync(&status, d_status, sizeof status, cudaMemcpyDeviceToHost, st));
  std::vector<uint8_t> lost;
  if (use_front) {
    lost.resize(np);
    FLN_CUDA(cudaMemcpyAsync(lost.data(), d_lost, np, cudaMemcpyDeviceToHost, st));
  }
  FLN_CUDA(cudaStreamSynchronize(st));
  ctx.stats.ms_main_kernel += ctx.elapsed(ctx.ev2, ctx.ev3);
  std::vector<int32_t> flags(np, 0), retry_slots;
  std::vector<char> retried(np, 0);
  for (int64_t s = 0; s < np; ++s) {
    const int64_t p = order[s];
    const double e = err[p] * prm.error_est_scale;
    err[p] = e;
    // With a positive target, beta* > beta0 needs e > target: below it
    // (e / target)^(1/4) <= 1 (pow is monotonic and exact at 1), and NaN
    // compares false either way. The test spares the host most pow calls
    // while the GPU waits.
    if (prm.target_error > 0 && !(e > prm.target_error)) continue;
    const double tb = std::min(std::pow(e / prm.target_error, 0.25) * b0, prm.barnes_hut_beta_limit);
    if (tb > b0) {
      retry_slots.push_back((int32_t)s);
      itol[s] = tb * tb;
      flags[p] |= FLN_PAIR_BETA_RETRIED;
      retried[p] = 1;
    }
  }
  ctx.stats.beta_retried = (int64_t)retry_slots.size();
  std::vector<double> far_leaf(8, 0.0);
  if (!retry_slots.empty()) {
    FLN_CUDA(cudaEventRecord(ctx.ev2, st));
    if (use_front && (status & 1) == 0) {
      // A node pair opened at beta0 is opened at beta* > beta0 (far at beta*
      // implies far at beta0), and an exact pair stays exact (the bucket test
      // does not depend on beta). So the beta* pass is the beta0 pass
      // continued from its far node pairs: the slot keeps its sums, the
      // frontier pairs still far keep their values, the ones that open give
      // theirs back (bh_traverse_cont). Slots whose frontier did not fit start
      // from the roots.
      std::vector<uint8_t> skip(np, 1);
      std::vector<int32_t> cont, from_roots;
      for (int32_t sl : retry_slots) {
        if (lost[sl]) {
          from_roots.push_back(sl);
        } else {
          cont.push_back(sl);
          skip[sl] = 0;
        }
      }
      FLN_CUDA(cudaMemcpyAsync(d_skip, skip.data(), np, cudaMemcpyHostToDevice, st));
      ctx.stats.bh_retry_from_roots = (int64_t)from_roots.size();
      pass(from_roots, itol, false, false, cont.empty() ? 0 : front_n);
    } else {
      ctx.stats.bh_retry_from_roots = (int64_t)retry_slots.size();
      pass(retry_slots, itol, false, false, 0);
    }
    FLN_CUDA(cudaEventRecord(ctx.ev3, st));
    finish_sums<<<(int)((np + 255) / 256), 256, 0, st>>>(d_acc, d_acc_err, d_acc_exact, d_slot_pair, np, d_lk_out,
                                                         d_err_out);
    FLN_CUDA(cudaGetLastError());
    ++launches;
    // The reported estimate is that of the final run, scaled like the first
    // (the reference stops using it after the retry; the margin check here
    // needs both on one scale).
    std::vector<double> e2(np);
    FLN_CUDA(cudaMemcpyAsync(e2.data(), d_err_out, np * sizeof(double), cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaMemcpyAsync(&status, d_status, sizeof status, cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaStreamSynchronize(st));
    const double ms = ctx.elapsed(ctx.ev2, ctx.ev3);
    ctx.stats.ms_main_kernel += ms;
    ctx.stats.ms_retry += ms;
    for (int64_t p = 0; p < np; ++p)
      if (retried[p]) err[p] = e2[p] * prm.error_est_scale;
  }
  // Escalation (beyond the reference): a pair whose estimate still exceeds
  // bh_err_limit is re-run with twice its beta, up to bh_escalations times
  // (beta <= 4 x beta_limit); what stays above goes to the FP64 direct sum.
  ctx.stats.bh_escalated = 0;
  for (int esc = 0; esc < prm.bh_escalations; ++esc) {
    std::vector<int32_t> up;
    for (int64_t s = 0; s < np; ++s) {
      const int64_t p = order[s];
      const double beta = std::sqrt(itol[s]);
      if (!(err[p] <= prm.bh_err_limit) && beta < 4.0 * prm.barnes_hut_beta_limit) {
        up.push_back((int32_t)s);
        const double nb = std::min(2.0 * beta, 4.0 * prm.barnes_hut_beta_limit);
        itol[s] = nb * nb;
        flags[p] |= FLN_PAIR_BETA_ESCALATED;
      }
    }
    if (up.empty()) break;
    ctx.stats.bh_escalated += (int64_t)up.size();
    FLN_CUDA(cudaEventRecord(ctx.ev2, st));
    pass(up, itol, false, false, 0);
    FLN_CUDA(cudaEventRecord(ctx.ev3, st));
    finish_sums<<<(int)((np + 255) / 256), 256, 0, st>>>(d_acc, d_acc_err, d_acc_exact, d_slot_pair, np, d_lk_out,
                                                         d_err_out);
    FLN_CUDA(cudaGetLastError());
    ++launches;
    std::vector<double> e3(np);
    FLN_CUDA(cudaMemcpyAsync(e3.data(), d_err_out, np * sizeof(double), cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaMemcpyAsync(&status, d_status, sizeof status, cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaStreamSynchronize(st));
    const double ms = ctx.elapsed(ctx.ev2, ctx.ev3);
    ctx.stats.ms_main_kernel += ms;
    ctx.stats.ms_retry += ms;
    for (int32_t s : up) err[order[s]] = e3[order[s]] * prm.error_est_scale;
  }
  FLN_CUDA(cudaMemcpyAsync(far_leaf.data(), d_counts, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaMemcpyAsync(d_err_out, err.data(), np * sizeof(double), cudaMemcpyHostToDevice, st));
  if (d_flags_out) FLN_CUDA(cudaMemcpyAsync(d_flags_out, flags.data(), np * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  FLN_CUDA(cudaStreamSynchronize(st));
  ctx.stats.bh_far_evals = far_leaf[0];
  ctx.stats.bh_leaf_evals = far_leaf[1];
  ctx.stats.bh_exact_entries = prm.bh_schedule == 0 ? far_leaf[5] : far_leaf[1];
  ctx.stats.bh_far_reused = far_leaf[6];
  ctx.stats.bh_far_subtracted = far_leaf[7];
  if (status & 1)
    throw Error(FLN_ERR_STACK_OVERFLOW, "Barnes-Hut traversal stack exceeded its bound (depth " +
                                            std::to_string(maxdepth) + ").");
  if (status & 16)
    throw Error(FLN_ERR_INTERNAL, "Barnes-Hut moment staging did not complete within its bounded wait.");
  if (status != 0)
    throw Error(FLN_ERR_INTERNAL, "Barnes-Hut work list exceeded its capacity (status " + std::to_string(status) +
                                      ").");
  return launches;
}

void learned_collect(Context &ctx, const double *d_xyz, const int64_t *d_off, const std::vector<int64_t> &h_off,
                     const std::vector<int32_t> &h_pairs, const fln_params &prm, float s_min, double keep,
                     int64_t cap, int64_t max_terms, std::vector<float> &X, std::vector<float> &T,
                     std::vector<float> &S, std::vector<float> &E, int64_t *recorded) {
  X.clear();
  T.clear();
  S.clear();
  E.clear();
  if (recorded) *recorded = 0;
  const int64_t np = (int64_t)h_pairs.size() / 2;
  if (np == 0 || cap <= 0) return;
  cudaStream_t st = ctx.stream;
  int4 *d_rec = ctx.d_learn[0].as<int4>(cap);
  unsigned long long *d_cnt = ctx.d_learn[1].as<unsigned long long>(1);
  fln_params p = prm;
  p.bh_tree = 0;
  p.bh_schedule = 0;
  double *d_lk = ctx.d_learn[2].as<double>(2 * np);
  const LearnedCfg saved = ctx.learned;
  unsigned long long cnt = 0;
  // Records are written in traversal order, so a run that records more than
  // cap would keep only its first (coarse) node pairs: such a run is repeated
  // with a proportionally lower keep rate, which keeps the sample uniform.
  for (int attempt = 0; attempt < 4; ++attempt) {
    FLN_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st));
    ctx.learned = LearnedCfg{nullptr, 0.f, 0.f, 0, 0};
    ctx.recording.rec = d_rec;
    ctx.recording.count = d_cnt;
    ctx.recording.cap = cap;
    ctx.recording.s_min = s_min;
    ctx.recording.keep = (uint32_t)std::min(4294967295.0, std::max(0.0, keep) * 4294967296.0);
    try {
      barnes_hut_device(ctx, d_xyz, d_off, h_off, h_pairs, p, d_lk, d_lk + np, nullptr);
    } catch (...) {
      ctx.learned = saved;
      ctx.recording = Recording{};
      throw;
    }
    ctx.learned = saved;
    ctx.recording = Recording{};
    FLN_CUDA(cudaMemcpyAsync(&cnt, d_cnt, sizeof cnt, cudaMemcpyDeviceToHost, st));
    FLN_CUDA(cudaStreamSynchronize(st));
    if ((int64_t)cnt <= cap) break;
    keep *= 0.9 * (double)cap / (double)cnt;
  }
  if (recorded) *recorded = (int64_t)cnt;
  const int64_t n = (int64_t)std::min<unsigned long long>(cnt, (unsigned long long)cap);
  if (n == 0) return;
  // The trees, node bases and slot loops of that call are still in place.
  const int64_t *d_base = static_cast<const int64_t *>(ctx.d_bh[1].ptr);
  const NodeHdr *d_hdr = static_cast<const NodeHdr *>(ctx.d_bh[9].ptr);
  const NodeMom *d_mom = static_cast<const NodeMom *>(ctx.d_bh[10].ptr);
  const int32_t *d_slots = static_cast<const int32_t *>(ctx.d_bh[11].ptr);
  float *d_X = ctx.d_learn[3].as<float>(kMlpIn * n);
  double *d_approx = ctx.d_learn[4].as<double>(n);
  float *d_T = ctx.d_learn[5].as<float>(3 * n);
  float *d_S = d_T + n, *d_E = d_T + 2 * n;
  int32_t *d_valid = ctx.d_learn[6].as<int32_t>(n);
  sample_features<<<(int)((n + 255) / 256), 256, 0, st>>>(d_base, d_hdr, d_mom, d_slots, d_rec, n, p.epssq, d_X,
                                                           d_approx, d_S, d_E, p.error_est_scale);
  FLN_CUDA(cudaGetLastError());
  for (int64_t k0 = 0; k0 < n; k0 += (int64_t)1 << 30) {
    const int64_t m = std::min<int64_t>(n - k0, (int64_t)1 << 30);
    sample_exact<<<(int)m, 128, 0, st>>>(d_xyz, d_off, d_slots, d_rec + k0, d_approx + k0, m, max_terms, d_T + k0,
                                         d_valid + k0);
    FLN_CUDA(cudaGetLastError());
  }
  std::vector<float> hx(kMlpIn * n), ht(n), hs(n), he(n);
  std::vector<int32_t> hv(n);
  FLN_CUDA(cudaMemcpyAsync(hx.data(), d_X, hx.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaMemcpyAsync(ht.data(), d_T, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaMemcpyAsync(hs.data(), d_S, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaMemcpyAsync(he.data(), d_E, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaMemcpyAsync(hv.data(), d_valid, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  FLN_CUDA(cudaStreamSynchronize(st));
  for (int64_t k = 0; k < n; ++k) {
    if (!hv[k] || !std::isfinite(ht[k])) continue;
    bool ok = true;
    for (int i = 0; i < kMlpIn; ++i) ok = ok && std::isfinite(hx[kMlpIn * k + i]);
    if (!ok) continue;
    X.insert(X.end(), hx.begin() + kMlpIn * k, hx.begin() + kMlpIn * (k + 1));
    T.push_back(ht[k]);
    S.push_back(hs[k]);
    E.push_back(he[k]);
  }
}

}  // namespace fln
