// walk_plain.cu -- FP64 tree walks (the drop-in "plain" form) and the
// traversal orchestration of pepc_traverse_tree.
//
// Two semantics, both exact:
//  * per target (module_tree_walk_pthreads.f90:558-765): every target keeps
//    its own next-node index in the RPO node order; a warp of 32 key-ordered
//    targets processes, at each step, the smallest next index among its lanes
//    (all lanes that wait for that node evaluate it together, the node data is
//    loaded once).  Each lane sees exactly its own LIFO sequence, so its
//    interaction list, order and counts equal the reference's.
//  * per tile (module_tree_walk_simple.f90:256-384): a warp holds one tile of
//    <= 32 targets; a twig is opened if any target fails the MAC, children are
//    visited first to last (key order) through the fwd pointers.
// Compiled with --fmad=false: results are bit-identical to the oracle.

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "internal.cuh"

namespace pepcg {

namespace {

constexpr int kWalkThreads = 128;

struct WalkArgs {
  int64_t nt;
  const double* tx;
  const double* ty;
  const double* tz;
  const double4* nc4;
  const int2* meta;
  const int2* fwd;
  const double* mom;
  const int32_t* nleaves;
  const double* bl2;   // boxlength2[0..20]
  const double* macb;  // per-twig MAC threshold, or nullptr: bl2 of the level (Barnes-Hut)
  const double* tq;    // force_law 5: the targets' charges
  double kinv, sqrtpi;  // force_law 5: kelbg_invsqrttemp, sqrt(acos(-1))
  const double* vbox;  // 3 * nbox
  int nbox;
  double theta2, eps2;
  int32_t M;
  int64_t npart;
  double* ex;
  double* ey;
  double* ez;
  double* pot;
  double* work;
  unsigned long long* counters;  // [0] leaf, [1] twig, [2] mac
  uint32_t* status;
  unsigned int* queue;           // bucket counter, zeroed before the launch
  // per tile
  const int2* tiles;  // (first target, count)
  int64_t ntiles;
  // packed per-tile walk
  const int2* fwdf;     // (first child, next after the subtree) as forward-preorder indices
  const int32_t* tflag;  // per target: length of the tile starting there, else 0
  const int32_t* pstart;  // packed per-tile walk: first target of each pack, then nt
  const int32_t* npacks;  // the number of packs (device)
  // spatial_interaction_cutoff (module_mirror_boxes.f90:52), when finite
  int has_cut;
  double cut[3];
};

// any(abs(delta) >= spatial_interaction_cutoff) (module_tree_walk_pthreads.f90:
// 622,639; module_tree_walk_simple.f90:330,377): the node is skipped.  The walks
// are instantiated with and without the test (kCut), so that a walk without a
// finite cutoff runs the code it ran before the option existed.
template <bool kCut>
__device__ __forceinline__ bool cut_off(const WalkArgs& A, double dx, double dy, double dz) {
  return kCut && (fabs(dx) >= A.cut[0] || fabs(dy) >= A.cut[1] || fabs(dz) >= A.cut[2]);
}

__device__ __forceinline__ void warp_add_counters(unsigned long long* ctr, unsigned long long a,
                                                  unsigned long long b, unsigned long long c) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&ctr[0], a);
    atomicAdd(&ctr[1], b);
    atomicAdd(&ctr[2], c);
  }
}

template <int kLaw, bool kCut>
__global__ void __launch_bounds__(kWalkThreads) k_walk_target64(WalkArgs A) {
  __shared__ double s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned M = (unsigned)A.M;
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(A.queue, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b * 32 >= A.nt) break;
    const int64_t t = (int64_t)b * 32 + lane;
    const bool valid = t < A.nt;
    double px = 0, py = 0, pz = 0, e0 = 0, e1 = 0, e2 = 0, ph = 0, w = 0;
    KelbgArgs kel{0.0, A.kinv, A.sqrtpi};
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      if (kLaw == 5) kel.tq = A.tq[t];
      e0 = A.ex[t]; e1 = A.ey[t]; e2 = A.ez[t]; ph = A.pot[t]; w = A.work[t];
    }
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      // shifted_particle_position = x - vbox (module_tree_walk_pthreads.f90:595)
      const double sx = px - s_vb[3 * ib], sy = py - s_vb[3 * ib + 1], sz = pz - s_vb[3 * ib + 2];
      // the root is never evaluated: the walk starts with its children (:601)
      unsigned next = valid ? 1u : M;
      int64_t partner = 0;
      for (;;) {
        const unsigned u = __reduce_min_sync(0xffffffffu, next);
        if (u >= M) break;
        if (next != u) continue;
        const double4 a = A.nc4[u];
        const int2 mu = A.meta[u];
        const double dx = sx - a.x, dy = sy - a.y, dz = sz - a.z;
        const double dist2 = (dx * dx + dy * dy) + dz * dz;
        if (mu.y & kLeafFlag) {
          partner += 1;
          w += 1.0;  // counted before the cutoff test (:620-622)
          if (!cut_off<kCut>(A, dx, dy, dz)) {
            ++c_leaf;
            if (dist2 > 0.0) {
              double fx, fy, fz, fp;
              law_leaf64<kLaw>(a.w, dx, dy, dz, dist2, A.eps2, fx, fy, fz, fp, kel);
              e0 += fx; e1 += fy; e2 += fz; ph += fp;
            }
          }
          next = u + 1;
        } else {
          ++c_mac;
          if (A.theta2 * dist2 > (A.macb ? A.macb[u] : s_bl2[mu.y & 0xff])) {
            partner += A.nleaves[u];
            if (!cut_off<kCut>(A, dx, dy, dz)) {
              double m[9];
#pragma unroll
              for (int k = 0; k < 9; ++k) m[k] = A.mom[kMomStride * (int64_t)u + k];
              double fx, fy, fz, fp;
              law_twig64<kLaw>(a.w, m, dx, dy, dz, dist2, A.eps2, fx, fy, fz, fp);
              e0 += fx; e1 += fy; e2 += fz; ph += fp;
              ++c_twig;
              w += 1.0;
            }
            next = (unsigned)mu.x;
          } else {
            next = u + 1;
          }
        }
      }
      if (valid && partner != A.npart) complete = false;
    }
    if (valid) {
      A.ex[t] = e0; A.ey[t] = e1; A.ez[t] = e2; A.pot[t] = ph; A.work[t] = w;
    }
    if (__any_sync(0xffffffffu, !complete) && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  warp_add_counters(A.counters, c_leaf, c_twig, c_mac);
}

// One warp per tile (PER_TILE tiles of up to 32 targets) or per group-walk
// bucket (GROUP: kTPL x 32 key-consecutive targets, kTPL targets per lane,
// lane k holding targets t0 + k + 32 s).  A twig is accepted only if every
// target of the tile passes the MAC (module_tree_walk_simple.f90:343-382);
// children are visited first to last through fwd, so each target's
// interactions come in the reference's order.
// Launch bounds: six resident blocks per SM for one target per lane (the
// plain group walk at 4M takes 223 ms against 270 ms at the unbounded 108
// registers), four for two.
template <int kLaw, int kTPL, bool kCut>
__global__ void __launch_bounds__(kWalkThreads, kTPL == 1 ? 6 : 4) k_walk_tile64(WalkArgs A) {
  __shared__ double s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned M = (unsigned)A.M;
  constexpr int kB = 32 * kTPL;  // GROUP bucket size
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(A.queue, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    const int64_t nbk = A.tiles ? A.ntiles : (A.nt + kB - 1) / kB;
    if ((int64_t)b >= nbk) break;
    const int2 tl = A.tiles ? A.tiles[b]
                            : make_int2((int)((int64_t)b * kB), (int)min((int64_t)kB, A.nt - (int64_t)b * kB));
    bool valid[kTPL];
    int64_t t[kTPL];
    double px[kTPL], py[kTPL], pz[kTPL], e0[kTPL], e1[kTPL], e2[kTPL], ph[kTPL], w[kTPL];
    KelbgArgs kel[kTPL];
#pragma unroll
    for (int s = 0; s < kTPL; ++s) {
      valid[s] = lane + 32 * s < tl.y;
      t[s] = (int64_t)tl.x + lane + 32 * s;
      px[s] = py[s] = pz[s] = e0[s] = e1[s] = e2[s] = ph[s] = w[s] = 0.0;
      kel[s] = KelbgArgs{0.0, A.kinv, A.sqrtpi};
      if (valid[s]) {
        px[s] = A.tx[t[s]]; py[s] = A.ty[t[s]]; pz[s] = A.tz[t[s]];
        if (kLaw == 5) kel[s].tq = A.tq[t[s]];
        e0[s] = A.ex[t[s]]; e1[s] = A.ey[t[s]]; e2[s] = A.ez[t[s]]; ph[s] = A.pot[t[s]];
        w[s] = A.work[t[s]];
      }
    }
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double vx = s_vb[3 * ib], vy = s_vb[3 * ib + 1], vz = s_vb[3 * ib + 2];
      unsigned u = 0;  // tree_walk_single_aux starts at the root (:286)
      int64_t partner = 0;
      while (u < M) {
        const double4 a = A.nc4[u];
        const int2 mu = A.meta[u];
        const int2 fw = A.fwd[u];
        // d = (x - vbox) - coc (module_tree_walk_simple.f90:328,345)
        double dx[kTPL], dy[kTPL], dz[kTPL], dist2[kTPL];
#pragma unroll
        for (int s = 0; s < kTPL; ++s) {
          dx[s] = (px[s] - vx) - a.x; dy[s] = (py[s] - vy) - a.y; dz[s] = (pz[s] - vz) - a.z;
          dist2[s] = (dx[s] * dx[s] + dy[s] * dy[s]) + dz[s] * dz[s];
        }
        if (mu.y & kLeafFlag) {
          partner += 1;
#pragma unroll
          for (int s = 0; s < kTPL; ++s)
            if (valid[s] && !cut_off<kCut>(A, dx[s], dy[s], dz[s])) {
              w[s] += 1.0;
              ++c_leaf;
              if (dist2[s] > 0.0) {
                double fx, fy, fz, fp;
                law_leaf64<kLaw>(a.w, dx[s], dy[s], dz[s], dist2[s], A.eps2, fx, fy, fz, fp, kel[s]);
                e0[s] += fx; e1[s] += fy; e2[s] += fz; ph[s] += fp;
              }
            }
          u = (unsigned)fw.y;
        } else {
          const double thr = A.macb ? A.macb[u] : s_bl2[mu.y & 0xff];
          // MAC evaluations stop at the tile's first failing target, in
          // target order (:343-370)
          int first_fail = kB;
          unsigned any_fail = 0;
#pragma unroll
          for (int s = 0; s < kTPL; ++s) {
            const bool ok = !valid[s] || (A.theta2 * dist2[s] > thr);
            const unsigned fail = __ballot_sync(0xffffffffu, !ok);
            if (fail && first_fail == kB) first_fail = 32 * s + __ffs(fail) - 1;
            any_fail |= fail;
          }
#pragma unroll
          for (int s = 0; s < kTPL; ++s)
            if (valid[s] && lane + 32 * s <= first_fail) ++c_mac;
          if (any_fail == 0) {
            partner += A.nleaves[u];
            double m[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) m[k] = A.mom[kMomStride * (int64_t)u + k];
#pragma unroll
            for (int s = 0; s < kTPL; ++s)
              if (valid[s] && !cut_off<kCut>(A, dx[s], dy[s], dz[s])) {
                double fx, fy, fz, fp;
                law_twig64<kLaw>(a.w, m, dx[s], dy[s], dz[s], dist2[s], A.eps2, fx, fy, fz, fp);
                e0[s] += fx; e1[s] += fy; e2[s] += fz; ph[s] += fp;
                w[s] += 1.0;
                ++c_twig;
              }
            u = (unsigned)fw.y;
          } else {
            u = (unsigned)fw.x;
          }
        }
      }
      if (partner != A.npart) complete = false;
    }
#pragma unroll
    for (int s = 0; s < kTPL; ++s)
      if (valid[s]) {
        A.ex[t[s]] = e0[s]; A.ey[t[s]] = e1[s]; A.ez[t[s]] = e2[s]; A.pot[t[s]] = ph[s];
        A.work[t[s]] = w[s];
      }
    if (!complete && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  warp_add_counters(A.counters, c_leaf, c_twig, c_mac);
}

// Tiles of the grown particles: tree nodes with <= T leaves whose parent has
// more than T (the key-prefix split of tree_walk_init_aux,
// module_tree_walk_simple.f90:168-211, is exactly this set of nodes).
// Several reference tiles per warp (simple-walk semantics, module_tree_walk_
// simple.f90:256-385).  Each warp takes one pack of consecutive whole tiles
// of at most 32 targets (k_pack_tiles).  Every tile walks the tree in forward
// preorder (children first to
// last); the warp steps through the union of its tiles' walks in that order:
// at each step the lanes whose tile stands at the smallest forward-preorder
// index f evaluate node f together (one load for all of them), and each tile
// decides accept / open by a ballot over its own lanes.  A lane's sequence of
// interactions is exactly its tile's, so fields, work and MAC counts equal
// the one-tile-per-warp walk's.
template <int kLaw, bool kCut>
// Six resident blocks per SM (80 registers, a few spilled): at 4M, T = 16,
// 260 ms against 296 ms at the unbounded 110 registers (four blocks).
__global__ void __launch_bounds__(kWalkThreads, 6) k_walk_tilepack64(WalkArgs A) {
  __shared__ double s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned M = (unsigned)A.M;
  const int64_t npk = *A.npacks;
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(A.queue, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b >= npk) break;
    int tl0, len;
    const int64_t t0 = A.pstart[b];
    const bool valid = pack_lane(A.pstart, A.tflag, b, lane, tl0, len);
    if (!__any_sync(0xffffffffu, valid)) {
      if (lane == 0) atomicOr(A.status, ST_INCOMPLETE);  // a pack must start with a tile
      continue;
    }
    const int64_t t = t0 + lane;
    const unsigned tmask = valid ? (((len >= 32) ? 0xffffffffu : ((1u << len) - 1u)) << tl0) : 0u;
    double px = 0, py = 0, pz = 0, e0 = 0, e1 = 0, e2 = 0, ph = 0, w = 0;
    KelbgArgs kel{0.0, A.kinv, A.sqrtpi};
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      if (kLaw == 5) kel.tq = A.tq[t];
      e0 = A.ex[t]; e1 = A.ey[t]; e2 = A.ez[t]; ph = A.pot[t]; w = A.work[t];
    }
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double vx = s_vb[3 * ib], vy = s_vb[3 * ib + 1], vz = s_vb[3 * ib + 2];
      unsigned u = 0, uf = 0;  // tree_walk_single_aux starts at the root (:286)
      int64_t partner = 0;
      for (;;) {
        const unsigned f = __reduce_min_sync(0xffffffffu, valid ? uf : 0xffffffffu);
        if (f >= M) break;
        // the lanes at node f: whole tiles, all at the same node, so they take
        // the same branch below
        const unsigned am = __ballot_sync(0xffffffffu, valid && uf == f);
        if (valid && uf == f) {
          const double4 a = A.nc4[u];
          const int2 mu = A.meta[u];
          const int2 fw = A.fwd[u];
          const int2 ff = A.fwdf[u];
          // d = (x - vbox) - coc (module_tree_walk_simple.f90:328,345)
          const double dx = (px - vx) - a.x, dy = (py - vy) - a.y, dz = (pz - vz) - a.z;
          const double dist2 = (dx * dx + dy * dy) + dz * dz;
          if (mu.y & kLeafFlag) {
            partner += 1;
            if (!cut_off<kCut>(A, dx, dy, dz)) {  // before the work count (:330)
              w += 1.0;
              ++c_leaf;
              if (dist2 > 0.0) {
                double fx, fy, fz, fp;
                law_leaf64<kLaw>(a.w, dx, dy, dz, dist2, A.eps2, fx, fy, fz, fp, kel);
                e0 += fx; e1 += fy; e2 += fz; ph += fp;
              }
            }
            u = (unsigned)fw.y;
            uf = (unsigned)ff.y;
          } else {
            const bool ok = A.theta2 * dist2 > (A.macb ? A.macb[u] : s_bl2[mu.y & 0xff]);
            const unsigned tf = __ballot_sync(am, !ok) & tmask;
            // MAC evaluations stop at the tile's first failing target (:343-370)
            const int first_fail = tf ? __ffs(tf) - 1 : 32;
            if (lane <= first_fail) ++c_mac;
            if (tf == 0) {
              partner += A.nleaves[u];
              if (!cut_off<kCut>(A, dx, dy, dz)) {  // :377
                double m[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) m[k] = A.mom[kMomStride * (int64_t)u + k];
                double fx, fy, fz, fp;
                law_twig64<kLaw>(a.w, m, dx, dy, dz, dist2, A.eps2, fx, fy, fz, fp);
                e0 += fx; e1 += fy; e2 += fz; ph += fp;
                w += 1.0;
                ++c_twig;
              }
              u = (unsigned)fw.y;
              uf = (unsigned)ff.y;
            } else {
              u = (unsigned)fw.x;
              uf = (unsigned)ff.x;
            }
          }
        }
        __syncwarp();
      }
      if (valid && partner != A.npart) complete = false;
    }
    if (valid) {
      A.ex[t] = e0; A.ey[t] = e1; A.ez[t] = e2; A.pot[t] = ph; A.work[t] = w;
    }
    if (__any_sync(0xffffffffu, !complete) && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  warp_add_counters(A.counters, c_leaf, c_twig, c_mac);
}

// Greedy packing of consecutive tiles into warps.  The targets are cut into
// chunks of kPackChunk, each chunk's bounds moved forward to the next tile
// start; one warp per chunk steps through its tiles in order and opens a new
// pack whenever the next tile would not fit the 32 lanes.  Two consecutive
// packs hold at least 33 targets between them, so a chunk of kPackChunk + 31
// targets has at most 127 packs (kPackSlots leaves a margin).  The packs are
// then compacted in chunk order into pstart.
constexpr int64_t kPackChunk = 2048;
constexpr int kPackSlots = 256;

// the first tile start at or after p, or nt: a tile holds at most 32
// targets, so one lies in [p, p + 31]
__device__ __forceinline__ int64_t first_tile_start(int64_t p, int64_t nt,
                                                    const int32_t* __restrict__ tflag, int lane) {
  if (p >= nt) return nt;
  const int64_t q = p + lane;
  const unsigned m = __ballot_sync(0xffffffffu, q >= nt || tflag[q] > 0);
  return m ? min(p + __ffs(m) - 1, nt) : nt;
}

__global__ void k_pack_tiles(int64_t nt, const int32_t* __restrict__ tflag,
                             int32_t* __restrict__ raw, int32_t* __restrict__ pcount,
                             uint32_t* status) {
  const int lane = threadIdx.x & 31;
  const int64_t nchunks = (nt + kPackChunk - 1) / kPackChunk;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t ch = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; ch < nchunks;
       ch += nwarps) {
    int64_t p = first_tile_start(ch * kPackChunk, nt, tflag, lane);
    const int64_t e = first_tile_start((ch + 1) * kPackChunk, nt, tflag, lane);
    int k = 0;
    while (p < e && k < kPackSlots) {
      if (lane == 0) raw[ch * kPackSlots + k] = (int32_t)p;
      ++k;
      // the pack ends at the last tile start (or e) in [p + 1, p + 32]
      const int64_t q = p + 1 + lane;
      const unsigned m = __ballot_sync(0xffffffffu, q <= e && (q == e || tflag[q] > 0));
      p = m ? p + 1 + (31 - __clz(m)) : e;
    }
    if (lane == 0) {
      if (p < e) atomicOr(status, ST_INCOMPLETE);
      pcount[ch] = k;
    }
  }
}

__global__ void k_pack_compact(int64_t nt, int64_t nchunks, const int32_t* __restrict__ raw,
                               const int32_t* __restrict__ pcount, const int32_t* __restrict__ poff,
                               int32_t* __restrict__ pstart) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nchunks * kPackSlots;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ch = i / kPackSlots;
    const int k = (int)(i % kPackSlots);
    if (k < pcount[ch]) pstart[poff[ch] + k] = raw[i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) pstart[poff[nchunks]] = (int32_t)nt;
}

// per-target tile lengths from the compact (first, count) list
__global__ void k_tile_flags(int64_t ntiles, const int2* __restrict__ tiles,
                             int32_t* __restrict__ tflag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ntiles;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int2 tl = tiles[i];
    tflag[tl.x] = tl.y;
  }
}

__global__ void k_tiles_from_tree(int32_t M, int T, const int32_t* __restrict__ nleaves,
                                  const int32_t* __restrict__ parent,
                                  const int32_t* __restrict__ first_part, int2* tiles,
                                  unsigned int* ntiles) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < M;
       u += (int64_t)gridDim.x * blockDim.x) {
    int lv = nleaves[u];
    int p = parent[u];
    if (lv <= T && (p < 0 || nleaves[p] > T)) {
      unsigned slot = atomicAdd(ntiles, 1u);
      tiles[slot] = make_int2(first_part[u], lv);
    }
  }
}

__global__ void k_same_keys(int64_t n, const int64_t* __restrict__ a, const int64_t* __restrict__ b,
                            unsigned int* differ) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (a[i] != b[i]) atomicOr(differ, 1u);
}

__global__ void k_reset_counter(unsigned int* q) { *q = 0; }

// calls f(law, cut) with both as compile-time constants (std::integral_constant)
template <class F>
void launch_law_cut(int law, bool cut, F&& f) {
  using T = std::true_type;
  using Fl = std::false_type;
  auto go = [&](auto L) {
    if (cut) f(L, T{});
    else f(L, Fl{});
  };
  if (law == 2) go(std::integral_constant<int, 2>{});
  else if (law == 4) go(std::integral_constant<int, 4>{});
  else if (law == 5) go(std::integral_constant<int, 5>{});
  else go(std::integral_constant<int, 3>{});
}

// mac (coulomb/module_interaction_specific.f90:256-275) for mac_select != 0,
// as a per-twig threshold t with "accept iff theta2 dist2 > t": the Bmax MAC
// has t = min(bmax^2, 3 boxlength2(level)); any other selection accepts
// nothing (the N^2 code), t = +inf.
__global__ void k_mac_thresholds(int64_t M, int mode, const int2* __restrict__ meta,
                                 const double* __restrict__ mom, const double* __restrict__ bl2,
                                 double* __restrict__ macb) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < M;
       u += (int64_t)gridDim.x * blockDim.x) {
    const int2 mu = meta[u];
    if (mu.y & kLeafFlag) continue;
    if (mode == 1) {
      const double bmax = mom[kMomStride * u + kMomBmax];
      macb[u] = fmin(bmax * bmax, 3.0 * bl2[mu.y & 0xff]);
    } else {
      macb[u] = INFINITY;
    }
  }
}

}  // namespace

int launch_walk_mixed(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                      double* ex, double* ey, double* ez, double* pot, double* work,
                      const int2* tiles, int64_t ntiles, bool per_target, const int32_t* tflag,
                      const int32_t* pstart, const int32_t* npacks, cudaStream_t s, int slot);

const double* grown_charges_if_same(Ctx* c, int64_t nt, const int64_t* d_tkeys) {
  if (!d_tkeys || nt != c->n) return nullptr;
  unsigned int* d_diff = reinterpret_cast<unsigned int*>(c->d_small + 7);
  unsigned int h_diff = 1;
  cudaMemsetAsync(d_diff, 0, 4, c->stream);
  COUNT_LAUNCH();
  k_same_keys<<<296, 256, 0, c->stream>>>(nt, d_tkeys, c->key.p, d_diff);
  if (!cuda_ok(c, cudaMemcpyAsync(&h_diff, d_diff, 4, cudaMemcpyDeviceToHost, c->stream), "keys") ||
      !cuda_ok(c, cudaStreamSynchronize(c->stream), "keys"))
    return nullptr;
  return h_diff == 0 ? c->q.p : nullptr;
}

int prepare_mac(Ctx* c, const double** macb) {
  *macb = nullptr;
  if (c->prm.mac_select == 0) return PEPCG_OK;
  const int64_t M = c->nnodes;
  if (!ensure(c, c->macb, M, "mac thresholds")) return PEPCG_ERR_OOM;
  COUNT_LAUNCH();
  const unsigned g = (unsigned)((M + 255) / 256 > 148 * 16 ? 148 * 16 : (M + 255) / 256);
  k_mac_thresholds<<<g, 256, 0, c->stream>>>(M, c->prm.mac_select, c->meta.p, c->mom.p,
                                             c->d_box + 9, c->macb.p);
  if (!cuda_ok(c, cudaGetLastError(), "mac thresholds")) return PEPCG_ERR_CUDA;
  *macb = c->macb.p;
  return PEPCG_OK;
}

int traverse_device(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                    const int64_t* tkeys, bool self, double* ex, double* ey, double* ez,
                    double* pot, double* work, const double* tq, const ChunkPlan* plan) {
  if (!c->has_tree) {
    c->err = "traverse called without a grown tree";
    return PEPCG_ERR_NO_TREE;
  }
  if (nt <= 0) return PEPCG_OK;
  if (c->prm.force_law == 5 && !tq) {
    c->err = "force_law 5 (Kelbg) needs the targets' charges: traverse the grown particles "
             "(pepcg_traverse_self_device, pepcg_traverse_range_device, or pepcg_traverse_tree "
             "with the grown keys)";
    return PEPCG_ERR_UNSUPPORTED;
  }
  cudaStream_t s = c->stream;
  const int walk = c->prm.walk;
  if (!cuda_ok(c, cudaMemsetAsync(c->counters.p, 0, 4 * sizeof(unsigned long long), s), "ctr") ||
      !cuda_ok(c, cudaMemsetAsync(c->d_status, 0, 4, s), "status"))
    return PEPCG_ERR_CUDA;
  int64_t ntiles = 0;
  if (walk == PEPCG_WALK_PER_TILE) {
    const int T = c->prm.tile_size < 1 ? 1 : (c->prm.tile_size > 32 ? 32 : c->prm.tile_size);
    bool from_tree = self;
    if (!self && tkeys && nt == c->n) {
      unsigned int* d_diff = reinterpret_cast<unsigned int*>(c->d_small + 4);
      unsigned int h_diff = 1;
      cudaMemsetAsync(d_diff, 0, 4, s);
      COUNT_LAUNCH();
      k_same_keys<<<296, 256, 0, s>>>(nt, tkeys, c->key.p, d_diff);
      if (!cuda_ok(c, cudaMemcpyAsync(&h_diff, d_diff, 4, cudaMemcpyDeviceToHost, s), "tiles") ||
          !cuda_ok(c, cudaStreamSynchronize(s), "tiles"))
        return PEPCG_ERR_CUDA;
      from_tree = (h_diff == 0);
    }
    if (!ensure(c, c->tiles, 2 * (nt + 1), "tiles")) return PEPCG_ERR_OOM;
    int2* d_tiles = reinterpret_cast<int2*>(c->tiles.p);
    if (from_tree) {
      unsigned int* d_nt = reinterpret_cast<unsigned int*>(c->d_small + 5);
      unsigned int h_nt = 0;
      cudaMemsetAsync(d_nt, 0, 4, s);
      COUNT_LAUNCH();
      k_tiles_from_tree<<<296, 256, 0, s>>>((int32_t)c->nnodes, T, c->nleaves_ptr(), c->parent.p,
                                            c->first_part.p, d_tiles, d_nt);
      if (!cuda_ok(c, cudaMemcpyAsync(&h_nt, d_nt, 4, cudaMemcpyDeviceToHost, s), "tiles") ||
          !cuda_ok(c, cudaStreamSynchronize(s), "tiles"))
        return PEPCG_ERR_CUDA;
      ntiles = h_nt;
    } else {
      int rc = host_tiles(c, nt, tkeys, T, d_tiles, &ntiles);
      if (rc) return rc;
    }
  }
  // per-tile walk: several whole tiles per warp.  Measured at 4M (Plummer,
  // theta 0.4): the packed FP64 walk beats one tile per warp at every tile
  // size (32: 278 vs 851 ms); in the mixed form the wide group kernel with
  // tiles as buckets wins at 32 targets (127 vs 148 ms) and loses at 24
  // (167 vs 146 ms)
  const bool packed = walk == PEPCG_WALK_PER_TILE &&
                      (c->prm.precision == PEPCG_PRECISION_PLAIN || c->prm.tile_size <= 24);
  const int32_t* pstart = nullptr;
  const int32_t* npacks = nullptr;
  if (packed) {
    if (!ensure(c, c->tflag, nt, "tile flags")) return PEPCG_ERR_OOM;
    if (!cuda_ok(c, cudaMemsetAsync(c->tflag.p, 0, nt * sizeof(int32_t), s), "tile flags"))
      return PEPCG_ERR_CUDA;
    COUNT_LAUNCH();
    k_tile_flags<<<296, 256, 0, s>>>(ntiles, reinterpret_cast<const int2*>(c->tiles.p),
                                     c->tflag.p);
    // packs of whole tiles, <= 32 targets each
    const int64_t nch = (nt + kPackChunk - 1) / kPackChunk;
    const int64_t ntmp = (nch + 1 + 2047) / 2048 + 1;
    const int64_t cap = nch * kPackSlots + 1;  // packs + the end; every slot may be used
    if (!ensure(c, c->tpack, (size_t)(nch * kPackSlots + 2 * (nch + 1) + ntmp + cap), "packs"))
      return PEPCG_ERR_OOM;
    int32_t* raw = c->tpack.p;
    int32_t* pcount = raw + nch * kPackSlots;
    int32_t* poff = pcount + nch + 1;
    int32_t* tmp = poff + nch + 1;
    int32_t* ps = tmp + ntmp;
    pstart = ps;
    npacks = poff + nch;
    if (!cuda_ok(c, cudaMemsetAsync(pcount, 0, (nch + 1) * sizeof(int32_t), s), "packs"))
      return PEPCG_ERR_CUDA;
    const unsigned gw = (unsigned)std::min<int64_t>((nch * 32 + 255) / 256, 148 * 8);
    COUNT_LAUNCH();
    k_pack_tiles<<<gw, 256, 0, s>>>(nt, c->tflag.p, raw, pcount, c->d_status);
    exclusive_scan_i32(pcount, poff, nch + 1, tmp, s);
    const unsigned gc = (unsigned)std::min<int64_t>((nch * kPackSlots + 255) / 256, 148 * 8);
    COUNT_LAUNCH();
    k_pack_compact<<<gc, 256, 0, s>>>(nt, nch, raw, pcount, poff, ps);
  }
  const int nchunks = plan ? plan->nchunks : 1;
  if (nchunks > 1) {
    bool ok = walk != PEPCG_WALK_PER_TILE && !c->far_field && nchunks <= Ctx::kMaxChunks &&
              plan->bounds[0] == 0 && plan->bounds[nchunks] == nt;
    for (int k = 1; ok && k < nchunks; ++k)
      ok = plan->bounds[k] % c->group_size() == 0 && plan->bounds[k] >= plan->bounds[k - 1];
    if (!ok) {
      c->err = "traverse: invalid chunk plan";
      return PEPCG_ERR_BAD_ARG;
    }
  }
  WalkArgs A;
  A.nc4 = c->nc4.p;
  A.meta = c->meta.p;
  A.fwd = c->fwd.p;
  A.mom = c->mom.p;
  A.nleaves = c->nleaves_ptr();
  A.bl2 = c->d_box + 9;
  {
    int rc = prepare_mac(c, &A.macb);
    if (rc) return rc;
  }
  A.vbox = c->d_vbox;
  A.nbox = c->nboxes;
  A.theta2 = c->prm.theta2;
  A.eps2 = c->prm.eps2;
  A.M = (int32_t)c->nnodes;
  A.npart = c->n;
  A.counters = c->counters.p;
  A.status = c->d_status;
  A.queue = c->walk_queue();
  A.tiles = reinterpret_cast<const int2*>(c->tiles.p);
  A.ntiles = ntiles;
  A.kinv = c->prm.kelbg_invsqrttemp;
  A.sqrtpi = std::sqrt(std::acos(-1.0));
  A.fwdf = c->fwdf.p;
  A.tflag = c->tflag.p;
  A.pstart = pstart;
  A.npacks = npacks;
  A.has_cut = has_spatial_cutoff(c->prm) ? 1 : 0;
  for (int k = 0; k < 3; ++k) A.cut[k] = c->prm.spatial_interaction_cutoff[k];
  const int blocks = 148 * 8;
  // chunks alternate between the context stream and walk2, so that each
  // chunk's walk starts while the previous one finishes its last buckets
  const bool two = nchunks > 1 && c->walk2;
  if (two && (!cuda_ok(c, cudaEventRecord(c->fork, s), "fork") ||
              !cuda_ok(c, cudaStreamWaitEvent(c->walk2, c->fork, 0), "fork")))
    return PEPCG_ERR_CUDA;
  for (int k = 0; k < nchunks; ++k) {
    const int64_t t0 = nchunks > 1 ? plan->bounds[k] : 0;
    const int64_t t1 = nchunks > 1 ? plan->bounds[k + 1] : nt;
    const int slot = two ? (k & 1) : 0;
    const cudaStream_t sk = slot ? c->walk2 : s;
    A.queue = c->walk_queue(slot);
    if (plan && plan->ready && !cuda_ok(c, cudaStreamWaitEvent(sk, plan->ready[k], 0), "chunk wait"))
      return PEPCG_ERR_CUDA;
    if (k == 0) cudaEventRecord(c->ev[5], s);
    if (t1 > t0) {
      A.nt = t1 - t0;
      A.tx = tx + t0; A.ty = ty + t0; A.tz = tz + t0;
      A.ex = ex + t0; A.ey = ey + t0; A.ez = ez + t0; A.pot = pot + t0; A.work = work + t0;
      A.tq = tq ? tq + t0 : nullptr;
      COUNT_LAUNCH();
      k_reset_counter<<<1, 1, 0, sk>>>(A.queue);
      if (c->prm.precision == PEPCG_PRECISION_PLAIN) {
        COUNT_LAUNCH();
        const int law = c->prm.force_law;
        const bool cut = A.has_cut != 0;
        if (walk == PEPCG_WALK_PER_TARGET) {
          launch_law_cut(law, cut, [&](auto L, auto C) {
            k_walk_target64<decltype(L)::value, decltype(C)::value><<<blocks, kWalkThreads, 0, sk>>>(A);
          });
        } else if (packed) {
          launch_law_cut(law, cut, [&](auto L, auto C) {
            k_walk_tilepack64<decltype(L)::value, decltype(C)::value><<<blocks, kWalkThreads, 0, sk>>>(A);
          });
        } else {
          if (walk == PEPCG_WALK_GROUP) A.tiles = nullptr;
          if (walk == PEPCG_WALK_GROUP && c->group_size() == 64) {
            launch_law_cut(law, cut, [&](auto L, auto C) {
              k_walk_tile64<decltype(L)::value, 2, decltype(C)::value><<<blocks, kWalkThreads, 0, sk>>>(A);
            });
          } else {
            launch_law_cut(law, cut, [&](auto L, auto C) {
              k_walk_tile64<decltype(L)::value, 1, decltype(C)::value><<<blocks, kWalkThreads, 0, sk>>>(A);
            });
          }
        }
      } else {
        int rc = launch_walk_mixed(c, t1 - t0, A.tx, A.ty, A.tz, A.ex, A.ey, A.ez, A.pot, A.work,
                                   walk == PEPCG_WALK_PER_TILE ? A.tiles : nullptr, ntiles,
                                   walk == PEPCG_WALK_PER_TARGET, packed ? c->tflag.p : nullptr,
                                   pstart, npacks, sk, slot);
        if (rc) return rc;
      }
      if (!cuda_ok(c, cudaGetLastError(), "walk launch")) return PEPCG_ERR_CUDA;
    }
    if (plan && plan->done) cudaEventRecord(plan->done[k], sk);
  }
  if (two && (!cuda_ok(c, cudaEventRecord(c->join, c->walk2), "join") ||
              !cuda_ok(c, cudaStreamWaitEvent(s, c->join, 0), "join")))
    return PEPCG_ERR_CUDA;
  cudaEventRecord(c->ev[6], s);
  if (c->far_field) {
    int rc = lattice_add(c, nt, tx, ty, tz, ex, ey, ez, pot, false);
    if (rc) return rc;
  }
  cudaEventRecord(c->ev[7], s);
  if (plan && plan->before_sync && !plan->before_sync()) return PEPCG_ERR_CUDA;
  unsigned long long ctr[4];
  uint32_t st = 0;
  if (!cuda_ok(c, cudaMemcpyAsync(ctr, c->counters.p, 4 * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, s), "counters") ||
      !cuda_ok(c, cudaMemcpyAsync(&st, c->d_status, 4, cudaMemcpyDeviceToHost, s), "status") ||
      !cuda_ok(c, cudaStreamSynchronize(s), "walk"))
    return PEPCG_ERR_CUDA;
  c->st.leaf_interactions = (int64_t)ctr[0];
  c->st.twig_interactions = (int64_t)ctr[1];
  c->st.interactions = (int64_t)(ctr[0] + ctr[1]);
  c->st.mac_evaluations = (int64_t)ctr[2];
  float ms = 0;
  if (cudaEventElapsedTime(&ms, c->ev[5], c->ev[6]) == cudaSuccess) c->st.t_walk_ms = ms;
  if (cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]) == cudaSuccess) c->st.t_lattice_ms = ms;
  if (st) return status_to_code(c, st);
  return PEPCG_OK;
}

}  // namespace pepcg
