// walk_mixed.cu -- the mixed-precision walks.
//
// Precision contract: the target-minus-node offset is formed in FP64 and
// rounded to FP32; the interaction (monopole + dipole + quadrupole, Plummer
// softened) is evaluated in FP32 with rsqrt; each target sums its FP32
// contributions over chunks of kChunk walk steps and adds every chunk sum to
// FP64 accumulators.  Node moments are computed in FP64 by the upward pass
// and rounded to FP32 once per grow (k_mom32 in grow.cu).
//
// The FP32 twig interaction is the reference's quadrupole kernel
// (coulomb/module_coulomb_kernels.f90:60-145) rewritten in the equivalent
// form
//   phi = q/r - (d.p)/r^3 + 3 (d.M.d)/r^5 - tr(Q)/r^3
//   E   = d [q/r^3 - 3 (d.p)/r^5 + 15 (d.M.d)/r^7 - 3 tr(Q)/r^5] + p/r^3 - 6 (M.d)/r^5
// with M = [[qxx, qxy/2, qzx/2], [qxy/2, qyy, qyz/2], [qzx/2, qyz/2, qzz]]
// (expanding the reference's fdx.. / pre2x.. terms gives exactly these
// polynomials), which needs ~45 FP32 operations instead of ~130.
//
// Walks:
//  * group / per tile: a warp holds one tile of targets (32 key-consecutive
//    targets in GROUP mode, the reference's <= tile_size key-prefix tiles in
//    PER_TILE mode) and visits nodes in the RPO order; a twig is accepted
//    only if every target passes the MAC (module_tree_walk_simple.f90:343-382
//    semantics), so accepted interactions are warp-uniform.
//  * per target: the same min-next-index schedule as the FP64 per-target walk
//    (module_tree_walk_pthreads.f90 semantics) with FP32 interactions.

#include "internal.cuh"

namespace pepcg {

__device__ unsigned int g_bucket_counter_mixed;

namespace {

constexpr int kMixThreads = 128;
constexpr int kChunk = 32;

struct MixArgs {
  int64_t nt;
  const double* tx;
  const double* ty;
  const double* tz;
  const double4* nc4;
  const int2* meta;
  const float4* mom32;  // 3 float4 per node
  const int32_t* nleaves;
  const double* bl2;
  const double* vbox;
  int nbox;
  float theta2;
  float eps2;
  double theta2_64;
  int32_t M;
  int64_t npart;
  double* ex;
  double* ey;
  double* ez;
  double* pot;
  double* work;
  unsigned long long* counters;
  uint32_t* status;
  const int2* tiles;  // PER_TILE tiles, or nullptr for GROUP (implicit 32-target buckets)
  int64_t ntiles;
};

__device__ __forceinline__ void leaf32(float q, float dx, float dy, float dz, float eps2,
                                       float& ax, float& ay, float& az, float& ap) {
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
  const float ri = rsqrtf(r2);
  const float qr = q * ri;
  const float qr3 = qr * ri * ri;
  ap += qr;
  ax = fmaf(qr3, dx, ax);
  ay = fmaf(qr3, dy, ay);
  az = fmaf(qr3, dz, az);
}

// m0 = (px, py, pz, qxx), m1 = (qyy, qzz, qxy/2, qyz/2), m2 = (qzx/2, tr, q, 0)
__device__ __forceinline__ void twig32(float4 m0, float4 m1, float4 m2, float dx, float dy,
                                       float dz, float eps2, float& ax, float& ay, float& az,
                                       float& ap) {
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
  const float ri = rsqrtf(r2);
  const float ri2 = ri * ri;
  const float rd3 = ri * ri2;
  const float rd5 = rd3 * ri2;
  const float rd7 = rd5 * ri2;
  const float q = m2.z, tr = m2.y;
  const float dp = fmaf(dx, m0.x, fmaf(dy, m0.y, dz * m0.z));
  const float vx = fmaf(m0.w, dx, fmaf(m1.z, dy, m2.x * dz));
  const float vy = fmaf(m1.z, dx, fmaf(m1.x, dy, m1.w * dz));
  const float vz = fmaf(m2.x, dx, fmaf(m1.w, dy, m1.y * dz));
  const float dqd = fmaf(dx, vx, fmaf(dy, vy, dz * vz));
  // phi = q/r - dp/r^3 + 3 dQd/r^5 - tr/r^3
  ap += fmaf(q, ri, fmaf(3.0f * dqd, rd5, -(dp + tr) * rd3));
  const float c = fmaf(q, rd3, fmaf(15.0f * dqd, rd7, -3.0f * (dp + tr) * rd5));
  const float s6 = 6.0f * rd5;
  ax = fmaf(c, dx, fmaf(rd3, m0.x, fmaf(-s6, vx, ax)));
  ay = fmaf(c, dy, fmaf(rd3, m0.y, fmaf(-s6, vy, ay)));
  az = fmaf(c, dz, fmaf(rd3, m0.z, fmaf(-s6, vz, az)));
}

__device__ __forceinline__ void warp_add3(unsigned long long* ctr, unsigned long long a,
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

__global__ void __launch_bounds__(kMixThreads) k_walk_group_mixed(MixArgs A) {
  __shared__ float s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = (float)A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned M = (unsigned)A.M;
  const int64_t nbuckets = A.tiles ? A.ntiles : (A.nt + 31) / 32;
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(&g_bucket_counter_mixed, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b >= nbuckets) break;
    int64_t t0;
    int cnt;
    if (A.tiles) {
      const int2 tl = A.tiles[b];
      t0 = tl.x;
      cnt = tl.y;
    } else {
      t0 = (int64_t)b * 32;
      cnt = (int)min((int64_t)32, A.nt - t0);
    }
    const bool valid = lane < cnt;
    const int64_t t = t0 + lane;
    double px = 0, py = 0, pz = 0;
    double E0 = 0, E1 = 0, E2 = 0, PH = 0, W = 0;
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      E0 = A.ex[t]; E1 = A.ey[t]; E2 = A.ez[t]; PH = A.pot[t]; W = A.work[t];
    }
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double sx = px - s_vb[3 * ib], sy = py - s_vb[3 * ib + 1], sz = pz - s_vb[3 * ib + 2];
      float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
      int steps = 0;
      int64_t partner = 0;
      unsigned nint = 0;
      unsigned u = 0;
      while (u < M) {
        const double4 a = A.nc4[u];
        const int2 mu = A.meta[u];
        const double dx64 = sx - a.x, dy64 = sy - a.y, dz64 = sz - a.z;
        const float dx = (float)dx64, dy = (float)dy64, dz = (float)dz64;
        if (mu.y & kLeafFlag) {
          partner += 1;
          ++nint;
          const bool self = (dx64 == 0.0 && dy64 == 0.0 && dz64 == 0.0);
          if (valid && !self) {
            leaf32((float)a.w, dx, dy, dz, A.eps2, ax, ay, az, ap);
            ++c_leaf;
          }
          u = u + 1;
        } else {
          const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          const bool ok = !valid || (A.theta2 * r2 > s_bl2[mu.y & 0xff]);
          const unsigned fail = __ballot_sync(0xffffffffu, !ok);
          // MAC evaluations stop at the first failing target (walk_simple :343-370)
          const int first_fail = fail ? __ffs(fail) - 1 : 32;
          if (valid && lane <= first_fail) ++c_mac;
          if (fail == 0) {
            partner += A.nleaves[u];
            ++nint;
            const float4 m0 = A.mom32[3 * (int64_t)u], m1 = A.mom32[3 * (int64_t)u + 1],
                         m2 = A.mom32[3 * (int64_t)u + 2];
            if (valid) {
              twig32(m0, m1, m2, dx, dy, dz, A.eps2, ax, ay, az, ap);
              ++c_twig;
            }
            u = (unsigned)mu.x;
          } else {
            u = u + 1;
          }
        }
        if (++steps == kChunk) {  // flush the FP32 chunk sums into FP64
          E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
          ax = ay = az = ap = 0.f;
          steps = 0;
        }
      }
      E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
      W += (double)nint;
      if (partner != A.npart) complete = false;
    }
    if (valid) {
      A.ex[t] = E0; A.ey[t] = E1; A.ez[t] = E2; A.pot[t] = PH; A.work[t] = W;
    }
    if (!complete && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  warp_add3(A.counters, c_leaf, c_twig, c_mac);
}

// Group walk in two phases per warp.
//  Phase A (traversal): the warp walks the RPO node order; at a twig every
//    lane evaluates the Barnes-Hut MAC in FP64 and the twig is accepted only if
//    all lanes pass (module_tree_walk_simple.f90:343-382 semantics).  Accepted
//    twigs and reached leaves are appended to per-warp shared-memory lists.
//  Phase B (evaluation): the listed nodes are staged 32 at a time, lane k
//    loading node k's record (independent loads, one latency per batch), and
//    every lane then evaluates all staged nodes from broadcast shared-memory
//    reads.  Each batch's FP32 sums are added to the FP64 accumulators.
constexpr int kListCap = 128;
struct __align__(16) Staged {
  double cx, cy, cz, q;  // coc (FP64) and charge
  float4 m0, m1, m2;     // FP32 moments (twigs)
};

__global__ void __launch_bounds__(kMixThreads) k_walk_group_mixed_ab(MixArgs A) {
  __shared__ double s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  __shared__ int s_tw[kMixThreads / 32][kListCap];
  __shared__ int s_lf[kMixThreads / 32][kListCap];
  __shared__ Staged s_st[kMixThreads / 32][32];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int* tw = s_tw[w];
  int* lf = s_lf[w];
  Staged* st = s_st[w];
  const unsigned M = (unsigned)A.M;
  const double theta2 = (double)A.theta2_64;
  const int64_t nbuckets = A.tiles ? A.ntiles : (A.nt + 31) / 32;
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(&g_bucket_counter_mixed, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b >= nbuckets) break;
    int64_t t0;
    int cnt;
    if (A.tiles) {
      const int2 tl = A.tiles[b];
      t0 = tl.x;
      cnt = tl.y;
    } else {
      t0 = (int64_t)b * 32;
      cnt = (int)min((int64_t)32, A.nt - t0);
    }
    const bool valid = lane < cnt;
    const int64_t t = t0 + lane;
    double px = 0, py = 0, pz = 0;
    double E0 = 0, E1 = 0, E2 = 0, PH = 0, W = 0;
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      E0 = A.ex[t]; E1 = A.ey[t]; E2 = A.ez[t]; PH = A.pot[t]; W = A.work[t];
    }
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double sx = px - s_vb[3 * ib], sy = py - s_vb[3 * ib + 1], sz = pz - s_vb[3 * ib + 2];
      int64_t partner = 0;
      unsigned u = 0;
      while (u < M) {
        // ---- phase A: fill the lists
        int nt_ = 0, nl_ = 0;
        while (u < M && nt_ < kListCap && nl_ < kListCap) {
          const double4 a = A.nc4[u];
          const int2 mu = A.meta[u];
          if (mu.y & kLeafFlag) {
            if (lane == 0) lf[nl_] = (int)u;
            ++nl_;
            partner += 1;
            u = u + 1;
          } else {
            const double dx = sx - a.x, dy = sy - a.y, dz = sz - a.z;
            const double d2 = (dx * dx + dy * dy) + dz * dz;
            const bool ok = !valid || (theta2 * d2 > s_bl2[mu.y & 0xff]);
            const unsigned fail = __ballot_sync(0xffffffffu, !ok);
            const int first_fail = fail ? __ffs(fail) - 1 : 32;
            if (valid && lane <= first_fail) ++c_mac;
            if (fail == 0) {
              if (lane == 0) tw[nt_] = (int)u;
              ++nt_;
              partner += A.nleaves[u];
              u = (unsigned)mu.x;
            } else {
              u = u + 1;
            }
          }
        }
        __syncwarp();
        W += (double)(nt_ + nl_);
        // ---- phase B: twigs
        for (int base = 0; base < nt_; base += 32) {
          const int k = base + lane;
          if (k < nt_) {
            const int nd = tw[k];
            const double4 a = A.nc4[nd];
            Staged sv;
            sv.cx = a.x; sv.cy = a.y; sv.cz = a.z; sv.q = a.w;
            sv.m0 = A.mom32[3 * (int64_t)nd];
            sv.m1 = A.mom32[3 * (int64_t)nd + 1];
            sv.m2 = A.mom32[3 * (int64_t)nd + 2];
            st[lane] = sv;
          }
          __syncwarp();
          const int cntb = min(32, nt_ - base);
          float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
          if (valid) {
            for (int j = 0; j < cntb; ++j) {
              const double cx = st[j].cx, cy = st[j].cy, cz = st[j].cz;
              const float dx = (float)(sx - cx), dy = (float)(sy - cy), dz = (float)(sz - cz);
              twig32(st[j].m0, st[j].m1, st[j].m2, dx, dy, dz, A.eps2, ax, ay, az, ap);
            }
            c_twig += (unsigned)cntb;
          }
          E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
          __syncwarp();
        }
        // ---- phase B: leaves
        for (int base = 0; base < nl_; base += 32) {
          const int k = base + lane;
          if (k < nl_) {
            const double4 a = A.nc4[lf[k]];
            st[lane].cx = a.x; st[lane].cy = a.y; st[lane].cz = a.z; st[lane].q = a.w;
          }
          __syncwarp();
          const int cntb = min(32, nl_ - base);
          float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
          if (valid) {
            for (int j = 0; j < cntb; ++j) {
              const double dx64 = sx - st[j].cx, dy64 = sy - st[j].cy, dz64 = sz - st[j].cz;
              if (dx64 == 0.0 && dy64 == 0.0 && dz64 == 0.0) continue;  // self
              leaf32((float)st[j].q, (float)dx64, (float)dy64, (float)dz64, A.eps2, ax, ay, az, ap);
              ++c_leaf;
            }
          }
          E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
          __syncwarp();
        }
      }
      if (partner != A.npart) complete = false;
    }
    if (valid) {
      A.ex[t] = E0; A.ey[t] = E1; A.ez[t] = E2; A.pot[t] = PH; A.work[t] = W;
    }
    if (!complete && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  warp_add3(A.counters, c_leaf, c_twig, c_mac);
}

// Group walk with a wide traversal (the default GROUP kernel).
// The warp's 32 targets form the group; the traversal pops up to 32 nodes
// from a per-warp LIFO stack (global memory) and lane k decides node k:
//   leaf   -> queued for direct evaluation,
//   twig   -> accepted if every target of the group passes the Barnes-Hut MAC
//             (module_tree_walk_simple.f90:343-382 semantics), else its
//             children (child8 table) are pushed.
// The MAC uses the targets' offsets from the group centre in FP32; a bounding
// sphere of the group gives a quick accept / quick open before the per-target
// loop.  Queued twigs and leaves are evaluated 32 at a time from a shared
// staging area (lane k loads node k, then every lane reads all of them), so
// node loads never sit on the per-interaction dependency chain.
// Stack bound: a pop takes <= 32 entries and pushes <= 8 per node, so the
// stack never holds more than (kMaxLevel + 1) * 8 * 32 entries; kStackCap
// leaves a margin and an overflow sets ST_INCOMPLETE instead of writing past it.
constexpr int kStackCap = 8192;
constexpr int kWW = kMixThreads / 32;  // warps per block

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int& total) {
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

__global__ void __launch_bounds__(kMixThreads) k_walk_group_wide(MixArgs A, int* __restrict__ gstack,
                                                                 const int4* __restrict__ child8,
                                                                 const int* __restrict__ nchild) {
  __shared__ float s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  __shared__ float4 s_t[kWW][32];
  __shared__ int s_tw[kWW][64];
  __shared__ int s_lf[kWW][64];
  __shared__ Staged s_st[kWW][32];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = (float)A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int* stack = gstack + (int64_t)(blockIdx.x * kWW + w) * kStackCap;
  float4* tt = s_t[w];
  int* tw = s_tw[w];
  int* lf = s_lf[w];
  Staged* st = s_st[w];
  const float theta2 = A.theta2;
  const int64_t nbuckets = A.tiles ? A.ntiles : (A.nt + 31) / 32;
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(&g_bucket_counter_mixed, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b >= nbuckets) break;
    int64_t t0;
    int cnt;
    if (A.tiles) {
      const int2 tl = A.tiles[b];
      t0 = tl.x;
      cnt = tl.y;
    } else {
      t0 = (int64_t)b * 32;
      cnt = (int)min((int64_t)32, A.nt - t0);
    }
    const bool valid = lane < cnt;
    const int64_t t = t0 + lane;
    double px = 0, py = 0, pz = 0;
    double E0 = 0, E1 = 0, E2 = 0, PH = 0, W = 0;
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      E0 = A.ex[t]; E1 = A.ey[t]; E2 = A.ez[t]; PH = A.pot[t]; W = A.work[t];
    }
    // group centre (FP64) and the targets' offsets from it (FP32)
    double lo[3] = {valid ? px : INFINITY, valid ? py : INFINITY, valid ? pz : INFINITY};
    double hi[3] = {valid ? px : -INFINITY, valid ? py : -INFINITY, valid ? pz : -INFINITY};
#pragma unroll
    for (int d = 0; d < 3; ++d)
      for (int o = 16; o > 0; o >>= 1) {
        lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
        hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
      }
    const double g0x = 0.5 * (lo[0] + hi[0]), g0y = 0.5 * (lo[1] + hi[1]), g0z = 0.5 * (lo[2] + hi[2]);
    const float rx = (float)(px - g0x), ry = (float)(py - g0y), rz = (float)(pz - g0z);
    float rg = valid ? sqrtf(rx * rx + ry * ry + rz * rz) : 0.f;
    for (int o = 16; o > 0; o >>= 1) rg = fmaxf(rg, __shfl_xor_sync(0xffffffffu, rg, o));
    rg = rg * 1.0001f + 1e-30f;  // the sphere must contain every target after rounding
    tt[lane] = make_float4(rx, ry, rz, valid ? 1.f : 0.f);
    __syncwarp();
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double vx = s_vb[3 * ib], vy = s_vb[3 * ib + 1], vz = s_vb[3 * ib + 2];
      const double sx = px - vx, sy = py - vy, sz = pz - vz;
      const double gx = g0x - vx, gy = g0y - vy, gz = g0z - vz;
      int64_t partner = 0;
      int nT = 0, nL = 0;
      int top = 1;
      if (lane == 0) stack[0] = 0;  // the root (walk_simple starts at the root, :286)
      __syncwarp();
      // evaluates the first n queued twigs / leaves and removes them
      auto flush_twigs = [&](int n) {
        if (lane < n) {
          const int nd = tw[lane];
          const double4 a = A.nc4[nd];
          Staged sv;
          sv.cx = a.x; sv.cy = a.y; sv.cz = a.z; sv.q = a.w;
          sv.m0 = A.mom32[3 * (int64_t)nd];
          sv.m1 = A.mom32[3 * (int64_t)nd + 1];
          sv.m2 = A.mom32[3 * (int64_t)nd + 2];
          st[lane] = sv;
        }
        __syncwarp();
        if (valid) {
          float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
          for (int j = 0; j < n; ++j) {
            const float dx = (float)(sx - st[j].cx), dy = (float)(sy - st[j].cy),
                        dz = (float)(sz - st[j].cz);
            twig32(st[j].m0, st[j].m1, st[j].m2, dx, dy, dz, A.eps2, ax, ay, az, ap);
          }
          E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
          c_twig += (unsigned)n;
        }
        W += (double)n;
        __syncwarp();
        if (lane + n < nT) tw[lane] = tw[lane + n];
        nT -= n;
        __syncwarp();
      };
      auto flush_leaves = [&](int n) {
        if (lane < n) {
          const double4 a = A.nc4[lf[lane]];
          st[lane].cx = a.x; st[lane].cy = a.y; st[lane].cz = a.z; st[lane].q = a.w;
        }
        __syncwarp();
        if (valid) {
          float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
          for (int j = 0; j < n; ++j) {
            const double dx64 = sx - st[j].cx, dy64 = sy - st[j].cy, dz64 = sz - st[j].cz;
            if (dx64 == 0.0 && dy64 == 0.0 && dz64 == 0.0) continue;  // self
            leaf32((float)st[j].q, (float)dx64, (float)dy64, (float)dz64, A.eps2, ax, ay, az, ap);
            ++c_leaf;
          }
          E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
        }
        W += (double)n;
        __syncwarp();
        if (lane + n < nL) lf[lane] = lf[lane + n];
        nL -= n;
        __syncwarp();
      };
      while (top > 0) {
        const int take = top < 32 ? top : 32;
        top -= take;
        const int node = lane < take ? stack[top + lane] : -1;
        __syncwarp();
        bool isleaf = false, accept = false, open = false;
        int nleaf_acc = 0;
        if (node >= 0) {
          const double4 a = A.nc4[node];
          const int2 mu = A.meta[node];
          if (mu.y & kLeafFlag) {
            isleaf = true;
          } else {
            const float cx = (float)(a.x - gx), cy = (float)(a.y - gy), cz = (float)(a.z - gz);
            const float bl = s_bl2[mu.y & 0xff];
            const float dc = sqrtf(cx * cx + cy * cy + cz * cz);
            const float dmin = dc - rg, dmax = dc + rg;
            if (dmin > 0.f && theta2 * (dmin * dmin) > bl) {
              accept = true;  // every target is farther than dmin
              c_mac += 1;
            } else if (!(theta2 * (dmax * dmax) > bl)) {
              open = true;    // no target can pass
              c_mac += 1;
            } else {
              accept = true;
              for (int j = 0; j < 32; ++j) {
                const float4 q4 = tt[j];
                if (q4.w == 0.f) continue;
                const float dx = q4.x - cx, dy = q4.y - cy, dz = q4.z - cz;
                ++c_mac;
                if (!(theta2 * fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > bl)) {
                  accept = false;
                  break;
                }
              }
              open = !accept;
            }
            if (accept) nleaf_acc = A.nleaves[node];
          }
        }
        const unsigned lb = __ballot_sync(0xffffffffu, isleaf);
        const unsigned ab = __ballot_sync(0xffffffffu, accept);
        if (isleaf) lf[nL + __popc(lb & lt)] = node;
        if (accept) tw[nT + __popc(ab & lt)] = node;
        nL += __popc(lb);
        nT += __popc(ab);
        int pl = nleaf_acc;
        for (int o = 16; o > 0; o >>= 1) pl += __shfl_xor_sync(0xffffffffu, pl, o);
        partner += (int64_t)pl + __popc(lb);
        // push the children of opened twigs
        const int nch = open ? min(8, nchild[node]) : 0;
        int total;
        const int off = warp_excl_scan(nch, lane, total);
        if (top + total > kStackCap) {
          complete = false;  // cannot happen within the bound above
          break;
        }
        if (nch > 0) {
          const int4 c0 = child8[2 * (int64_t)node], c1 = child8[2 * (int64_t)node + 1];
          const int cc[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
          for (int k = 0; k < nch; ++k) stack[top + off + k] = cc[k];
        }
        top += total;
        __syncwarp();
        if (nT >= 32) flush_twigs(32);
        if (nL >= 32) flush_leaves(32);
      }
      if (nT > 0) flush_twigs(nT);
      if (nL > 0) flush_leaves(nL);
      if (partner != A.npart) complete = false;
    }
    if (valid) {
      A.ex[t] = E0; A.ey[t] = E1; A.ez[t] = E2; A.pot[t] = PH; A.work[t] = W;
    }
    if (__any_sync(0xffffffffu, !complete) && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  warp_add3(A.counters, c_leaf, c_twig, c_mac);
}

// per-target semantics (module_tree_walk_pthreads.f90:558-765) with FP32
// interactions; the MAC is evaluated on the FP32 offsets
__global__ void __launch_bounds__(kMixThreads) k_walk_target_mixed(MixArgs A) {
  __shared__ float s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = (float)A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned M = (unsigned)A.M;
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(&g_bucket_counter_mixed, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b * 32 >= A.nt) break;
    const int64_t t = (int64_t)b * 32 + lane;
    const bool valid = t < A.nt;
    double px = 0, py = 0, pz = 0, E0 = 0, E1 = 0, E2 = 0, PH = 0, W = 0;
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      E0 = A.ex[t]; E1 = A.ey[t]; E2 = A.ez[t]; PH = A.pot[t]; W = A.work[t];
    }
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double sx = px - s_vb[3 * ib], sy = py - s_vb[3 * ib + 1], sz = pz - s_vb[3 * ib + 2];
      float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
      int steps = 0;
      unsigned next = valid ? 1u : M;
      int64_t partner = 0;
      for (;;) {
        const unsigned u = __reduce_min_sync(0xffffffffu, next);
        if (u >= M) break;
        if (next == u) {
          const double4 a = A.nc4[u];
          const int2 mu = A.meta[u];
          const double dx64 = sx - a.x, dy64 = sy - a.y, dz64 = sz - a.z;
          const float dx = (float)dx64, dy = (float)dy64, dz = (float)dz64;
          if (mu.y & kLeafFlag) {
            partner += 1;
            W += 1.0;
            if (!(dx64 == 0.0 && dy64 == 0.0 && dz64 == 0.0)) {
              leaf32((float)a.w, dx, dy, dz, A.eps2, ax, ay, az, ap);
              ++c_leaf;
            }
            next = u + 1;
          } else {
            ++c_mac;
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (A.theta2 * r2 > s_bl2[mu.y & 0xff]) {
              partner += A.nleaves[u];
              const float4 m0 = A.mom32[3 * (int64_t)u], m1 = A.mom32[3 * (int64_t)u + 1],
                           m2 = A.mom32[3 * (int64_t)u + 2];
              twig32(m0, m1, m2, dx, dy, dz, A.eps2, ax, ay, az, ap);
              ++c_twig;
              W += 1.0;
              next = (unsigned)mu.x;
            } else {
              next = u + 1;
            }
          }
          if (++steps == kChunk) {
            E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
            ax = ay = az = ap = 0.f;
            steps = 0;
          }
        }
      }
      E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
      if (valid && partner != A.npart) complete = false;
    }
    if (valid) {
      A.ex[t] = E0; A.ey[t] = E1; A.ez[t] = E2; A.pot[t] = PH; A.work[t] = W;
    }
    if (__any_sync(0xffffffffu, !complete) && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  warp_add3(A.counters, c_leaf, c_twig, c_mac);
}

__global__ void k_reset_mixed() { g_bucket_counter_mixed = 0; }

}  // namespace

int launch_walk_mixed(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                      double* ex, double* ey, double* ez, double* pot, double* work,
                      const int2* tiles, int64_t ntiles, bool per_target) {
  const int blocks = 148 * 8;
  MixArgs A;
  A.nt = nt;
  A.tx = tx; A.ty = ty; A.tz = tz;
  A.nc4 = c->nc4.p;
  A.meta = c->meta.p;
  A.mom32 = reinterpret_cast<const float4*>(c->mom32.p);
  A.nleaves = c->nleaves.p;
  A.bl2 = c->d_box + 9;
  A.vbox = c->d_vbox;
  A.nbox = c->nboxes;
  A.theta2 = (float)c->prm.theta2;
  A.theta2_64 = c->prm.theta2;
  A.eps2 = (float)c->prm.eps2;
  A.M = (int32_t)c->nnodes;
  A.npart = c->n;
  A.ex = ex; A.ey = ey; A.ez = ez; A.pot = pot; A.work = work;
  A.counters = c->counters.p;
  A.status = c->d_status;
  A.tiles = tiles;
  A.ntiles = ntiles;
  cudaStream_t s = c->stream;
  COUNT_LAUNCH();
  k_reset_mixed<<<1, 1, 0, s>>>();
  COUNT_LAUNCH();
  if (per_target) {
    k_walk_target_mixed<<<blocks, kMixThreads, 0, s>>>(A);
  } else if (c->prm.reserved[0] == 1) {
    k_walk_group_mixed<<<blocks, kMixThreads, 0, s>>>(A);
  } else if (c->prm.reserved[0] == 2) {
    k_walk_group_mixed_ab<<<blocks, kMixThreads, 0, s>>>(A);
  } else {
    if (!ensure(c, c->wstack, (size_t)blocks * kWW * kStackCap, "walk stacks")) return PEPCG_ERR_OOM;
    k_walk_group_wide<<<blocks, kMixThreads, 0, s>>>(A, c->wstack.p, c->child8.p, c->nchild.p);
  }
  return cuda_ok(c, cudaGetLastError(), "mixed walk launch") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

}  // namespace pepcg
