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
  if (per_target)
    k_walk_target_mixed<<<148 * 8, kMixThreads, 0, s>>>(A);
  else
    k_walk_group_mixed<<<148 * 8, kMixThreads, 0, s>>>(A);
  return cuda_ok(c, cudaGetLastError(), "mixed walk launch") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

}  // namespace pepcg
