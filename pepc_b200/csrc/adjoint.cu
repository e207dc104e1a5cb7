// adjoint.cu -- the adjoint of the tree-code force evaluation: given dL/dE and
// dL/dphi at the targets, dL/dq and dL/dx of the sources.  The reference has
// no adjoint; the forward model is its walk (per-target semantics,
// module_tree_walk_pthreads.f90:558-765, or per-tile semantics,
// module_tree_walk_simple.f90:256-384) with the Coulomb kernels
// (module_coulomb_kernels.f90:60-145, :242-257) and the multipole
// construction (coulomb/module_interaction_specific.f90:84-140), with the
// interaction lists held fixed (the MAC and the keys are piecewise constant).
//
// Writing the twig potential as
//   phi = q D0 + p_k D1_k + sum_{kl in xx,yy,zz,xy,yz,zx} Q_kl D2_kl,
// D the Cartesian derivative tensors of 1/r with r^2 = |d|^2 + eps^2, one
// target-node pair (dL/dphi = gphi, dL/dE = gE) contributes
//   qbar += gphi D0 - gE.D1,   pbar_k += gphi D1_k - gE_i D2_ik,
//   Qbar_kl += gphi D2_kl - gE_i D3_ikl,   cocbar += gphi E + H gE,
// where E = -grad phi and H the Hessian of phi (D4 enters only through gE).
// Pass 1 (walk): the lists are recomputed exactly as in the forward walk;
//   the contributions of a warp's targets to a node are reduced across the
//   warp and added to the node's adjoint (14 doubles) with atomics.
// Pass 2 (top-down, one launch per level): the transpose of
//   shift_multipoles_up moves every twig's adjoint to its children,
//   including the dependence of the centre of charge on the children's
//   positions and abs_charge weights; a node has one parent, so no atomics.
// Pass 3: the leaves' adjoints become dL/dq (plus abs_charge adjoint times
//   sign(q)) and dL/dx in the caller's original particle order.
// Compiled with --fmad=false.

#include "internal.cuh"

namespace pepcg {

__device__ unsigned int g_bucket_counter_adj;

namespace {

constexpr int kAdjThreads = 128;
constexpr int kNA = 16;  // adjoint record: q, p(3), Q(6), coc(3), A, pad(2)

struct Tens {
  double d[3], R[5];
  __device__ __forceinline__ void set(double dx, double dy, double dz, double eps2) {
    d[0] = dx; d[1] = dy; d[2] = dz;
    const double r2 = ((dx * dx + dy * dy) + dz * dz) + eps2;
    const double r0 = 1.0 / sqrt(r2);
    const double r02 = r0 * r0;
    R[0] = r0;
    R[1] = R[0] * r02;
    R[2] = R[1] * r02;
    R[3] = R[2] * r02;
    R[4] = R[3] * r02;
  }
  __device__ __forceinline__ static double dl(int i, int j) { return i == j ? 1.0 : 0.0; }
  __device__ __forceinline__ double D1(int i) const { return -d[i] * R[1]; }
  __device__ __forceinline__ double D2(int i, int j) const {
    return 3.0 * d[i] * d[j] * R[2] - dl(i, j) * R[1];
  }
  __device__ __forceinline__ double D3(int i, int j, int k) const {
    return -15.0 * d[i] * d[j] * d[k] * R[3] +
           3.0 * R[2] * (dl(i, j) * d[k] + dl(i, k) * d[j] + dl(j, k) * d[i]);
  }
  __device__ __forceinline__ double D4(int i, int j, int k, int l) const {
    return 105.0 * d[i] * d[j] * d[k] * d[l] * R[4] -
           15.0 * R[3] *
               (dl(i, j) * d[k] * d[l] + dl(i, k) * d[j] * d[l] + dl(i, l) * d[j] * d[k] +
                dl(j, k) * d[i] * d[l] + dl(j, l) * d[i] * d[k] + dl(k, l) * d[i] * d[j]) +
           3.0 * R[2] * (dl(i, j) * dl(k, l) + dl(i, k) * dl(j, l) + dl(i, l) * dl(j, k));
  }
};

__constant__ int c_QK[6] = {0, 1, 2, 0, 1, 2};  // moment order xx yy zz xy yz zx
__constant__ int c_QL[6] = {0, 1, 2, 1, 2, 0};

// a[0] q, a[1..3] p, a[4..9] Q, a[10..12] coc, a[13] abs_charge
template <bool kWithE>
__device__ __forceinline__ void twig_adj(double q, const double* m, double dx, double dy,
                                         double dz, double eps2, double gphi, const double gE[3],
                                         double a[14]) {
  Tens T;
  T.set(dx, dy, dz, eps2);
  const double p[3] = {m[0], m[1], m[2]};
  const double Q[6] = {m[3], m[4], m[5], m[6], m[7], m[8]};
  a[0] += gphi * T.R[0];
  if (kWithE)
#pragma unroll
    for (int i = 0; i < 3; ++i) a[0] -= gE[i] * T.D1(i);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double v = gphi * T.D1(k);
    if (kWithE)
#pragma unroll
      for (int i = 0; i < 3; ++i) v -= gE[i] * T.D2(i, k);
    a[1 + k] += v;
  }
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    double v = gphi * T.D2(c_QK[s], c_QL[s]);
    if (kWithE)
#pragma unroll
      for (int i = 0; i < 3; ++i) v -= gE[i] * T.D3(i, c_QK[s], c_QL[s]);
    a[4 + s] += v;
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double E = q * T.D1(j);
#pragma unroll
    for (int k = 0; k < 3; ++k) E += p[k] * T.D2(j, k);
#pragma unroll
    for (int s = 0; s < 6; ++s) E += Q[s] * T.D3(j, c_QK[s], c_QL[s]);
    E = -E;
    double hg = 0.0;
    if (kWithE) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double H = q * T.D2(i, j);
#pragma unroll
        for (int k = 0; k < 3; ++k) H += p[k] * T.D3(i, j, k);
#pragma unroll
        for (int s = 0; s < 6; ++s) H += Q[s] * T.D4(i, j, c_QK[s], c_QL[s]);
        hg += H * gE[i];
      }
    }
    a[10 + j] += gphi * E + hg;
  }
}

__device__ __forceinline__ void leaf_adj(double q, double dx, double dy, double dz, double eps2,
                                         double gphi, const double gE[3], double a[14]) {
  Tens T;
  T.set(dx, dy, dz, eps2);
  a[0] += gphi * T.R[0];
#pragma unroll
  for (int i = 0; i < 3; ++i) a[0] -= gE[i] * T.D1(i);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double E = -q * T.D1(j);
    double hg = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) hg += q * T.D2(i, j) * gE[i];
    a[10 + j] += gphi * E + hg;
  }
}

// warp-reduce the lanes' contributions and add them to the node's adjoint
__device__ __forceinline__ void flush_node(double* __restrict__ adj, unsigned u, double a[14],
                                           int lane) {
#pragma unroll
  for (int k = 0; k < 14; ++k) {
    double v = a[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0 && v != 0.0) atomicAdd(&adj[(int64_t)kNA * u + k], v);
    a[k] = 0.0;
  }
}

struct AdjArgs {
  int64_t nt;
  const double* tx;
  const double* ty;
  const double* tz;
  const double* gex;
  const double* gey;
  const double* gez;
  const double* gphi;
  const double4* nc4;
  const int2* meta;
  const int2* fwd;
  const double* mom;
  const double* bl2;
  const double* vbox;
  int nbox;
  double theta2, eps2;
  int32_t M;
  double* adj;
  const int2* tiles;  // per tile: (first, count); nullptr: per-target semantics
  int64_t ntiles;
};

// per-target semantics: the min-next-index schedule of k_walk_target64
template <bool kWithE>
__global__ void __launch_bounds__(kAdjThreads) k_adj_target(AdjArgs A) {
  __shared__ double s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned M = (unsigned)A.M;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(&g_bucket_counter_adj, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b * 32 >= A.nt) break;
    const int64_t t = (int64_t)b * 32 + lane;
    const bool valid = t < A.nt;
    double px = 0, py = 0, pz = 0, gp = 0, gE[3] = {0, 0, 0};
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      gp = A.gphi[t];
      gE[0] = A.gex[t]; gE[1] = A.gey[t]; gE[2] = A.gez[t];
    }
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double sx = px - s_vb[3 * ib], sy = py - s_vb[3 * ib + 1], sz = pz - s_vb[3 * ib + 2];
      unsigned next = valid ? 1u : M;
      double a[14];
#pragma unroll
      for (int k = 0; k < 14; ++k) a[k] = 0.0;
      for (;;) {
        const unsigned u = __reduce_min_sync(0xffffffffu, next);
        if (u >= M) break;
        const double4 nd = A.nc4[u];
        const int2 mu = A.meta[u];
        if (next == u) {
          const double dx = sx - nd.x, dy = sy - nd.y, dz = sz - nd.z;
          const double dist2 = (dx * dx + dy * dy) + dz * dz;
          if (mu.y & kLeafFlag) {
            if (dist2 > 0.0) leaf_adj(nd.w, dx, dy, dz, A.eps2, gp, gE, a);
            next = u + 1;
          } else if (A.theta2 * dist2 > s_bl2[mu.y & 0xff]) {
            double m[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) m[k] = A.mom[9 * (int64_t)u + k];
            twig_adj<kWithE>(nd.w, m, dx, dy, dz, A.eps2, gp, gE, a);
            next = (unsigned)mu.x;
          } else {
            next = u + 1;
          }
        }
        flush_node(A.adj, u, a, lane);
      }
    }
  }
}

// per-tile / group semantics: the warp's targets share every node; a twig is
// accepted if all of them pass the MAC (module_tree_walk_simple.f90:343-382)
template <bool kWithE>
__global__ void __launch_bounds__(kAdjThreads) k_adj_group(AdjArgs A) {
  __shared__ double s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned M = (unsigned)A.M;
  const int64_t nbk = A.ntiles;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(&g_bucket_counter_adj, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b >= nbk) break;
    const int2 tl = A.tiles[b];
    const bool valid = lane < tl.y;
    const int64_t t = (int64_t)tl.x + lane;
    double px = 0, py = 0, pz = 0, gp = 0, gE[3] = {0, 0, 0};
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      gp = A.gphi[t];
      gE[0] = A.gex[t]; gE[1] = A.gey[t]; gE[2] = A.gez[t];
    }
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double vx = s_vb[3 * ib], vy = s_vb[3 * ib + 1], vz = s_vb[3 * ib + 2];
      double a[14];
#pragma unroll
      for (int k = 0; k < 14; ++k) a[k] = 0.0;
      unsigned u = 0;
      while (u < M) {
        const double4 nd = A.nc4[u];
        const int2 mu = A.meta[u];
        const int2 fw = A.fwd[u];
        const double dx = (px - vx) - nd.x, dy = (py - vy) - nd.y, dz = (pz - vz) - nd.z;
        const double dist2 = (dx * dx + dy * dy) + dz * dz;
        if (mu.y & kLeafFlag) {
          if (valid && dist2 > 0.0) leaf_adj(nd.w, dx, dy, dz, A.eps2, gp, gE, a);
          flush_node(A.adj, u, a, lane);
          u = (unsigned)fw.y;
        } else {
          const bool ok = !valid || (A.theta2 * dist2 > s_bl2[mu.y & 0xff]);
          if (__all_sync(0xffffffffu, ok)) {
            if (valid) {
              double m[9];
#pragma unroll
              for (int k = 0; k < 9; ++k) m[k] = A.mom[9 * (int64_t)u + k];
              twig_adj<kWithE>(nd.w, m, dx, dy, dz, A.eps2, gp, gE, a);
            }
            flush_node(A.adj, u, a, lane);
            u = (unsigned)fw.y;
          } else {
            u = (unsigned)fw.x;
          }
        }
      }
    }
  }
}

// transpose of shift_multipoles_up for the twigs of one level (top-down)
__global__ void k_adj_down_level(int64_t M, int level, const int2* __restrict__ meta,
                                 const double4* __restrict__ nc4, const double* __restrict__ mom,
                                 const double2* __restrict__ aux, double* __restrict__ adj) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < M;
       u += (int64_t)gridDim.x * blockDim.x) {
    const int2 mu = meta[u];
    if ((mu.y & kLeafFlag) || (mu.y & 0xff) != level) continue;
    const double4 pc = nc4[u];
    const double A = aux[u].x;
    const double* pa = adj + kNA * u;
    const double Pq = pa[0];
    const double Pp[3] = {pa[1], pa[2], pa[3]};
    const double PQ[6] = {pa[4], pa[5], pa[6], pa[7], pa[8], pa[9]};
    double cocbar[3] = {pa[10], pa[11], pa[12]};
    const double PA = pa[13];
    int64_t ch[8];
    int nc = 0;
    for (int64_t c = u + 1; c < mu.x && nc < 8; c = meta[c].x) ch[nc++] = c;
    // first pass: everything except the centre-of-charge chain rule
    for (int k = 0; k < nc; ++k) {
      const int64_t c = ch[k];
      const double4 cc = nc4[c];
      const bool leafc = (meta[c].y & kLeafFlag) != 0;
      double pcv[3] = {0, 0, 0};
      if (!leafc)
        for (int i = 0; i < 3; ++i) pcv[i] = mom[9 * c + i];
      const double qc = cc.w;
      const double sc[3] = {pc.x - cc.x, pc.y - cc.y, pc.z - cc.z};
      double sbar[3] = {0, 0, 0};
      for (int i = 0; i < 3; ++i) sbar[i] += Pp[i] * qc;
      for (int i = 0; i < 3; ++i) sbar[i] += PQ[i] * (pcv[i] + qc * sc[i]);
      sbar[0] += PQ[3] * (pcv[1] + qc * sc[1]); sbar[1] += PQ[3] * (pcv[0] + qc * sc[0]);
      sbar[1] += PQ[4] * (pcv[2] + qc * sc[2]); sbar[2] += PQ[4] * (pcv[1] + qc * sc[1]);
      sbar[2] += PQ[5] * (pcv[0] + qc * sc[0]); sbar[0] += PQ[5] * (pcv[2] + qc * sc[2]);
      double* a = adj + kNA * c;
      double aq = Pq;
      for (int i = 0; i < 3; ++i) aq += Pp[i] * sc[i] + PQ[i] * 0.5 * sc[i] * sc[i];
      aq += PQ[3] * sc[0] * sc[1] + PQ[4] * sc[1] * sc[2] + PQ[5] * sc[2] * sc[0];
      a[0] += aq;
      a[1] += Pp[0] + PQ[0] * sc[0] + PQ[3] * sc[1] + PQ[5] * sc[2];
      a[2] += Pp[1] + PQ[1] * sc[1] + PQ[3] * sc[0] + PQ[4] * sc[2];
      a[3] += Pp[2] + PQ[2] * sc[2] + PQ[4] * sc[1] + PQ[5] * sc[0];
      for (int s = 0; s < 6; ++s) a[4 + s] += PQ[s];
      for (int i = 0; i < 3; ++i) {
        a[10 + i] -= sbar[i];
        cocbar[i] += sbar[i];
      }
      a[13] += PA;
    }
    // second pass: coc = sum coc_c A_c / A (or the plain mean when A = 0)
    for (int k = 0; k < nc; ++k) {
      const int64_t c = ch[k];
      const double4 cc = nc4[c];
      const bool leafc = (meta[c].y & kLeafFlag) != 0;
      double* a = adj + kNA * c;
      if (A != 0.0) {
        const double Ac = leafc ? fabs(cc.w) : aux[c].x;
        const double w = Ac / A;
        const double cv[3] = {cc.x, cc.y, cc.z};
        const double pv[3] = {pc.x, pc.y, pc.z};
        double g = 0.0;
        for (int i = 0; i < 3; ++i) {
          a[10 + i] += cocbar[i] * w;
          g += cocbar[i] * (cv[i] - pv[i]);
        }
        a[13] += g / A;
      } else {
        for (int i = 0; i < 3; ++i) a[10 + i] += cocbar[i] / (double)nc;
      }
    }
  }
}

// leaves -> particles in the caller's original order
__global__ void k_adj_out(int64_t n, const int32_t* __restrict__ leafnode,
                          const int32_t* __restrict__ perm, const double* __restrict__ q,
                          const double* __restrict__ adj, double* dq, double* dx, double* dy,
                          double* dz) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double* a = adj + (int64_t)kNA * leafnode[i];
    const int64_t o = perm[i];
    const double sg = (double)((q[i] > 0.0) - (q[i] < 0.0));
    dq[o] = a[0] + a[13] * sg;
    dx[o] = a[10];
    dy[o] = a[11];
    dz[o] = a[12];
  }
}

__global__ void k_reset_adj() { g_bucket_counter_adj = 0; }

__global__ void k_any_nonzero(int64_t n, const double* a, const double* b, const double* c,
                              unsigned int* flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (a[i] != 0.0 || b[i] != 0.0 || c[i] != 0.0) atomicOr(flag, 1u);
}

__global__ void k_buckets32(int64_t nt, int2* tiles) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b * 32 < nt;
       b += (int64_t)gridDim.x * blockDim.x)
    tiles[b] = make_int2((int)(b * 32), (int)min((int64_t)32, nt - b * 32));
}

}  // namespace

int adjoint_device(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                   const double* gex, const double* gey, const double* gez, const double* gphi,
                   double* dq, double* dx, double* dy, double* dz) {
  if (!c->has_tree) {
    c->err = "adjoint called without a grown tree";
    return PEPCG_ERR_NO_TREE;
  }
  if (c->far_field) {
    c->err = "adjoint of the periodic far-lattice term is not implemented";
    return PEPCG_ERR_UNSUPPORTED;
  }
  cudaStream_t s = c->stream;
  const int64_t M = c->nnodes;
  if (!ensure(c, c->adj, (size_t)kNA * M, "adjoint")) return PEPCG_ERR_OOM;
  if (!cuda_ok(c, cudaMemsetAsync(c->adj.p, 0, sizeof(double) * kNA * M, s), "adjoint"))
    return PEPCG_ERR_CUDA;
  // is dL/dE zero everywhere?  (then the Hessian terms are skipped)
  unsigned int* d_flag = reinterpret_cast<unsigned int*>(c->d_small + 6);
  unsigned int h_flag = 1;
  cudaMemsetAsync(d_flag, 0, 4, s);
  COUNT_LAUNCH();
  k_any_nonzero<<<148, 256, 0, s>>>(nt, gex, gey, gez, d_flag);
  AdjArgs A;
  A.nt = nt;
  A.tx = tx; A.ty = ty; A.tz = tz;
  A.gex = gex; A.gey = gey; A.gez = gez; A.gphi = gphi;
  A.nc4 = c->nc4.p;
  A.meta = c->meta.p;
  A.fwd = c->fwd.p;
  A.mom = c->mom.p;
  A.bl2 = c->d_box + 9;
  A.vbox = c->d_vbox;
  A.nbox = c->nboxes;
  A.theta2 = c->prm.theta2;
  A.eps2 = c->prm.eps2;
  A.M = (int32_t)M;
  A.adj = c->adj.p;
  A.tiles = nullptr;
  A.ntiles = 0;
  const bool per_target = (c->prm.walk == PEPCG_WALK_PER_TARGET);
  if (!per_target) {
    // the same tiles as the forward walk of these targets
    if (!ensure(c, c->tiles, 2 * (nt + 32), "tiles")) return PEPCG_ERR_OOM;
    int2* d_tiles = reinterpret_cast<int2*>(c->tiles.p);
    int64_t ntiles = 0;
    if (c->prm.walk == PEPCG_WALK_GROUP) {
      ntiles = (nt + 31) / 32;
      COUNT_LAUNCH();
      k_buckets32<<<148, 256, 0, s>>>(nt, d_tiles);
    } else {
      const int T = c->prm.tile_size;
      int rc = host_tiles(c, nt, nullptr, T, d_tiles, &ntiles);
      if (rc) return rc;
    }
    A.tiles = d_tiles;
    A.ntiles = ntiles;
  }
  if (!cuda_ok(c, cudaMemcpyAsync(&h_flag, d_flag, 4, cudaMemcpyDeviceToHost, s), "flag") ||
      !cuda_ok(c, cudaStreamSynchronize(s), "flag"))
    return PEPCG_ERR_CUDA;
  COUNT_LAUNCH();
  k_reset_adj<<<1, 1, 0, s>>>();
  COUNT_LAUNCH();
  const int blocks = 148 * 8;
  if (per_target) {
    if (h_flag) k_adj_target<true><<<blocks, kAdjThreads, 0, s>>>(A);
    else k_adj_target<false><<<blocks, kAdjThreads, 0, s>>>(A);
  } else {
    if (h_flag) k_adj_group<true><<<blocks, kAdjThreads, 0, s>>>(A);
    else k_adj_group<false><<<blocks, kAdjThreads, 0, s>>>(A);
  }
  const unsigned g = (unsigned)((M + 255) / 256 > 148 * 16 ? 148 * 16 : (M + 255) / 256);
  for (int L = 0; L < c->max_level; ++L) {
    COUNT_LAUNCH();
    k_adj_down_level<<<g, 256, 0, s>>>(M, L, c->meta.p, c->nc4.p, c->mom.p, c->aux.p, c->adj.p);
  }
  COUNT_LAUNCH();
  k_adj_out<<<g, 256, 0, s>>>(c->n, c->leafnode.p, c->perm.p, c->q.p, c->adj.p, dq, dx, dy, dz);
  return cuda_ok(c, cudaGetLastError(), "adjoint") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

}  // namespace pepcg
