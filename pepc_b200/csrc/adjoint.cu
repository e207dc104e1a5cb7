// adjoint.cu -- the adjoint of the tree-code force evaluation: given dL/dE and
// dL/dphi at the targets, dL/dq and dL/dx of the sources.  The reference has
// no adjoint; the forward model is its walk (per-target semantics,
// module_tree_walk_pthreads.f90:558-765, or per-tile semantics,
// module_tree_walk_simple.f90:256-384) with the Coulomb kernels
// (module_coulomb_kernels.f90:60-145, :242-257) and the multipole
// construction (coulomb/module_interaction_specific.f90:84-140), with the
// interaction lists held fixed (the MAC and the keys are piecewise constant).
//
// Pass 1 (walk): the lists are recomputed exactly as in the forward walk;
//   each target-node pair contributes to the node's adjoint record
//   (q, p, Q, coc, abs_charge); the contributions of a warp's targets to a
//   node are reduced across the warp and added with FP64 atomics.
// Pass 2 (top-down, one launch per level): the transpose of
//   shift_multipoles_up moves every twig's adjoint to its children,
//   including the dependence of the centre of charge on the children's
//   positions and abs_charge weights; a node has one parent, so no atomics.
// Pass 3: the leaves' adjoints become dL/dq (plus abs_charge adjoint times
//   sign(q)) and dL/dx in the caller's original particle order.

#include <algorithm>

#include "internal.cuh"

namespace pepcg {

namespace {

constexpr int kAdjThreads = 128;
constexpr int kNA = 16;  // adjoint record: q, p(3), Q(6), coc(3), A, pad(2)
// per-target walk: up to this many contributing lanes add their records directly
constexpr int kDirectLanes = 2;

// Closed forms of the contractions.  With r^2 = |d|^2 + eps^2 and
// R_n = r^-(2n+1), the derivative tensors of 1/r are
//   D1_i = -d_i R1,   D2_ij = 3 d_i d_j R2 - delta_ij R1,
//   D3_ijk = -15 d_i d_j d_k R3 + 3 R2 (delta_ij d_k + delta_ik d_j + delta_jk d_i),
//   D4_ijkl = 105 d_i d_j d_k d_l R4 - 15 R3 (six delta d d terms) + 3 R2 (three delta delta terms).
// The twig potential is phi = q R0 + p.D1 + M:D2 with M the quadrupole
// matrix (diagonal qxx qyy qzz, off-diagonal halves of qxy qyz qzx), so with
// g = dL/dE, a = g.d, pd = p.d, dMd = d.M.d, tr = trace M:
//   qbar  += gphi R0 + a R1
//   pbar  += -gphi R1 d - 3 a R2 d + R1 g
//   Mbar  += gphi D2 + 15 a R3 d d^T - 3 R2 (g d^T + d g^T + a I)
//   cocbar += gphi E + H g, with E = -grad phi the forward field and
//   H g = q (3 a R2 d - R1 g)
//       + 3 R2 (pd g + (g.p) d + a p) - 15 a pd R3 d
//       + 105 R4 a dMd d - 15 R3 (dMd g + 2 (g.M.d) d + 2 a M d + a tr d) + 3 R2 (tr g + 2 M g).
// The stored quadrupole slots take dphi/dq_kl = D2_kl (an off-diagonal
// q_kl = 2 M_kl enters twice through M).
// a[0] q, a[1..3] p, a[4..9] Q (xx yy zz xy yz zx), a[10..12] coc, a[13] abs_charge
template <bool kWithE>
__host__ __device__ __forceinline__ void twig_adj(double q, const double* m, double dx, double dy,
                                                  double dz, double eps2, double gphi,
                                                  const double gE[3], double a[14]) {
  const double r2 = ((dx * dx + dy * dy) + dz * dz) + eps2;
  const double R0 = 1.0 / sqrt(r2);
  const double i2 = R0 * R0;
  const double R1 = R0 * i2, R2 = R1 * i2, R3 = R2 * i2;
  const double d[3] = {dx, dy, dz};
  const double p[3] = {m[0], m[1], m[2]};
  const double Mx[3] = {m[3], 0.5 * m[6], 0.5 * m[8]};
  const double My[3] = {0.5 * m[6], m[4], 0.5 * m[7]};
  const double Mz[3] = {0.5 * m[8], 0.5 * m[7], m[5]};
  const double Md[3] = {Mx[0] * dx + Mx[1] * dy + Mx[2] * dz, My[0] * dx + My[1] * dy + My[2] * dz,
                        Mz[0] * dx + Mz[1] * dy + Mz[2] * dz};
  const double dMd = dx * Md[0] + dy * Md[1] + dz * Md[2];
  const double tr = m[3] + m[4] + m[5];
  const double pd = p[0] * dx + p[1] * dy + p[2] * dz;
  // forward field E = d [q R1 - 3 pd R2 + 15 dMd R3 - 3 tr R2] + p R1 - 6 R2 M d
  const double ce = q * R1 - 3.0 * pd * R2 + 15.0 * dMd * R3 - 3.0 * tr * R2;
  a[0] += gphi * R0;
#pragma unroll
  for (int k = 0; k < 3; ++k) a[1 + k] -= gphi * R1 * d[k];
  a[4] += gphi * (3.0 * dx * dx * R2 - R1);
  a[5] += gphi * (3.0 * dy * dy * R2 - R1);
  a[6] += gphi * (3.0 * dz * dz * R2 - R1);
  a[7] += gphi * (3.0 * dx * dy * R2);
  a[8] += gphi * (3.0 * dy * dz * R2);
  a[9] += gphi * (3.0 * dz * dx * R2);
#pragma unroll
  for (int j = 0; j < 3; ++j) a[10 + j] += gphi * (ce * d[j] + p[j] * R1 - 6.0 * R2 * Md[j]);
  if (kWithE) {
    const double R4 = R3 * i2;
    const double g[3] = {gE[0], gE[1], gE[2]};
    const double ga = g[0] * dx + g[1] * dy + g[2] * dz;
    const double gp = g[0] * p[0] + g[1] * p[1] + g[2] * p[2];
    const double Mg[3] = {Mx[0] * g[0] + Mx[1] * g[1] + Mx[2] * g[2],
                          My[0] * g[0] + My[1] * g[1] + My[2] * g[2],
                          Mz[0] * g[0] + Mz[1] * g[1] + Mz[2] * g[2]};
    const double gMd = g[0] * Md[0] + g[1] * Md[1] + g[2] * Md[2];
    a[0] += ga * R1;
#pragma unroll
    for (int k = 0; k < 3; ++k) a[1 + k] += R1 * g[k] - 3.0 * ga * R2 * d[k];
    // -g_i D3_ikl = 15 a R3 d_k d_l - 3 R2 (g_k d_l + g_l d_k + delta_kl a)
    const double a15 = 15.0 * ga * R3, r3 = 3.0 * R2;
    a[4] += a15 * dx * dx - r3 * (2.0 * g[0] * dx + ga);
    a[5] += a15 * dy * dy - r3 * (2.0 * g[1] * dy + ga);
    a[6] += a15 * dz * dz - r3 * (2.0 * g[2] * dz + ga);
    a[7] += a15 * dx * dy - r3 * (g[0] * dy + g[1] * dx);
    a[8] += a15 * dy * dz - r3 * (g[1] * dz + g[2] * dy);
    a[9] += a15 * dz * dx - r3 * (g[2] * dx + g[0] * dz);
    const double cd = 3.0 * q * ga * R2 - 15.0 * ga * pd * R3 + r3 * gp + 105.0 * R4 * ga * dMd -
                      15.0 * R3 * (2.0 * gMd + ga * tr);
    const double cg = -q * R1 + r3 * pd - 15.0 * R3 * dMd + r3 * tr;
#pragma unroll
    for (int j = 0; j < 3; ++j)
      a[10 + j] += cd * d[j] + cg * g[j] + r3 * ga * p[j] - 30.0 * R3 * ga * Md[j] + 6.0 * R2 * Mg[j];
  }
}

__host__ __device__ __forceinline__ void leaf_adj(double q, double dx, double dy, double dz,
                                                  double eps2, double gphi, const double gE[3],
                                                  double a[14]) {
  const double r2 = ((dx * dx + dy * dy) + dz * dz) + eps2;
  const double R0 = 1.0 / sqrt(r2);
  const double R1 = R0 * R0 * R0, R2 = R1 * R0 * R0;
  const double ga = gE[0] * dx + gE[1] * dy + gE[2] * dz;
  a[0] += gphi * R0 + ga * R1;
  const double cd = q * (gphi * R1 + 3.0 * ga * R2);
  a[10] += cd * dx - q * R1 * gE[0];
  a[11] += cd * dy - q * R1 * gE[1];
  a[12] += cd * dz - q * R1 * gE[2];
}

// The adjoint of one interaction for force_law 2 (2D Coulomb) and 4
// (Lennard-Jones), from the forward kernels themselves (law_leaf64 /
// law_twig64's calls): the 2D fields are linear in the node's charge and
// moments, so dL/dq and dL/dm are L of the unit moments (the Lennard-Jones
// fields depend on neither); dL/d(offset) comes from one evaluation on D3
// offsets (forward-mode derivatives along x, y, z) with the node's own
// charge and moments.  The offset is target minus node centre, so the centre's
// adjoint takes the negative.  FP64 throughout.
template <int kLaw>
__device__ __forceinline__ void law_adj(bool leaf, double q, const double* m, double dx, double dy,
                                        double dz, double eps2, double gphi, const double gE[3],
                                        double a[14]) {
  auto L = [&](double qq, const double* mm) {
    double ex, ey, ez, ph;
    if (leaf) {
      force_leaf_2d64(qq, dx, dy, (dx * dx + dy * dy) + eps2, ex, ey, ez, ph);
    } else {
      force_twig_2d64(qq, mm, dx, dy, (dx * dx + dy * dy) + eps2, ex, ey, ez, ph);
    }
    return gphi * ph + ((gE[0] * ex + gE[1] * ey) + gE[2] * ez);
  };
  if (kLaw == 2) {
    double u[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    a[0] += L(1.0, u);
    if (!leaf) {
      // only the moments the 2D kernel reads: p_x, p_y, q_xx, q_yy, q_xy
      const int used[5] = {0, 1, 3, 4, 6};
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        u[used[k]] = 1.0;
        a[1 + used[k]] += L(0.0, u);
        u[used[k]] = 0.0;
      }
    }
  }
  const D3 X(dx, 1.0, 0.0, 0.0), Y(dy, 0.0, 1.0, 0.0), Z(dz, 0.0, 0.0, 1.0);
  D3 ex, ey, ez, ph;
  if (kLaw == 2) {
    if (leaf) force_leaf_2d64(q, X, Y, (X * X + Y * Y) + eps2, ex, ey, ez, ph);
    else force_twig_2d64(q, m, X, Y, (X * X + Y * Y) + eps2, ex, ey, ez, ph);
  } else {
    force_lj64(X, Y, Z, (X * X + Y * Y) + Z * Z, eps2, ex, ey, ez, ph);
  }
#pragma unroll
  for (int j = 0; j < 3; ++j)
    a[10 + j] -= gphi * ph.g[j] + ((gE[0] * ex.g[j] + gE[1] * ey.g[j]) + gE[2] * ez.g[j]);
}

// the interaction adjoints of force law kLaw (3: the closed forms above)
template <bool kWithE, int kLaw>
__device__ __forceinline__ void twig_adj_law(double q, const double* m, double dx, double dy,
                                             double dz, double eps2, double gphi,
                                             const double gE[3], double a[14]) {
  if constexpr (kLaw == 3) twig_adj<kWithE>(q, m, dx, dy, dz, eps2, gphi, gE, a);
  else law_adj<kLaw>(false, q, m, dx, dy, dz, eps2, gphi, gE, a);
}
template <int kLaw>
__device__ __forceinline__ void leaf_adj_law(double q, double dx, double dy, double dz,
                                             double eps2, double gphi, const double gE[3],
                                             double a[14]) {
  if constexpr (kLaw == 3) leaf_adj(q, dx, dy, dz, eps2, gphi, gE, a);
  else law_adj<kLaw>(true, q, nullptr, dx, dy, dz, eps2, gphi, gE, a);
}

// The warp's records for one node summed through shared memory (a leaf's
// record has charge and position terms only, a[0] and a[10..12]; a twig's
// everything but the abs_charge slot, which only the downward pass fills):
// every lane
// writes its values into a column of buf (zeros where it did not contribute),
// then lane k sums row k over the 32 lanes, in lane order with four partial
// sums, and adds it to the node with one atomic.  13 stores, 32 loads and 35
// additions per node; a butterfly of warp shuffles needs 13 x 5 double
// shuffles (measured: the shared-memory form halves the per-target adjoint).
constexpr int kRedRow = 33;  // padded row: lanes k = 0..12 read distinct banks
__device__ __forceinline__ void flush_smem(double* __restrict__ adj, unsigned u, double a[14],
                                           int lane, bool leaf, double* __restrict__ buf) {
#pragma unroll
  for (int k = 0; k < 13; ++k) {
    if (leaf && k >= 1 && k < 10) continue;
    buf[k * kRedRow + lane] = a[k];
    a[k] = 0.0;
  }
  __syncwarp();
  if (lane < 13 && !(leaf && lane >= 1 && lane < 10)) {
    const double* row = buf + lane * kRedRow;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
    for (int j = 0; j < 32; j += 4) {
      s0 += row[j];
      s1 += row[j + 1];
      s2 += row[j + 2];
      s3 += row[j + 3];
    }
    const double v = (s0 + s1) + (s2 + s3);
    if (v != 0.0) atomicAdd(adj + (int64_t)kNA * u + lane, v);
  }
  __syncwarp();
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
  const double* macb;  // per-twig MAC threshold, or nullptr: bl2 of the level (Barnes-Hut)
  const double* vbox;
  int nbox;
  double theta2, eps2;
  int32_t M;
  double* adj;
  const int2* tiles;  // per tile: (first, count); nullptr: per-target semantics
  int64_t ntiles;
  // per-target work split (k_adj_target): the nsub twigs on split_level
  int split_level;
  int nsub;
  const int32_t* sublist;
  const int32_t* parent;
  const int32_t* lvlpos;  // RPO index -> the adjoint record's position (level order)
  unsigned int* queue;             // bucket counter (k_adj_group), zeroed before the launch
  unsigned long long* item_queue;  // item counter (k_adj_target), zeroed before the launch
  // spatial_interaction_cutoff: an interaction whose offset has any |component|
  // >= cut is skipped, as in the forward walks (after the leaf / MAC decision)
  int has_cut;
  double cut[3];
};

__device__ __forceinline__ bool adj_cut(const AdjArgs& A, double dx, double dy, double dz) {
  return A.has_cut && (fabs(dx) >= A.cut[0] || fabs(dy) >= A.cut[1] || fabs(dz) >= A.cut[2]);
}

// per-target semantics: the min-next-index schedule of k_walk_target64.
// With few targets the walk of a 32-target bucket is cut into work items so
// that enough warps run: item 0 covers the nodes above the split level (and
// the leaves on it) and skips the twigs on it; item k >= 1 covers the subtree
// of the k-th twig S on the split level for the lanes that reach S, i.e.
// whose walk opened every ancestor of S below the root.  The union of the
// items is exactly each target's interaction list; only the order of the
// (atomic) adjoint sums changes.
// Five resident blocks per SM (at most 102 registers; 126 unbounded): the
// 262,144-target self adjoint takes 10.0 / 13.2 ms against 11.2 / 13.6 ms.
template <bool kWithE, int kLaw>
__global__ void __launch_bounds__(kAdjThreads, 5) k_adj_target(AdjArgs A) {
  __shared__ double s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  __shared__ double s_red[kAdjThreads / 32][13 * kRedRow];  // per warp: flush_smem's rows
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  double* sred = s_red[threadIdx.x >> 5];
  const unsigned M = (unsigned)A.M;
  const int64_t per = 1 + (int64_t)A.nsub;
  const int64_t nitems = (A.nt + 31) / 32 * per;
  for (;;) {
    unsigned long long item = 0;
    if (lane == 0) item = atomicAdd(A.item_queue, 1ull);
    item = __shfl_sync(0xffffffffu, item, 0);
    if ((int64_t)item >= nitems) break;
    const int64_t b = (int64_t)item / per;
    const int sub = (int)((int64_t)item % per);
    const int64_t t = b * 32 + lane;
    const bool valid = t < A.nt;
    double px = 0, py = 0, pz = 0, gp = 0, gE[3] = {0, 0, 0};
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      gp = A.gphi[t];
      gE[0] = A.gex[t]; gE[1] = A.gey[t]; gE[2] = A.gez[t];
    }
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double sx = px - s_vb[3 * ib], sy = py - s_vb[3 * ib + 1], sz = pz - s_vb[3 * ib + 2];
      unsigned next = valid ? 1u : M, end = M;
      if (sub > 0) {
        const int S = A.sublist[sub - 1];
        end = (unsigned)A.meta[S].x;
        bool reach = valid;
        for (int p = A.parent[S]; p > 0; p = A.parent[p]) {
          const double4 pn = A.nc4[p];
          const double dx = sx - pn.x, dy = sy - pn.y, dz = sz - pn.z;
          const double dist2 = (dx * dx + dy * dy) + dz * dz;
          const double thr = A.macb ? A.macb[p] : s_bl2[A.meta[p].y & 0xff];
          if (A.theta2 * dist2 > thr) reach = false;  // accepted above S
        }
        next = reach ? (unsigned)S : end;
      }
      double a[14];
#pragma unroll
      for (int k = 0; k < 14; ++k) a[k] = 0.0;
      for (;;) {
        const unsigned u = __reduce_min_sync(0xffffffffu, next);
        if (u >= end) break;
        const double4 nd = A.nc4[u];
        const int2 mu = A.meta[u];
        const bool leaf = (mu.y & kLeafFlag) != 0;  // the same node for every lane
        if (sub == 0 && A.nsub > 0 && !leaf && (mu.y & 0xff) == A.split_level) {
          if (next == u) next = (unsigned)mu.x;  // the subtree items cover it
          continue;
        }
        bool contrib = false;
        if (next == u) {
          const double dx = sx - nd.x, dy = sy - nd.y, dz = sz - nd.z;
          const double dist2 = (dx * dx + dy * dy) + dz * dz;
          if (leaf) {
            if (dist2 > 0.0 && !adj_cut(A, dx, dy, dz)) {
              leaf_adj_law<kLaw>(nd.w, dx, dy, dz, A.eps2, gp, gE, a);
              contrib = true;
            }
            next = u + 1;
          } else if (A.theta2 * dist2 > (A.macb ? A.macb[u] : s_bl2[mu.y & 0xff])) {
            if (!adj_cut(A, dx, dy, dz)) {
              double m[9];
#pragma unroll
              for (int k = 0; k < 9; ++k) m[k] = A.mom[kMomStride * (int64_t)u + k];
              twig_adj_law<kWithE, kLaw>(nd.w, m, dx, dy, dz, A.eps2, gp, gE, a);
              contrib = true;
            }
            next = (unsigned)mu.x;
          } else {
            next = u + 1;
          }
        }
        const unsigned cm = __ballot_sync(0xffffffffu, contrib);
        if (cm != 0u && __popc(cm) <= kDirectLanes) {
          // few contributors: each adds its own record, no warp reduction
          if (contrib) {
            double* d = A.adj + (int64_t)kNA * A.lvlpos[u];
#pragma unroll
            for (int k = 0; k < 13; ++k) {
              if ((leaf && k >= 1 && k < 10) || a[k] == 0.0) continue;
              atomicAdd(d + k, a[k]);
              a[k] = 0.0;
            }
          }
        } else if (cm != 0u) {
          flush_smem(A.adj, (unsigned)A.lvlpos[u], a, lane, leaf, sred);
        }
      }
    }
  }
}

// per-tile / group semantics: the warp's targets share every node; a twig is
// accepted if all of them pass the MAC (module_tree_walk_simple.f90:343-382).
// kTPL targets per lane (2: the 64-target buckets of group_size 64, lane k
// holding targets t0 + k and t0 + 32 + k, as the FP64 group walk does); a
// lane's targets add into the same node record before the warp's reduction.
template <bool kWithE, int kTPL, int kLaw>
__global__ void __launch_bounds__(kAdjThreads, 5) k_adj_group(AdjArgs A) {
  __shared__ double s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  __shared__ double s_red[kAdjThreads / 32][13 * kRedRow];  // per warp: flush_smem's rows
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  double* sred = s_red[threadIdx.x >> 5];
  const unsigned M = (unsigned)A.M;
  const int64_t nbk = A.ntiles;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(A.queue, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b >= nbk) break;
    const int2 tl = A.tiles[b];
    bool valid[kTPL];
    double px[kTPL], py[kTPL], pz[kTPL], gp[kTPL], gE[kTPL][3];
#pragma unroll
    for (int s = 0; s < kTPL; ++s) {
      valid[s] = lane + 32 * s < tl.y;
      const int64_t t = (int64_t)tl.x + lane + 32 * s;
      px[s] = py[s] = pz[s] = gp[s] = 0.0;
      gE[s][0] = gE[s][1] = gE[s][2] = 0.0;
      if (valid[s]) {
        px[s] = A.tx[t]; py[s] = A.ty[t]; pz[s] = A.tz[t];
        gp[s] = A.gphi[t];
        gE[s][0] = A.gex[t]; gE[s][1] = A.gey[t]; gE[s][2] = A.gez[t];
      }
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
        double dx[kTPL], dy[kTPL], dz[kTPL], dist2[kTPL];
#pragma unroll
        for (int s = 0; s < kTPL; ++s) {
          dx[s] = (px[s] - vx) - nd.x; dy[s] = (py[s] - vy) - nd.y; dz[s] = (pz[s] - vz) - nd.z;
          dist2[s] = (dx[s] * dx[s] + dy[s] * dy[s]) + dz[s] * dz[s];
        }
        if (mu.y & kLeafFlag) {
#pragma unroll
          for (int s = 0; s < kTPL; ++s)
            if (valid[s] && dist2[s] > 0.0 && !adj_cut(A, dx[s], dy[s], dz[s]))
              leaf_adj_law<kLaw>(nd.w, dx[s], dy[s], dz[s], A.eps2, gp[s], gE[s], a);
          flush_smem(A.adj, (unsigned)A.lvlpos[u], a, lane, true, sred);
          u = (unsigned)fw.y;
        } else {
          const double thr = A.macb ? A.macb[u] : s_bl2[mu.y & 0xff];
          bool ok = true;
#pragma unroll
          for (int s = 0; s < kTPL; ++s) ok = ok && (!valid[s] || (A.theta2 * dist2[s] > thr));
          if (__all_sync(0xffffffffu, ok)) {
            if (valid[0]) {
              double m[9];
#pragma unroll
              for (int k = 0; k < 9; ++k) m[k] = A.mom[kMomStride * (int64_t)u + k];
#pragma unroll
              for (int s = 0; s < kTPL; ++s)
                if (valid[s] && !adj_cut(A, dx[s], dy[s], dz[s]))
                  twig_adj_law<kWithE, kLaw>(nd.w, m, dx[s], dy[s], dz[s], A.eps2, gp[s],
                                             gE[s], a);
            }
            flush_smem(A.adj, (unsigned)A.lvlpos[u], a, lane, false, sred);
            u = (unsigned)fw.y;
          } else {
            u = (unsigned)fw.x;
          }
        }
      }

    }
  }
}

// transpose of shift_multipoles_up for the twigs of one level (top-down);
// the twigs of a level come from the per-level lists built by the grow, and
// each twig's children are read as one run of the grow's level-ordered
// records (drec: centre and charge, abs_charge; link.w the RPO index of the
// child's adjoint record) and its twig children's dipoles from dmom at their
// twig-list positions -- the values of nc4 and mom, without chasing the
// children through meta.  Children in key order, as shift_multipoles_up.
__global__ void k_adj_down_level(int level, const int32_t* __restrict__ lvl,
                                 const int32_t* __restrict__ twiglist,
                                 const int2* __restrict__ tinfo,
                                 const int32_t* __restrict__ cfirst,
                                 const int32_t* __restrict__ tfirst,
                                 const LevelRecord* __restrict__ drec,
                                 const double* __restrict__ dmom, double* __restrict__ adj) {
  int base = 0;
  for (int l = 0; l < level; ++l) base += lvl[l];
  const int cnt = lvl[level];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int P = base + i;
    const int64_t u = twiglist[P];
    const int2 ti = tinfo[P];
    const int nc = ti.x & 0xff;
    const unsigned lm = (unsigned)ti.x >> 8;  // leaf children, by slot
    const LevelRecord* rc = drec + cfirst[P] + 1;  // child slot 0
    const int ts = tfirst[P] + 1;                  // twig-list position of the first twig child
    const double4 pc = drec[ti.y].pos;
    const double A = drec[ti.y].ab.x;
    const double* pa = adj + kNA * (int64_t)ti.y;
    const double Pq = pa[0];
    const double Pp[3] = {pa[1], pa[2], pa[3]};
    const double PQ[6] = {pa[4], pa[5], pa[6], pa[7], pa[8], pa[9]};
    double cocbar[3] = {pa[10], pa[11], pa[12]};
    const double PA = pa[13];
    // first pass: everything except the centre-of-charge chain rule
    for (int k = 0; k < nc; ++k) {
      const double4 cc = rc[k].pos;
      const bool leafc = (lm >> k) & 1u;
      double pcv[3] = {0, 0, 0};
      if (!leafc) {
        const double* dm = dmom + kDmomStride * (int64_t)(ts + __popc(~lm & ((1u << k) - 1u)));
        for (int j = 0; j < 3; ++j) pcv[j] = dm[j];
      }
      const double qc = cc.w;
      const double sc[3] = {pc.x - cc.x, pc.y - cc.y, pc.z - cc.z};
      double sbar[3] = {0, 0, 0};
      for (int j = 0; j < 3; ++j) sbar[j] += Pp[j] * qc;
      for (int j = 0; j < 3; ++j) sbar[j] += PQ[j] * (pcv[j] + qc * sc[j]);
      sbar[0] += PQ[3] * (pcv[1] + qc * sc[1]); sbar[1] += PQ[3] * (pcv[0] + qc * sc[0]);
      sbar[1] += PQ[4] * (pcv[2] + qc * sc[2]); sbar[2] += PQ[4] * (pcv[1] + qc * sc[1]);
      sbar[2] += PQ[5] * (pcv[0] + qc * sc[0]); sbar[0] += PQ[5] * (pcv[2] + qc * sc[2]);
      double* a = adj + kNA * (int64_t)(cfirst[P] + 1 + k);
      double aq = Pq;
      for (int j = 0; j < 3; ++j) aq += Pp[j] * sc[j] + PQ[j] * 0.5 * sc[j] * sc[j];
      aq += PQ[3] * sc[0] * sc[1] + PQ[4] * sc[1] * sc[2] + PQ[5] * sc[2] * sc[0];
      a[0] += aq;
      a[1] += Pp[0] + PQ[0] * sc[0] + PQ[3] * sc[1] + PQ[5] * sc[2];
      a[2] += Pp[1] + PQ[1] * sc[1] + PQ[3] * sc[0] + PQ[4] * sc[2];
      a[3] += Pp[2] + PQ[2] * sc[2] + PQ[4] * sc[1] + PQ[5] * sc[0];
      for (int s2 = 0; s2 < 6; ++s2) a[4 + s2] += PQ[s2];
      for (int j = 0; j < 3; ++j) {
        a[10 + j] -= sbar[j];
        cocbar[j] += sbar[j];
      }
      a[13] += PA;
    }
    // second pass: coc = sum coc_c A_c / A (or the plain mean when A = 0)
    for (int k = 0; k < nc; ++k) {
      const double4 cc = rc[k].pos;
      double* a = adj + kNA * (int64_t)(cfirst[P] + 1 + k);
      if (A != 0.0) {
        const double Ac = rc[k].ab.x;  // abs_charge (a leaf's |q|)
        const double w = Ac / A;
        const double cv[3] = {cc.x, cc.y, cc.z};
        const double pv[3] = {pc.x, pc.y, pc.z};
        double g = 0.0;
        for (int j = 0; j < 3; ++j) {
          a[10 + j] += cocbar[j] * w;
          g += cocbar[j] * (cv[j] - pv[j]);
        }
        a[13] += g / A;
      } else {
        for (int j = 0; j < 3; ++j) a[10 + j] += cocbar[j] / (double)nc;
      }
    }
  }
}

// leaves -> particles in the caller's original order
__global__ void k_adj_out(int64_t n, const int32_t* __restrict__ leafnode,
                          const int32_t* __restrict__ lvlpos,
                          const int32_t* __restrict__ perm, const double* __restrict__ q,
                          const double* __restrict__ adj, double* dq, double* dx, double* dy,
                          double* dz) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double* a = adj + (int64_t)kNA * lvlpos[leafnode[i]];
    const int64_t o = perm[i];
    const double sg = (double)((q[i] > 0.0) - (q[i] < 0.0));
    dq[o] = a[0] + a[13] * sg;
    dx[o] = a[10];
    dy[o] = a[11];
    dz[o] = a[12];
  }
}

__global__ void k_reset_adj(unsigned int* q, unsigned long long* items) {
  *q = 0;
  *items = 0;
}

__global__ void k_any_nonzero(int64_t n, const double* a, const double* b, const double* c,
                              unsigned int* flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (a[i] != 0.0 || b[i] != 0.0 || c[i] != 0.0) atomicOr(flag, 1u);
}

// the group walk's buckets of bs key-consecutive targets as (first, count)
__global__ void k_buckets(int64_t nt, int bs, int2* tiles) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b * bs < nt;
       b += (int64_t)gridDim.x * blockDim.x)
    tiles[b] = make_int2((int)(b * bs), (int)min((int64_t)bs, nt - b * bs));
}

// the FP64 adjoint walk of the context's semantics and force law
template <int kLaw>
void launch_adj(bool per_target, int tpl, bool with_e, int blocks, cudaStream_t s,
                const AdjArgs& A) {
  if (per_target) {
    if (with_e) k_adj_target<true, kLaw><<<blocks, kAdjThreads, 0, s>>>(A);
    else k_adj_target<false, kLaw><<<blocks, kAdjThreads, 0, s>>>(A);
  } else if (tpl == 2) {
    if (with_e) k_adj_group<true, 2, kLaw><<<blocks, kAdjThreads, 0, s>>>(A);
    else k_adj_group<false, 2, kLaw><<<blocks, kAdjThreads, 0, s>>>(A);
  } else {
    if (with_e) k_adj_group<true, 1, kLaw><<<blocks, kAdjThreads, 0, s>>>(A);
    else k_adj_group<false, 1, kLaw><<<blocks, kAdjThreads, 0, s>>>(A);
  }
}
void launch_adj_law(int law, bool per_target, int tpl, bool with_e, int blocks, cudaStream_t s,
                    const AdjArgs& A) {
  if (law == 2) launch_adj<2>(per_target, tpl, with_e, blocks, s, A);
  else if (law == 4) launch_adj<4>(per_target, tpl, with_e, blocks, s, A);
  else launch_adj<3>(per_target, tpl, with_e, blocks, s, A);
}

}  // namespace

int adjoint_device(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                   const double* gex, const double* gey, const double* gez, const double* gphi,
                   double* dq, double* dx, double* dy, double* dz) {
  if (!c->has_tree) {
    c->err = "adjoint called without a grown tree";
    return PEPCG_ERR_NO_TREE;
  }
  if (c->prm.force_law == 5) {
    c->err = "the adjoint of the Kelbg law (force_law = 5) is not built: its leaf kernel needs "
             "each target's own charge, which the adjoint's targets do not carry";
    return PEPCG_ERR_UNSUPPORTED;
  }
  // the mixed walks refuse a finite cutoff already (check_params); the FP64
  // adjoint walks skip the interactions the forward skips
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
  {
    int rc = prepare_mac(c, &A.macb);
    if (rc) return rc;
  }
  A.vbox = c->d_vbox;
  A.nbox = c->nboxes;
  A.theta2 = c->prm.theta2;
  A.eps2 = c->prm.eps2;
  A.M = (int32_t)M;
  A.adj = c->adj.p;
  A.queue = c->walk_queue();
  A.item_queue = c->item_queue();
  A.tiles = nullptr;
  A.ntiles = 0;
  A.split_level = 0;
  A.nsub = 0;
  A.sublist = nullptr;
  A.parent = c->parent.p;
  A.lvlpos = c->lvlpos.p;
  A.has_cut = has_spatial_cutoff(c->prm) ? 1 : 0;
  for (int k = 0; k < 3; ++k) A.cut[k] = c->prm.spatial_interaction_cutoff[k];
  const bool per_target = (c->prm.walk == PEPCG_WALK_PER_TARGET);
  // the mixed group walk with 64-target buckets (the benchmark's walk) has
  // its own adjoint walk, on the forward's FP32 lists (walk_mixed.cu)
  const bool mixed64 = c->prm.precision != PEPCG_PRECISION_PLAIN &&
                       c->prm.walk == PEPCG_WALK_GROUP && c->group_size() == 64;
  if (per_target) {
    // split the per-target walk until about 16 warps per SM have work
    const int64_t nb = (nt + 31) / 32;
    const int64_t want = 148 * 16;
    int base = 0;
    for (int L = 0; L <= 4 && L < c->max_level && nb * (1 + A.nsub) < want; ++L) {
      if (L >= 1 && c->lvl_host[L] > 0) {
        A.split_level = L;
        A.nsub = c->lvl_host[L];
        A.sublist = c->twiglist.p + base;
      }
      base += c->lvl_host[L];
    }
  }
  if (!per_target && !mixed64) {
    // the same tiles as the forward walk of these targets
    if (!ensure(c, c->tiles, 2 * (nt + 32), "tiles")) return PEPCG_ERR_OOM;
    int2* d_tiles = reinterpret_cast<int2*>(c->tiles.p);
    int64_t ntiles = 0;
    if (c->prm.walk == PEPCG_WALK_GROUP) {
      const int bs = c->group_size();
      ntiles = (nt + bs - 1) / bs;
      COUNT_LAUNCH();
      k_buckets<<<148, 256, 0, s>>>(nt, bs, d_tiles);
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
  k_reset_adj<<<1, 1, 0, s>>>(A.queue, A.item_queue);
  const int blocks = 148 * 8;
  if (mixed64) {
    int rc = launch_adjoint_group64(c, nt, tx, ty, tz, gex, gey, gez, gphi, h_flag != 0, s);
    if (rc) return rc;
  } else {
    const int tpl = (!per_target && c->prm.walk == PEPCG_WALK_GROUP && c->group_size() == 64) ? 2 : 1;
    COUNT_LAUNCH();
    launch_adj_law(c->prm.force_law, per_target, tpl, h_flag != 0, blocks, s, A);
  }
  const unsigned g = (unsigned)((M + 255) / 256 > 148 * 16 ? 148 * 16 : (M + 255) / 256);
  for (int L = 0; L < c->max_level; ++L) {
    const int64_t cnt = c->lvl_host[L];
    if (cnt <= 0) continue;
    const unsigned gl = (unsigned)std::min<int64_t>((cnt + 255) / 256, 148 * 16);
    COUNT_LAUNCH();
    k_adj_down_level<<<gl, 256, 0, s>>>(L, c->lvlcnt.p, c->twiglist.p, c->tinfo.p,
                                        c->tcounts.p, c->tcounts.p + c->ntwig, c->drec.p,
                                        c->dmom.p, c->adj.p);
  }
  COUNT_LAUNCH();
  k_adj_out<<<g, 256, 0, s>>>(c->n, c->leafnode.p, c->lvlpos.p, c->perm.p, c->q.p, c->adj.p, dq,
                              dx, dy, dz);
  if (!cuda_ok(c, cudaGetLastError(), "adjoint")) return PEPCG_ERR_CUDA;
  // the periodic far-lattice term's adjoint (FP64, lattice.cu) adds to the walk's
  return c->far_field ? lattice_adjoint(c, nt, tx, ty, tz, gex, gey, gez, gphi, dq, dx, dy, dz)
                      : PEPCG_OK;
}

}  // namespace pepcg
