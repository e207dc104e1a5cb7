// walk_mixed.cu -- the mixed-precision walks.
//
// Precision contract.  Every interaction offset is formed in FP64 from the
// FP64 positions and then rounded to FP32; the interaction (monopole + dipole
// + quadrupole, Plummer softened) is evaluated in FP32 with rsqrt; per target
// the FP32 sums of each batch of <= 32 interactions are added to FP64
// accumulators; node moments are computed in FP64 by the upward pass and
// rounded to FP32 once per grow (k_upward_level in grow.cu).
//  * Group walk: the offsets of the target and of the node centre from the
//    group centre g (the centre of the 32 targets' bounding box) are each
//    formed in FP64 and rounded once; the interaction offset is their FP32
//    difference.  Against the FP64 offset rounded once, the extra error is at
//    most 2u (|t - g| + |d|) with u = 2^-24: 2u (1 + r_g/|d|) relative, r_g
//    the group radius.  A leaf whose FP32 offset is exactly zero is re-tested
//    in FP64, so the self test is the reference's dist2 == 0.
//  * Per-target walk: target minus node centre in FP64, then rounded.
//
// The FP32 twig interaction is the reference's quadrupole kernel
// (coulomb/module_coulomb_kernels.f90:60-145) rewritten in the equivalent
// form
//   phi = q/r - (d.p)/r^3 + 3 (d.M.d)/r^5 - tr(Q)/r^3
//   E   = d [q/r^3 - 3 (d.p)/r^5 + 15 (d.M.d)/r^7 - 3 tr(Q)/r^5] + p/r^3 - 6 (M.d)/r^5
// with M = [[qxx, qxy/2, qzx/2], [qxy/2, qyy, qyz/2], [qzx/2, qyz/2, qzz]]
// (expanding the reference's fdx.. / pre2x.. terms gives exactly these
// polynomials), which needs 39 FP32 operations instead of ~130.

#include <type_traits>

#include "internal.cuh"

namespace pepcg {

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
  const float4* mom32;  // kMom32Stride float4 per node, the first 3 used
  const int32_t* nleaves;
  const LevelRecord* drec;  // level-ordered node records with walk links (grow.cu)
  const double* bl2;
  const double* macb;  // per-twig MAC threshold, or nullptr: bl2 of the level (Barnes-Hut)
  const double* vbox;
  int nbox;
  float theta2;
  float eps2;
  double theta2d;  // theta2 in FP64 (the strict form's exact MAC)
  int32_t M;
  int64_t npart;
  double* ex;
  double* ey;
  double* ez;
  double* pot;
  double* work;
  unsigned long long* counters;
  uint32_t* status;
  unsigned int* queue;  // bucket counter, zeroed before the launch
  const int2* tiles;  // PER_TILE tiles, or nullptr for GROUP (implicit 32-target buckets)
  int64_t ntiles;
  // packed per-tile walk
  const int2* fwd;       // (first child, next after the subtree), RPO indices
  const int2* fwdf;      // the same as forward-preorder indices
  const int32_t* tflag;  // per target: length of the tile starting there, else 0
  const int32_t* pstart;  // packed per-tile walk: first target of each pack, then nt
  const int32_t* npacks;  // the number of packs (device)
};

// 1/sqrt(x) by the PTX instruction rsqrt.approx.ftz.f32 (relative error below
// 2^-22, subnormal inputs and results flushed to zero).  The arguments here are
// squared distances plus eps2; a zero argument gives +inf and is selected away
// by the callers that can meet it (the leaves' self pairs).  rsqrtf would add a
// range fix-up for subnormal arguments on every call: at 4M this form takes the
// benchmark's walk from 38.5 to 36.0 ms with identical results.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ void leaf32(float q, float dx, float dy, float dz, float eps2,
                                       float& ax, float& ay, float& az, float& ap) {
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
  const float ri = rsqrt_ftz(r2);
  const float qr = q * ri;
  const float qr3 = qr * ri * ri;
  ap += qr;
  ax = fmaf(qr3, dx, ax);
  ay = fmaf(qr3, dy, ay);
  az = fmaf(qr3, dz, az);
}

// m0 = (px, py, pz, 3qxx), m1 = (3qyy, 3qzz, 1.5qxy, 1.5qyz), m2 = (1.5qzx, tr, q, -),
// i.e. 3M with M the quadrupole matrix with halved off-diagonals; with
// A = d.p + tr, v = 3M d and B = d.v, in Horner form in 1/r^2:
//   phi += (q + (B/r^2 - A)/r^2) / r
//   E   += [d (q + (5B/r^2 - 3A)/r^2) + p - 2 v/r^2] / r^3
// where 5B/r^2 - 3A = 5 (B/r^2 - A) + 2A reuses the potential's inner term:
// 39 FP32 operations and one rsqrt per interaction.
__device__ __forceinline__ void twig32(float4 m0, float4 m1, float4 m2, float dx, float dy,
                                       float dz, float eps2, float& ax, float& ay, float& az,
                                       float& ap) {
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
  const float ri = rsqrt_ftz(r2);
  const float ri2 = ri * ri;
  const float rd3 = ri * ri2;
  const float q = m2.z;
  const float A = fmaf(dx, m0.x, fmaf(dy, m0.y, fmaf(dz, m0.z, m2.y)));
  const float vx = fmaf(m0.w, dx, fmaf(m1.z, dy, m2.x * dz));
  const float vy = fmaf(m1.z, dx, fmaf(m1.x, dy, m1.w * dz));
  const float vz = fmaf(m2.x, dx, fmaf(m1.w, dy, m1.y * dz));
  const float B = fmaf(dx, vx, fmaf(dy, vy, dz * vz));
  const float t1 = fmaf(ri2, B, -A);
  ap = fmaf(ri, fmaf(ri2, t1, q), ap);
  const float t4 = fmaf(ri2, fmaf(5.0f, t1, A + A), q);
  const float m2r = -2.0f * ri2;
  ax = fmaf(rd3, fmaf(t4, dx, fmaf(m2r, vx, m0.x)), ax);
  ay = fmaf(rd3, fmaf(t4, dy, fmaf(m2r, vy, m0.y)), ay);
  az = fmaf(rd3, fmaf(t4, dz, fmaf(m2r, vz, m0.z)), az);
}

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// twig32 for two targets against the same node in packed FP32 (sm_100
// FFMA2 / FMUL2 / FADD2): each operation evaluates both targets' terms, and
// the node's moments enter as (m, m) pairs.  Per target the arithmetic is
// twig32's, operation for operation.
__device__ __forceinline__ void twig32x2(float4 m0, float4 m1, float4 m2, float2 dx, float2 dy,
                                         float2 dz, float2 eps2, float2& ax, float2& ay,
                                         float2& az, float2& ap) {
  const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
  const float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
  const float2 ri2 = __fmul2_rn(ri, ri);
  const float2 rd3 = __fmul2_rn(ri, ri2);
  const float2 q = f2(m2.z);
  const float2 A = __ffma2_rn(dx, f2(m0.x), __ffma2_rn(dy, f2(m0.y), __ffma2_rn(dz, f2(m0.z), f2(m2.y))));
  const float2 vx = __ffma2_rn(f2(m0.w), dx, __ffma2_rn(f2(m1.z), dy, __fmul2_rn(f2(m2.x), dz)));
  const float2 vy = __ffma2_rn(f2(m1.z), dx, __ffma2_rn(f2(m1.x), dy, __fmul2_rn(f2(m1.w), dz)));
  const float2 vz = __ffma2_rn(f2(m2.x), dx, __ffma2_rn(f2(m1.w), dy, __fmul2_rn(f2(m1.y), dz)));
  const float2 B = __ffma2_rn(dx, vx, __ffma2_rn(dy, vy, __fmul2_rn(dz, vz)));
  const float2 t1 = __ffma2_rn(ri2, B, make_float2(-A.x, -A.y));
  ap = __ffma2_rn(ri, __ffma2_rn(ri2, t1, q), ap);
  const float2 t4 = __ffma2_rn(ri2, __ffma2_rn(f2(5.0f), t1, __fadd2_rn(A, A)), q);
  const float2 m2r = __fmul2_rn(f2(-2.0f), ri2);
  ax = __ffma2_rn(rd3, __ffma2_rn(t4, dx, __ffma2_rn(m2r, vx, f2(m0.x))), ax);
  ay = __ffma2_rn(rd3, __ffma2_rn(t4, dy, __ffma2_rn(m2r, vy, f2(m0.y))), ay);
  az = __ffma2_rn(rd3, __ffma2_rn(t4, dz, __ffma2_rn(m2r, vz, f2(m0.z))), az);
}

// twig32x2's terms of one interaction, returned instead of accumulated (the
// strict form adds them with compensation)
__device__ __forceinline__ void twig32x2_terms(float4 m0, float4 m1, float4 m2, float2 dx,
                                               float2 dy, float2 dz, float2 eps2, float2& ax,
                                               float2& ay, float2& az, float2& ap) {
  const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
  const float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
  const float2 ri2 = __fmul2_rn(ri, ri);
  const float2 rd3 = __fmul2_rn(ri, ri2);
  const float2 q = f2(m2.z);
  const float2 A = __ffma2_rn(dx, f2(m0.x), __ffma2_rn(dy, f2(m0.y), __ffma2_rn(dz, f2(m0.z), f2(m2.y))));
  const float2 vx = __ffma2_rn(f2(m0.w), dx, __ffma2_rn(f2(m1.z), dy, __fmul2_rn(f2(m2.x), dz)));
  const float2 vy = __ffma2_rn(f2(m1.z), dx, __ffma2_rn(f2(m1.x), dy, __fmul2_rn(f2(m1.w), dz)));
  const float2 vz = __ffma2_rn(f2(m2.x), dx, __ffma2_rn(f2(m1.w), dy, __fmul2_rn(f2(m1.y), dz)));
  const float2 B = __ffma2_rn(dx, vx, __ffma2_rn(dy, vy, __fmul2_rn(dz, vz)));
  const float2 t1 = __ffma2_rn(ri2, B, make_float2(-A.x, -A.y));
  ap = __fmul2_rn(ri, __ffma2_rn(ri2, t1, q));
  const float2 t4 = __ffma2_rn(ri2, __ffma2_rn(f2(5.0f), t1, __fadd2_rn(A, A)), q);
  const float2 m2r = __fmul2_rn(f2(-2.0f), ri2);
  ax = __fmul2_rn(rd3, __ffma2_rn(t4, dx, __ffma2_rn(m2r, vx, f2(m0.x))));
  ay = __fmul2_rn(rd3, __ffma2_rn(t4, dy, __ffma2_rn(m2r, vy, f2(m0.y))));
  az = __fmul2_rn(rd3, __ffma2_rn(t4, dz, __ffma2_rn(m2r, vz, f2(m0.z))));
}

// Kahan (compensated) summation, both lanes of a pair: s += v with the
// running compensation c (the sum is s - c)
__device__ __forceinline__ void kahan2(float2& s, float2& c, float2 v) {
  const float2 y = __fadd2_rn(v, make_float2(-c.x, -c.y));
  const float2 t = __fadd2_rn(s, y);
  c = __fadd2_rn(__fadd2_rn(t, make_float2(-s.x, -s.y)), make_float2(-y.x, -y.y));
  s = t;
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

// Group walk (GROUP and PER_TILE modes): per-tile semantics
// (module_tree_walk_simple.f90:256-384) -- a twig is accepted only if every
// target of the warp's group passes the Barnes-Hut MAC, else it is opened --
// with a wide traversal.  The traversal pops up to 32 nodes from a per-warp
// LIFO stack (global memory) and lane k decides node k:
//   leaf -> queued for evaluation;
//   twig -> the group's bounding sphere decides most nodes at once (every
//           target farther than the MAC distance: accept; none: open); the
//           rest get the exact test one node at a time across the warp
//           (lane = target, a ballot of the failures); opened twigs push
//           their children (child8 table).
// A popped node's centre, level, leaf count and child table are loaded in
// one round.  The MAC is evaluated on the FP32 group-centred offsets, and
// the same offsets go straight into the node's staging record: accepted
// twigs and leaves are written into per-warp ring buffers in shared memory
// at decision time (the twig moments by cp.async), so a batch of 32 is
// evaluated without a load on its critical path; every lane then reads all
// staged records by broadcast.
// Stack bound: a pop takes <= 32 entries and pushes <= 8 per node, so the
// stack never holds more than (kMaxLevel + 1) * 8 * 32 entries; kStackCap
// leaves a margin and an overflow sets ST_INCOMPLETE instead of writing past it.
constexpr int kStackCap = 8192;
constexpr int kWW = kMixThreads / 32;  // warps per block
constexpr int kRing = 64;              // staging ring (<= 31 pending + 32 new)

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

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

struct __align__(16) StagedTwig {
  float4 c;   // (coc - g) rounded from FP64 (k_walk_group64: its negation), charge
  float4 m0;  // px py pz 3qxx
  float4 m1;  // 3qyy 3qzz 1.5qxy 1.5qyz
  float4 m2;  // 1.5qzx, trace, charge, -
};
// the strict form's twig record: the FP64 node centre, then the moments
struct __align__(16) StagedTwigS {
  double cx, cy, cz;
  float pad[2];
  float4 m0, m1, m2;
};
struct __align__(16) StagedLeaf {
  float4 c;          // (x - g) rounded from FP64, charge
  double x, y, z;    // FP64 position, for the exact self test
};

__global__ void __launch_bounds__(kMixThreads, 5)
    k_walk_group_wide(MixArgs A, int* __restrict__ gstack, const int4* __restrict__ child8,
                      const int* __restrict__ nchild) {
  __shared__ float s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  __shared__ StagedTwig s_tw[kWW][kRing];
  __shared__ StagedLeaf s_lf[kWW][kRing];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = (float)A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int* stack = gstack + (int64_t)(blockIdx.x * kWW + w) * kStackCap;
  StagedTwig* stw = s_tw[w];
  StagedLeaf* stl = s_lf[w];
  const float theta2 = A.theta2;
  const int64_t nbuckets = A.tiles ? A.ntiles : (A.nt + 31) / 32;
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(A.queue, 1u);
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
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
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
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double vx = s_vb[3 * ib], vy = s_vb[3 * ib + 1], vz = s_vb[3 * ib + 2];
      const double sx = px - vx, sy = py - vy, sz = pz - vz;
      const double gx = g0x - vx, gy = g0y - vy, gz = g0z - vz;
      int64_t partner = 0;  // leaves covered by this lane's nodes (summed over the warp at the end)
      int nT = 0, hT = 0, nL = 0, hL = 0;  // ring counts and heads
      int top = 1;
      if (lane == 0) stack[0] = 0;  // the root (walk_simple starts at the root, :286)
      __syncwarp();
      // evaluates the n staged twigs / leaves at the ring heads
      auto flush_twigs = [&](int n) {
        cp_async_wait_all();
        __syncwarp();
        if (valid) {
          float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
          // the batch is at most two contiguous runs of the ring
          const int n1 = min(n, kRing - hT);
          const StagedTwig* r = stw + hT;
#pragma unroll 16
          for (int j = 0; j < n1; ++j) {
            const float4 c = r[j].c;
            twig32(r[j].m0, r[j].m1, r[j].m2, rx - c.x, ry - c.y, rz - c.z, A.eps2, ax, ay, az, ap);
          }
#pragma unroll 8
          for (int j = 0; j < n - n1; ++j) {
            const float4 c = stw[j].c;
            twig32(stw[j].m0, stw[j].m1, stw[j].m2, rx - c.x, ry - c.y, rz - c.z, A.eps2, ax, ay,
                   az, ap);
          }
          E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
          c_twig += (unsigned)n;
        }
        W += (double)n;
        hT = (hT + n) & (kRing - 1);
        nT -= n;
        __syncwarp();
      };
      auto flush_leaves = [&](int n) {
        __syncwarp();
        if (valid) {
          float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
          auto leaf = [&](const StagedLeaf& r) {
            const float4 c = r.c;
            float dx = rx - c.x, dy = ry - c.y, dz = rz - c.z;
            if (dx == 0.f && dy == 0.f && dz == 0.f) {
              // self (dist2 == 0 in FP64) or two points closer than the FP32
              // resolution at the group scale: decide and evaluate in FP64
              const double ex = sx - r.x, ey = sy - r.y, ez = sz - r.z;
              if (ex == 0.0 && ey == 0.0 && ez == 0.0) return;
              dx = (float)ex; dy = (float)ey; dz = (float)ez;
            }
            leaf32(c.w, dx, dy, dz, A.eps2, ax, ay, az, ap);
            ++c_leaf;
          };
          // the batch is at most two contiguous runs of the ring
          const int n1 = min(n, kRing - hL);
          const StagedLeaf* r = stl + hL;
#pragma unroll 8
          for (int j = 0; j < n1; ++j) leaf(r[j]);
#pragma unroll 4
          for (int j = 0; j < n - n1; ++j) leaf(stl[j]);
          E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
        }
        W += (double)n;
        hL = (hL + n) & (kRing - 1);
        nL -= n;
        __syncwarp();
      };
      while (top > 0) {
        const int take = top < 32 ? top : 32;
        top -= take;
        const int node = lane < take ? stack[top + lane] : -1;
        __syncwarp();
        bool isleaf = false, accept = false, open = false, amb = false;
        float cx = 0.f, cy = 0.f, cz = 0.f, bl = 0.f;
        double4 a = make_double4(0, 0, 0, 0);
        int nlv = 0, nch = 0;
        int4 c0 = make_int4(0, 0, 0, 0), c1 = c0;
        if (node >= 0) {
          // one round of loads: what accept, open and leaf each need
          a = A.nc4[node];
          const int2 mu = A.meta[node];
          nlv = A.nleaves[node];
          nch = nchild[node];
          c0 = child8[2 * (int64_t)node];
          c1 = child8[2 * (int64_t)node + 1];
          cx = (float)(a.x - gx); cy = (float)(a.y - gy); cz = (float)(a.z - gz);
          if (mu.y & kLeafFlag) {
            isleaf = true;
          } else {
            bl = A.macb ? (float)A.macb[node] : s_bl2[mu.y & 0xff];
            const float dc = sqrtf(cx * cx + cy * cy + cz * cz);
            const float dmin = dc - rg, dmax = dc + rg;
            if (dmin > 0.f && theta2 * (dmin * dmin) > bl) {
              accept = true;  // every target is farther than dmin
              c_mac += 1;
            } else if (!(theta2 * (dmax * dmax) > bl)) {
              open = true;    // no target can pass
              c_mac += 1;
            } else {
              amb = true;
            }
          }
        }
        // the exact MAC for the undecided nodes, one node at a time across
        // the targets (lane = target): accepted iff no target fails
        unsigned am = __ballot_sync(0xffffffffu, amb);
        while (am) {
          const int j = __ffs(am) - 1;
          am &= am - 1;
          const float ux = __shfl_sync(0xffffffffu, cx, j);
          const float uy = __shfl_sync(0xffffffffu, cy, j);
          const float uz = __shfl_sync(0xffffffffu, cz, j);
          const float ub = __shfl_sync(0xffffffffu, bl, j);
          const float dx = rx - ux, dy = ry - uy, dz = rz - uz;
          const bool fail = valid && !(theta2 * fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > ub);
          const unsigned f = __ballot_sync(0xffffffffu, fail);
          if (lane == j) {
            accept = (f == 0);
            open = !accept;
            // MAC evaluations up to the first failing target, in target order
            c_mac += (unsigned)__popc(f ? (vmask & ((2u << (__ffs(f) - 1)) - 1u)) : vmask);
          }
        }
        const unsigned lb = __ballot_sync(0xffffffffu, isleaf);
        const unsigned ab = __ballot_sync(0xffffffffu, accept);
        if (isleaf) {
          StagedLeaf& r = stl[(hL + nL + __popc(lb & lt)) & (kRing - 1)];
          r.c = make_float4(cx, cy, cz, (float)a.w);
          r.x = a.x; r.y = a.y; r.z = a.z;
          partner += 1;
        }
        if (accept) {
          StagedTwig& r = stw[(hT + nT + __popc(ab & lt)) & (kRing - 1)];
          r.c = make_float4(cx, cy, cz, (float)a.w);
          const float4* m = A.mom32 + kMom32Stride * (int64_t)node;
          cp_async16(&r.m0, m);
          cp_async16(&r.m1, m + 1);
          cp_async16(&r.m2, m + 2);
          partner += nlv;
        }
        nL += __popc(lb);
        nT += __popc(ab);
        // push the children of opened twigs
        const int npush = open ? min(8, nch) : 0;
        int total;
        const int off = warp_excl_scan(npush, lane, total);
        if (top + total > kStackCap) {
          complete = false;  // cannot happen within the bound above
          break;
        }
        if (npush > 0) {
          int* dst = stack + top + off;
          dst[0] = c0.x;
          if (npush > 1) dst[1] = c0.y;
          if (npush > 2) dst[2] = c0.z;
          if (npush > 3) dst[3] = c0.w;
          if (npush > 4) dst[4] = c1.x;
          if (npush > 5) dst[5] = c1.y;
          if (npush > 6) dst[6] = c1.z;
          if (npush > 7) dst[7] = c1.w;
        }
        top += total;
        __syncwarp();
        if (nT >= 32) flush_twigs(32);
        if (nL >= 32) flush_leaves(32);
      }
      if (nT > 0) flush_twigs(nT);
      if (nL > 0) flush_leaves(nL);
      for (int o = 16; o > 0; o >>= 1) partner += __shfl_xor_sync(0xffffffffu, partner, o);
      if (partner != A.npart) complete = false;
    }
    if (valid) {
      A.ex[t] = E0; A.ey[t] = E1; A.ez[t] = E2; A.pot[t] = PH; A.work[t] = W;
    }
    if (__any_sync(0xffffffffu, !complete) && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  cp_async_wait_all();
  warp_add3(A.counters, c_leaf, c_twig, c_mac);
}

// Group walk over buckets of 64 key-consecutive targets (group_size 64), two
// per lane: lane k holds targets t0 + k and t0 + 32 + k.  The traversal, the
// MAC rule (a twig is accepted only if all 64 targets pass) and the staging
// are those of k_walk_group_wide.  Each staged record is read from shared
// memory once for both of the lane's targets, and the twig interactions of
// the pair run as packed FP32 (twig32x2).  Twig records store the node's
// offset from the group centre negated, so that the pair's offsets are one
// packed add.  Against 32-target buckets the larger group is opened more
// often (about 9 % more interactions at 4M, theta 0.4); the packed pair
// arithmetic and the halved traversal per target more than pay for it.
//
// kStrict (PEPCG_PRECISION_MIXED_STRICT): every interaction offset is the
// target minus the node centre formed in FP64 and then rounded, the FP32 sums
// of a batch are Kahan-compensated, and the group's MAC decisions equal the
// FP64 group walk's (k_walk_tile64 with two targets per lane): the bounding-
// sphere test is made conservative by a relative margin, and every node it
// leaves undecided gets the reference's FP64 test per target.  Twig records
// carry the FP64 node centre; four blocks per SM (128 registers).
template <bool kStrict>
__global__ void __launch_bounds__(kMixThreads, kStrict ? 4 : 5)
    k_walk_group64(MixArgs A, int* __restrict__ gstack) {
  using TwigRec = typename std::conditional<kStrict, StagedTwigS, StagedTwig>::type;
  __shared__ float s_bl2[kMaxLevel + 1];
  __shared__ double s_bl2d[kStrict ? kMaxLevel + 1 : 1];
  __shared__ double s_vb[3 * 125];
  __shared__ TwigRec s_tw[kWW][kRing];
  __shared__ StagedLeaf s_lf[kWW][kRing];
  // the two targets' FP64 sums (E, phi) live here rather than in registers: they
  // change once per batch of 32 records, and the registers go to the batches
  __shared__ double s_acc[8][kMixThreads];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) {
    s_bl2[i] = (float)A.bl2[i];
    if constexpr (kStrict) s_bl2d[i] = A.bl2[i];
  }
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int* stack = gstack + (int64_t)(blockIdx.x * kWW + w) * kStackCap;
  TwigRec* stw = s_tw[w];
  StagedLeaf* stl = s_lf[w];
  const float theta2 = A.theta2;
  const int64_t nbuckets = (A.nt + 63) / 64;
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(A.queue, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b >= nbuckets) break;
    const int64_t t0 = (int64_t)b * 64;
    const int cnt = (int)min((int64_t)64, A.nt - t0);
    const bool v0 = lane < cnt, v1 = lane + 32 < cnt;
    const unsigned vm0 = __ballot_sync(0xffffffffu, v0), vm1 = __ballot_sync(0xffffffffu, v1);
    const int64_t ta = t0 + lane, tb = t0 + 32 + lane;
    double pxa = 0, pya = 0, pza = 0, pxb = 0, pyb = 0, pzb = 0;
    double &Ea0 = s_acc[0][threadIdx.x], &Ea1 = s_acc[1][threadIdx.x], &Ea2 = s_acc[2][threadIdx.x],
           &PHa = s_acc[3][threadIdx.x], &Eb0 = s_acc[4][threadIdx.x], &Eb1 = s_acc[5][threadIdx.x],
           &Eb2 = s_acc[6][threadIdx.x], &PHb = s_acc[7][threadIdx.x];
    Ea0 = Ea1 = Ea2 = PHa = Eb0 = Eb1 = Eb2 = PHb = 0.0;
    double W = 0;  // interactions of this call (the same list for all targets)
    if (v0) {
      pxa = A.tx[ta]; pya = A.ty[ta]; pza = A.tz[ta];
      Ea0 = A.ex[ta]; Ea1 = A.ey[ta]; Ea2 = A.ez[ta]; PHa = A.pot[ta];
    }
    if (v1) {
      pxb = A.tx[tb]; pyb = A.ty[tb]; pzb = A.tz[tb];
      Eb0 = A.ex[tb]; Eb1 = A.ey[tb]; Eb2 = A.ez[tb]; PHb = A.pot[tb];
    }
    double lo[3] = {v0 ? pxa : INFINITY, v0 ? pya : INFINITY, v0 ? pza : INFINITY};
    double hi[3] = {v0 ? pxa : -INFINITY, v0 ? pya : -INFINITY, v0 ? pza : -INFINITY};
    if (v1) {
      lo[0] = fmin(lo[0], pxb); lo[1] = fmin(lo[1], pyb); lo[2] = fmin(lo[2], pzb);
      hi[0] = fmax(hi[0], pxb); hi[1] = fmax(hi[1], pyb); hi[2] = fmax(hi[2], pzb);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
      for (int o = 16; o > 0; o >>= 1) {
        lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
        hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
      }
    const double g0x = 0.5 * (lo[0] + hi[0]), g0y = 0.5 * (lo[1] + hi[1]), g0z = 0.5 * (lo[2] + hi[2]);
    const float rxa = (float)(pxa - g0x), rya = (float)(pya - g0y), rza = (float)(pza - g0z);
    const float rxb = (float)(pxb - g0x), ryb = (float)(pyb - g0y), rzb = (float)(pzb - g0z);
    float rg = fmaxf(v0 ? sqrtf(rxa * rxa + rya * rya + rza * rza) : 0.f,
                     v1 ? sqrtf(rxb * rxb + ryb * ryb + rzb * rzb) : 0.f);
    for (int o = 16; o > 0; o >>= 1) rg = fmaxf(rg, __shfl_xor_sync(0xffffffffu, rg, o));
    rg = rg * 1.0001f + 1e-30f;  // the sphere must contain every target after rounding
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double vx = s_vb[3 * ib], vy = s_vb[3 * ib + 1], vz = s_vb[3 * ib + 2];
      const double gx = g0x - vx, gy = g0y - vy, gz = g0z - vz;
      // the targets' shifted positions x - vbox (the strict form's offsets)
      const double sxa = pxa - vx, sya = pya - vy, sza = pza - vz;
      const double sxb = pxb - vx, syb = pyb - vy, szb = pzb - vz;
      int64_t partner = 0;
      int nT = 0, hT = 0, nL = 0, hL = 0;
      int top = 1;
      if (lane == 0) stack[0] = 0;
      __syncwarp();
      auto flush_twigs = [&](int n) {
        cp_async_wait_all();
        __syncwarp();
        if constexpr (kStrict) {
          if (v0) {
            float2 PX = f2(0.f), PY = f2(0.f), PZ = f2(0.f), PP = f2(0.f);
            float2 CX = f2(0.f), CY = f2(0.f), CZ = f2(0.f), CP = f2(0.f);
            const float2 E2 = f2(A.eps2);
            auto one = [&](const TwigRec& r) {
              // target minus node centre in FP64, rounded once
              const float2 dx = make_float2((float)(sxa - r.cx), (float)(sxb - r.cx));
              const float2 dy = make_float2((float)(sya - r.cy), (float)(syb - r.cy));
              const float2 dz = make_float2((float)(sza - r.cz), (float)(szb - r.cz));
              float2 tx, ty, tz, tp;
              twig32x2_terms(r.m0, r.m1, r.m2, dx, dy, dz, E2, tx, ty, tz, tp);
              kahan2(PX, CX, tx);
              kahan2(PY, CY, ty);
              kahan2(PZ, CZ, tz);
              kahan2(PP, CP, tp);
            };
            const int n1 = min(n, kRing - hT);
            const TwigRec* r = stw + hT;
#pragma unroll 4
            for (int j = 0; j < n1; ++j) one(r[j]);
#pragma unroll 2
            for (int j = 0; j < n - n1; ++j) one(stw[j]);
            // the compensated sum is s - c
            Ea0 += (double)PX.x - (double)CX.x; Ea1 += (double)PY.x - (double)CY.x;
            Ea2 += (double)PZ.x - (double)CZ.x; PHa += (double)PP.x - (double)CP.x;
            Eb0 += (double)PX.y - (double)CX.y; Eb1 += (double)PY.y - (double)CY.y;
            Eb2 += (double)PZ.y - (double)CZ.y; PHb += (double)PP.y - (double)CP.y;
            c_twig += (unsigned)n * (v1 ? 2u : 1u);
          }
        } else if (v0) {
          float2 PX = f2(0.f), PY = f2(0.f), PZ = f2(0.f), PP = f2(0.f);
          const float2 RX = make_float2(rxa, rxb), RY = make_float2(rya, ryb),
                       RZ = make_float2(rza, rzb);
          const float2 E2 = f2(A.eps2);
          const int n1 = min(n, kRing - hT);
          const TwigRec* r = stw + hT;
#pragma unroll 16
          for (int j = 0; j < n1; ++j) {
            // c is the negated offset: one packed add per axis
            const float4 c = r[j].c, m0 = r[j].m0, m1 = r[j].m1, m2 = r[j].m2;
            twig32x2(m0, m1, m2, __fadd2_rn(RX, f2(c.x)), __fadd2_rn(RY, f2(c.y)),
                     __fadd2_rn(RZ, f2(c.z)), E2, PX, PY, PZ, PP);
          }
#pragma unroll 4
          for (int j = 0; j < n - n1; ++j) {
            // c is the negated offset: one packed add per axis
            const float4 c = stw[j].c, m0 = stw[j].m0, m1 = stw[j].m1, m2 = stw[j].m2;
            twig32x2(m0, m1, m2, __fadd2_rn(RX, f2(c.x)), __fadd2_rn(RY, f2(c.y)),
                     __fadd2_rn(RZ, f2(c.z)), E2, PX, PY, PZ, PP);
          }
          Ea0 += (double)PX.x; Ea1 += (double)PY.x; Ea2 += (double)PZ.x; PHa += (double)PP.x;
          Eb0 += (double)PX.y; Eb1 += (double)PY.y; Eb2 += (double)PZ.y; PHb += (double)PP.y;
          c_twig += (unsigned)n * (v1 ? 2u : 1u);
        }
        W += (double)n;
        hT = (hT + n) & (kRing - 1);
        nT -= n;
        __syncwarp();
      };
      auto flush_leaves = [&](int n) {
        __syncwarp();
        if (kStrict && v0) {
          float2 PX = f2(0.f), PY = f2(0.f), PZ = f2(0.f), PP = f2(0.f);
          float2 CX = f2(0.f), CY = f2(0.f), CZ = f2(0.f), CP = f2(0.f);
          const float2 E2 = f2(A.eps2);
          unsigned nuse = 0;
          auto leaf = [&](const StagedLeaf& r) {
            const double exa = sxa - r.x, eya = sya - r.y, eza = sza - r.z;
            const double exb = sxb - r.x, eyb = syb - r.y, ezb = szb - r.z;
            float2 wq = f2(r.c.w);
            // self: dist2 == 0 in FP64 (module_tree_walk_pthreads.f90:625)
            if (exa == 0.0 && eya == 0.0 && eza == 0.0) { wq.x = 0.f; ++nuse; }
            if (v1 && exb == 0.0 && eyb == 0.0 && ezb == 0.0) { wq.y = 0.f; ++nuse; }
            const float2 dx = make_float2((float)exa, (float)exb);
            const float2 dy = make_float2((float)eya, (float)eyb);
            const float2 dz = make_float2((float)eza, (float)ezb);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, E2)));
            const float2 ri = make_float2(r2.x > 0.f ? rsqrt_ftz(r2.x) : 0.f, r2.y > 0.f ? rsqrt_ftz(r2.y) : 0.f);
            const float2 qr = __fmul2_rn(wq, ri);
            const float2 qr3 = __fmul2_rn(__fmul2_rn(qr, ri), ri);
            kahan2(PP, CP, qr);
            kahan2(PX, CX, __fmul2_rn(qr3, dx));
            kahan2(PY, CY, __fmul2_rn(qr3, dy));
            kahan2(PZ, CZ, __fmul2_rn(qr3, dz));
          };
          const int n1 = min(n, kRing - hL);
          const StagedLeaf* r = stl + hL;
#pragma unroll 4
          for (int j = 0; j < n1; ++j) leaf(r[j]);
#pragma unroll 2
          for (int j = 0; j < n - n1; ++j) leaf(stl[j]);
          Ea0 += (double)PX.x - (double)CX.x; Ea1 += (double)PY.x - (double)CY.x;
          Ea2 += (double)PZ.x - (double)CZ.x; PHa += (double)PP.x - (double)CP.x;
          Eb0 += (double)PX.y - (double)CX.y; Eb1 += (double)PY.y - (double)CY.y;
          Eb2 += (double)PZ.y - (double)CZ.y; PHb += (double)PP.y - (double)CP.y;
          c_leaf += (unsigned)n * (v1 ? 2u : 1u) - nuse;
        } else if (v0) {
          float2 PX = f2(0.f), PY = f2(0.f), PZ = f2(0.f), PP = f2(0.f);
          const float2 RX = make_float2(rxa, rxb), RY = make_float2(rya, ryb),
                       RZ = make_float2(rza, rzb);
          const float2 E2 = f2(A.eps2);
          unsigned nuse = 0;
          auto leaf = [&](const StagedLeaf& r, int k, unsigned& pend) {
            const float4 c = r.c;
            const float2 dx = __fadd2_rn(RX, f2(-c.x)), dy = __fadd2_rn(RY, f2(-c.y)),
                         dz = __fadd2_rn(RZ, f2(-c.z));
            const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            // a zero FP32 offset (the target's own leaf, or two points closer
            // than FP32 resolves at the group scale) enters with charge 0 here,
            // without a branch, and is decided and evaluated in FP64 after the
            // batch (pend: one bit per record of the batch)
            const bool za = d2.x == 0.f, zb = v1 && d2.y == 0.f;
            pend |= (za || zb) ? (1u << k) : 0u;
            const float2 wq = make_float2(za ? 0.f : c.w, zb ? 0.f : c.w);
            // the pair's leaf32 in packed FP32; a zero r2 (eps2 = 0) gives no
            // contribution instead of inf
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, E2)));
            const float2 ri = make_float2(r2.x > 0.f ? rsqrt_ftz(r2.x) : 0.f, r2.y > 0.f ? rsqrt_ftz(r2.y) : 0.f);
            const float2 qr = __fmul2_rn(wq, ri);
            const float2 qr3 = __fmul2_rn(__fmul2_rn(qr, ri), ri);
            PP = __fadd2_rn(PP, qr);
            PX = __ffma2_rn(qr3, dx, PX);
            PY = __ffma2_rn(qr3, dy, PY);
            PZ = __ffma2_rn(qr3, dz, PZ);
          };
          unsigned pend = 0;
          const int n1 = min(n, kRing - hL);
          const StagedLeaf* r = stl + hL;
#pragma unroll 4
          for (int j = 0; j < n1; ++j) leaf(r[j], j, pend);
#pragma unroll 2
          for (int j = 0; j < n - n1; ++j) leaf(stl[j], n1 + j, pend);
          // the zero-offset pairs: self when the FP64 offset is exactly zero
          // (dist2 == 0, module_tree_walk_pthreads.f90:625), else evaluated on
          // the FP64 offset rounded once
          while (pend) {
            const int k = __ffs(pend) - 1;
            pend &= pend - 1;
            const StagedLeaf& rr = stl[(hL + k) & (kRing - 1)];
            const float4 c = rr.c;
            for (int s2 = 0; s2 < 2; ++s2) {
              if (s2 == 1 && !v1) break;
              const float fx = (s2 ? rxb : rxa) - c.x, fy = (s2 ? ryb : rya) - c.y,
                          fz = (s2 ? rzb : rza) - c.z;
              if (fx * fx + fy * fy + fz * fz != 0.f) continue;  // evaluated in the batch
              const int64_t tt = s2 ? tb : ta;
              const double ex = (A.tx[tt] - vx) - rr.x, ey = (A.ty[tt] - vy) - rr.y,
                           ez = (A.tz[tt] - vz) - rr.z;
              if (ex == 0.0 && ey == 0.0 && ez == 0.0) {
                ++nuse;
                continue;
              }
              float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
              leaf32(c.w, (float)ex, (float)ey, (float)ez, A.eps2, ax, ay, az, ap);
              if (s2) { PX.y += ax; PY.y += ay; PZ.y += az; PP.y += ap; }
              else { PX.x += ax; PY.x += ay; PZ.x += az; PP.x += ap; }
            }
          }
          Ea0 += (double)PX.x; Ea1 += (double)PY.x; Ea2 += (double)PZ.x; PHa += (double)PP.x;
          Eb0 += (double)PX.y; Eb1 += (double)PY.y; Eb2 += (double)PZ.y; PHb += (double)PP.y;
          c_leaf += (unsigned)n * (v1 ? 2u : 1u) - nuse;
        }
        W += (double)n;
        hL = (hL + n) & (kRing - 1);
        nL -= n;
        __syncwarp();
      };
      while (top > 0) {
        const int take = top < 32 ? top : 32;
        top -= take;
        const int node = lane < take ? stack[top + lane] : -1;
        __syncwarp();
        bool isleaf = false, accept = false, open = false, amb = false;
        float cx = 0.f, cy = 0.f, cz = 0.f, bl = 0.f;
        double bld = 0.0;  // the strict form's FP64 MAC threshold
        double4 a = make_double4(0, 0, 0, 0);
        // the node's level-ordered record: centre and charge, then its links
        // (first child, level | leaf flag | child count, leaves, RPO index);
        // siblings are consecutive, so one round's loads are mostly runs
        int4 lk = make_int4(0, 0, 0, 0);
        if (node >= 0) {
          const LevelRecord* rec = A.drec + node;
          a = ld256(&rec->pos);
          lk = rec->link;
          cx = (float)(a.x - gx); cy = (float)(a.y - gy); cz = (float)(a.z - gz);
          if (lk.y & kLeafFlag) {
            isleaf = true;
          } else {
            bl = A.macb ? (float)A.macb[lk.w] : s_bl2[lk.y & 0xff];
            const float dc = sqrtf(cx * cx + cy * cy + cz * cz);
            float dmin = dc - rg, dmax = dc + rg;
            if constexpr (kStrict) {
              // conservative: the sphere decides only where the FP64 test of
              // every target certainly agrees
              bld = A.macb ? A.macb[lk.w] : s_bl2d[lk.y & 0xff];
              dmin = dc * (1.0f - 1e-5f) - rg;
              dmax = dc * (1.0f + 1e-5f) + rg;
            }
            if (dmin > 0.f && theta2 * (dmin * dmin) > bl) {
              accept = true;
              c_mac += 1;
            } else if (!(theta2 * (dmax * dmax) > bl)) {
              open = true;
              c_mac += 1;
            } else {
              amb = true;
            }
          }
        }
        unsigned am = __ballot_sync(0xffffffffu, amb);
        while (am) {
          const int j = __ffs(am) - 1;
          am &= am - 1;
          bool fa, fb;
          if constexpr (kStrict) {
            // mac (coulomb/module_interaction_specific.f90:256-275) in FP64, in
            // the reference's operation order: theta2 * dist2 > boxlength2
            const double ux = __shfl_sync(0xffffffffu, a.x, j);
            const double uy = __shfl_sync(0xffffffffu, a.y, j);
            const double uz = __shfl_sync(0xffffffffu, a.z, j);
            const double ub = __shfl_sync(0xffffffffu, bld, j);
            double dx = sxa - ux, dy = sya - uy, dz = sza - uz;
            double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            fa = v0 && !(__dmul_rn(A.theta2d, d2) > ub);
            dx = sxb - ux; dy = syb - uy; dz = szb - uz;
            d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            fb = v1 && !(__dmul_rn(A.theta2d, d2) > ub);
          } else {
            const float ux = __shfl_sync(0xffffffffu, cx, j);
            const float uy = __shfl_sync(0xffffffffu, cy, j);
            const float uz = __shfl_sync(0xffffffffu, cz, j);
            const float ub = __shfl_sync(0xffffffffu, bl, j);
            float dx = rxa - ux, dy = rya - uy, dz = rza - uz;
            fa = v0 && !(theta2 * fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > ub);
            dx = rxb - ux; dy = ryb - uy; dz = rzb - uz;
            fb = v1 && !(theta2 * fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > ub);
          }
          const unsigned f0 = __ballot_sync(0xffffffffu, fa);
          const unsigned f1 = __ballot_sync(0xffffffffu, fb);
          if (lane == j) {
            accept = (f0 | f1) == 0;
            open = !accept;
            // MAC evaluations up to the first failing target, in target order
            c_mac += (unsigned)(f0 ? __popc(vm0 & ((2u << (__ffs(f0) - 1)) - 1u))
                                   : __popc(vm0) + (f1 ? __popc(vm1 & ((2u << (__ffs(f1) - 1)) - 1u))
                                                       : __popc(vm1)));
          }
        }
        const unsigned lb = __ballot_sync(0xffffffffu, isleaf);
        const unsigned ab = __ballot_sync(0xffffffffu, accept);
        if (isleaf) {
          StagedLeaf& r = stl[(hL + nL + __popc(lb & lt)) & (kRing - 1)];
          r.c = make_float4(cx, cy, cz, (float)a.w);
          r.x = a.x; r.y = a.y; r.z = a.z;
          partner += 1;
        }
        if (accept) {
          TwigRec& r = stw[(hT + nT + __popc(ab & lt)) & (kRing - 1)];
          if constexpr (kStrict) {
            r.cx = a.x;
            r.cy = a.y;
            r.cz = a.z;
          } else {
            r.c = make_float4(-cx, -cy, -cz, (float)a.w);
          }
          const float4* m = A.mom32 + kMom32Stride * (int64_t)lk.w;
          cp_async16(&r.m0, m);
          cp_async16(&r.m1, m + 1);
          cp_async16(&r.m2, m + 2);
          partner += lk.z;
        }
        nL += __popc(lb);
        nT += __popc(ab);
        // an opened twig's children: level-order positions first .. first + nch - 1
        const int npush = open ? min(8, lk.y >> 16) : 0;
        int total;
        const int off = warp_excl_scan(npush, lane, total);
        if (top + total > kStackCap) {
          complete = false;
          break;
        }
        if (npush > 0) {
          int* dst = stack + top + off;
#pragma unroll
          for (int k = 0; k < 8; ++k)
            if (k < npush) dst[k] = lk.x + k;
        }
        top += total;
        __syncwarp();
        if (nT >= 32) flush_twigs(32);
        if (nL >= 32) flush_leaves(32);
      }
      if (nT > 0) flush_twigs(nT);
      if (nL > 0) flush_leaves(nL);
      for (int o = 16; o > 0; o >>= 1) partner += __shfl_xor_sync(0xffffffffu, partner, o);
      if (partner != A.npart) complete = false;
    }
    if (v0) {
      A.ex[ta] = Ea0; A.ey[ta] = Ea1; A.ez[ta] = Ea2; A.pot[ta] = PHa; A.work[ta] = A.work[ta] + W;
    }
    if (v1) {
      A.ex[tb] = Eb0; A.ey[tb] = Eb1; A.ez[tb] = Eb2; A.pot[tb] = PHb; A.work[tb] = A.work[tb] + W;
    }
    if (__any_sync(0xffffffffu, !complete) && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  cp_async_wait_all();
  warp_add3(A.counters, c_leaf, c_twig, c_mac);
}

// Simple-walk semantics (module_tree_walk_simple.f90:256-385) with several
// reference tiles per warp and FP32 interactions: the whole tiles of one
// pack (at most 32 targets, k_pack_tiles) walk the tree together in forward
// preorder -- at each step the lanes whose tile stands at
// the smallest forward-preorder index evaluate that node, and each tile
// decides accept / open by a ballot over its own lanes (the MAC on the FP32
// offsets, target minus node centre formed in FP64).  Sums as in the
// per-target mixed walk: FP32 over chunks of kChunk steps, then FP64.
__global__ void __launch_bounds__(kMixThreads) k_walk_tilepack_mixed(MixArgs A) {
  __shared__ float s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = (float)A.bl2[i];
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
    const bool valid = pack_lane(A.pstart, A.tflag, b, lane, tl0, len);
    if (!__any_sync(0xffffffffu, valid)) {
      if (lane == 0) atomicOr(A.status, ST_INCOMPLETE);  // a pack must start with a tile
      continue;
    }
    const int64_t t = A.pstart[b] + lane;
    const unsigned tmask = valid ? (((len >= 32) ? 0xffffffffu : ((1u << len) - 1u)) << tl0) : 0u;
    double px = 0, py = 0, pz = 0, E0 = 0, E1 = 0, E2 = 0, PH = 0, W8 = 0;
    if (valid) {
      px = A.tx[t]; py = A.ty[t]; pz = A.tz[t];
      E0 = A.ex[t]; E1 = A.ey[t]; E2 = A.ez[t]; PH = A.pot[t]; W8 = A.work[t];
    }
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double sx = px - s_vb[3 * ib], sy = py - s_vb[3 * ib + 1], sz = pz - s_vb[3 * ib + 2];
      float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
      int steps = 0;
      unsigned u = 0, uf = 0;  // the root
      int64_t partner = 0;
      for (;;) {
        const unsigned f = __reduce_min_sync(0xffffffffu, valid ? uf : 0xffffffffu);
        if (f >= M) break;
        // the lanes at node f: whole tiles at the same node
        const unsigned am = __ballot_sync(0xffffffffu, valid && uf == f);
        if (valid && uf == f) {
          // one round of loads, the moments and leaf count included
          const double4 a = A.nc4[u];
          const int2 mu = A.meta[u];
          const int2 fw = A.fwd[u];
          const int2 ff = A.fwdf[u];
          const float4* mu4 = A.mom32 + kMom32Stride * (int64_t)u;
          const float4 m0 = mu4[0], m1 = mu4[1], m2 = mu4[2];
          const int nlv = A.nleaves[u];
          const double dx64 = sx - a.x, dy64 = sy - a.y, dz64 = sz - a.z;
          const float dx = (float)dx64, dy = (float)dy64, dz = (float)dz64;
          if (mu.y & kLeafFlag) {
            partner += 1;
            W8 += 1.0;
            if (!(dx64 == 0.0 && dy64 == 0.0 && dz64 == 0.0)) {
              leaf32((float)a.w, dx, dy, dz, A.eps2, ax, ay, az, ap);
              ++c_leaf;
            }
            u = (unsigned)fw.y;
            uf = (unsigned)ff.y;
          } else {
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const bool ok = A.theta2 * r2 > (A.macb ? (float)A.macb[u] : s_bl2[mu.y & 0xff]);
            const unsigned tf = __ballot_sync(am, !ok) & tmask;
            // MAC evaluations stop at the tile's first failing target
            const int first_fail = tf ? __ffs(tf) - 1 : 32;
            if (lane <= first_fail) ++c_mac;
            if (tf == 0) {
              partner += nlv;
              twig32(m0, m1, m2, dx, dy, dz, A.eps2, ax, ay, az, ap);
              ++c_twig;
              W8 += 1.0;
              u = (unsigned)fw.y;
              uf = (unsigned)ff.y;
            } else {
              u = (unsigned)fw.x;
              uf = (unsigned)ff.x;
            }
          }
          if (++steps == kChunk) {
            E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
            ax = ay = az = ap = 0.f;
            steps = 0;
          }
        }
        __syncwarp();
      }
      E0 += (double)ax; E1 += (double)ay; E2 += (double)az; PH += (double)ap;
      if (valid && partner != A.npart) complete = false;
    }
    if (valid) {
      A.ex[t] = E0; A.ey[t] = E1; A.ez[t] = E2; A.pot[t] = PH; A.work[t] = W8;
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
    if (lane == 0) b = atomicAdd(A.queue, 1u);
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
          // one round of loads: the moments and leaf count are requested with
          // the centre, before the MAC decides whether they are used
          const double4 a = A.nc4[u];
          const int2 mu = A.meta[u];
          const float4* mu4 = A.mom32 + kMom32Stride * (int64_t)u;
          const float4 m0 = mu4[0], m1 = mu4[1], m2 = mu4[2];
          const int nlv = A.nleaves[u];
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
            if (A.theta2 * r2 > (A.macb ? (float)A.macb[u] : s_bl2[mu.y & 0xff])) {
              partner += nlv;
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

// ---------------------------------------------------------------------------
// Adjoint of the mixed group walk with 64-target buckets.  The traversal, the
// FP32 group-centred MAC and the staging are k_walk_group64's, so each
// bucket's interaction list is the forward list.  The staged batches are
// evaluated transposed: lane j takes node record j of the batch and loops over
// the bucket's 64 targets, whose group-centred FP32 offsets and gradients are
// broadcast from shared memory two at a time (one packed FP32 operation per
// target pair).  A lane thus sums its node's adjoint record over the bucket
// without any cross-lane reduction, in FP32 as the forward sums its batches,
// and adds it to the node's FP64 record with one atomic per value.  The terms
// are the transposes of the forward's (the FP64 forms and their derivation
// are in adjoint.cu, twig_adj / leaf_adj), rewritten with T = 3M, v = T d and
// dTd = d.v: with s1 = gphi R1 and s3 = 3 gphi R2,
//   qbar   += gphi R0                      (+ (g.d) R1)
//   pbar   -= s1 d                         (+ R1 g - 3 (g.d) R2 d)
//   Qbar_kl += s3 d_k d_l - delta_kl s1    (+ 15 (g.d) R3 d_k d_l - 3 R2 (g_k d_l + g_l d_k + delta_kl g.d))
//   cocbar += gphi [ce d + R1 p - 2 R2 v]  (+ the Hessian terms of twig_adj)
// with ce = q R1 - 3 R2 (p.d + tr) + 5 R3 dTd; sums over the targets of a
// node-constant factor (the p terms, the delta terms) are taken once per batch.
// ---------------------------------------------------------------------------
struct AdjMixArgs {
  int64_t nt;
  const double *tx, *ty, *tz;
  const double *gex, *gey, *gez, *gphi;
  const double4* nc4;
  const int2* meta;
  const float4* mom32;
  const int32_t* nleaves;
  const LevelRecord* drec;  // level-ordered node records with walk links (grow.cu)
  const double* bl2;
  const double* macb;
  const double* vbox;
  int nbox;
  float theta2, eps2;
  int64_t npart;
  double* adj;  // 16 doubles per node, level order: q, p(3), Q(6: xx yy zz xy yz zx), coc(3), abs_charge, pad
  unsigned long long* counters;
  uint32_t* status;
  unsigned int* queue;
};

constexpr int kNAdj = 16;

struct __align__(16) StagedLeafA {
  float4 c;        // (x - g) rounded from FP64, charge
  double x, y, z;  // FP64 position, for the exact self test
  int node;
  int pad;
};

__device__ __forceinline__ void adj_add(double* __restrict__ a, float2 v) {
  const double s = (double)v.x + (double)v.y;
  if (s != 0.0) atomicAdd(a, s);
}

// Four resident blocks per SM (128 registers, the twig terms' pair
// accumulators and node constants stay in registers): at 4M the full
// gradient takes 88 ms against 111 ms at five blocks (96 registers, spills).
template <bool kWithE>
__global__ void __launch_bounds__(kMixThreads, 4)
    k_adj_group64(AdjMixArgs A, int* __restrict__ gstack) {
  __shared__ float s_bl2[kMaxLevel + 1];
  __shared__ double s_vb[3 * 125];
  __shared__ StagedTwig s_tw[kWW][kRing];
  __shared__ StagedLeafA s_lf[kWW][kRing];
  // per warp and target pair p (targets t0 + p, t0 + 32 + p): (rx, rx', ry, ry'),
  // (rz, rz', gphi, gphi'), (gx, gx', gy, gy'), (gz, gz', -, -)
  __shared__ float4 s_tg[kWW][32][kWithE ? 4 : 2];
  for (int i = threadIdx.x; i <= kMaxLevel; i += blockDim.x) s_bl2[i] = (float)A.bl2[i];
  for (int i = threadIdx.x; i < 3 * A.nbox; i += blockDim.x) s_vb[i] = A.vbox[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int* stack = gstack + (int64_t)(blockIdx.x * kWW + w) * kStackCap;
  StagedTwig* stw = s_tw[w];
  StagedLeafA* stl = s_lf[w];
  float4(*tg)[kWithE ? 4 : 2] = s_tg[w];
  const float theta2 = A.theta2;
  const float2 E2 = f2(A.eps2);
  const int64_t nbuckets = (A.nt + 63) / 64;
  unsigned long long c_leaf = 0, c_twig = 0, c_mac = 0;
  for (;;) {
    unsigned b = 0;
    if (lane == 0) b = atomicAdd(A.queue, 1u);
    b = __shfl_sync(0xffffffffu, b, 0);
    if ((int64_t)b >= nbuckets) break;
    const int64_t t0 = (int64_t)b * 64;
    const int cnt = (int)min((int64_t)64, A.nt - t0);
    const bool v0 = lane < cnt, v1 = lane + 32 < cnt;
    const unsigned vm0 = __ballot_sync(0xffffffffu, v0), vm1 = __ballot_sync(0xffffffffu, v1);
    const int nvalid = __popc(vm0) + __popc(vm1);
    const int64_t ta = t0 + lane, tb = t0 + 32 + lane;
    double pxa = 0, pya = 0, pza = 0, pxb = 0, pyb = 0, pzb = 0;
    float gpa = 0.f, gpb = 0.f, gxa = 0.f, gya = 0.f, gza = 0.f, gxb = 0.f, gyb = 0.f, gzb = 0.f;
    if (v0) {
      pxa = A.tx[ta]; pya = A.ty[ta]; pza = A.tz[ta];
      gpa = (float)A.gphi[ta];
      if (kWithE) { gxa = (float)A.gex[ta]; gya = (float)A.gey[ta]; gza = (float)A.gez[ta]; }
    }
    if (v1) {
      pxb = A.tx[tb]; pyb = A.ty[tb]; pzb = A.tz[tb];
      gpb = (float)A.gphi[tb];
      if (kWithE) { gxb = (float)A.gex[tb]; gyb = (float)A.gey[tb]; gzb = (float)A.gez[tb]; }
    }
    double lo[3] = {v0 ? pxa : INFINITY, v0 ? pya : INFINITY, v0 ? pza : INFINITY};
    double hi[3] = {v0 ? pxa : -INFINITY, v0 ? pya : -INFINITY, v0 ? pza : -INFINITY};
    if (v1) {
      lo[0] = fmin(lo[0], pxb); lo[1] = fmin(lo[1], pyb); lo[2] = fmin(lo[2], pzb);
      hi[0] = fmax(hi[0], pxb); hi[1] = fmax(hi[1], pyb); hi[2] = fmax(hi[2], pzb);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
      for (int o = 16; o > 0; o >>= 1) {
        lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
        hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
      }
    const double g0x = 0.5 * (lo[0] + hi[0]), g0y = 0.5 * (lo[1] + hi[1]), g0z = 0.5 * (lo[2] + hi[2]);
    const float rxa = (float)(pxa - g0x), rya = (float)(pya - g0y), rza = (float)(pza - g0z);
    const float rxb = (float)(pxb - g0x), ryb = (float)(pyb - g0y), rzb = (float)(pzb - g0z);
    float rg = fmaxf(v0 ? sqrtf(rxa * rxa + rya * rya + rza * rza) : 0.f,
                     v1 ? sqrtf(rxb * rxb + ryb * ryb + rzb * rzb) : 0.f);
    for (int o = 16; o > 0; o >>= 1) rg = fmaxf(rg, __shfl_xor_sync(0xffffffffu, rg, o));
    rg = rg * 1.0001f + 1e-30f;  // the sphere must contain every target after rounding
    // an absent target sits far away with zero gradients: it adds exact zeros
    tg[lane][0] = make_float4(v0 ? rxa : 1e10f, v1 ? rxb : 1e10f, v0 ? rya : 1e10f, v1 ? ryb : 1e10f);
    tg[lane][1] = make_float4(v0 ? rza : 1e10f, v1 ? rzb : 1e10f, gpa, gpb);
    if constexpr (kWithE) {
      tg[lane][2] = make_float4(gxa, gxb, gya, gyb);
      tg[lane][3] = make_float4(gza, gzb, 0.f, 0.f);
    }
    __syncwarp();
    bool complete = true;
    for (int ib = 0; ib < A.nbox; ++ib) {
      const double vx = s_vb[3 * ib], vy = s_vb[3 * ib + 1], vz = s_vb[3 * ib + 2];
      const double gx = g0x - vx, gy = g0y - vy, gz = g0z - vz;
      int64_t partner = 0;
      int nT = 0, hT = 0, nL = 0, hL = 0;
      int top = 1;
      if (lane == 0) stack[0] = 0;
      __syncwarp();
      // twig records: lane j sums node j's record over the bucket's targets
      auto flush_twigs = [&](int n) {
        cp_async_wait_all();
        __syncwarp();
        if (lane < n) {
          const StagedTwig& r = stw[(hT + lane) & (kRing - 1)];
          const float4 c = r.c, m0 = r.m0, m1 = r.m1, m2 = r.m2;
          const int node = __float_as_int(c.w);
          const float2 CX = f2(c.x), CY = f2(c.y), CZ = f2(c.z);  // d = r_t + c
          const float2 PX = f2(m0.x), PY = f2(m0.y), PZ = f2(m0.z);
          // -(p.d + tr) = (-p).d + (-tr): the negated dipole and trace, once per record
          const float2 NPX = f2(-m0.x), NPY = f2(-m0.y), NPZ = f2(-m0.z), NTR = f2(-m2.y);
          const float2 Txx = f2(m0.w), Tyy = f2(m1.x), Tzz = f2(m1.y), Txy = f2(m1.z),
                       Tyz = f2(m1.w), Tzx = f2(m2.x), Q = f2(m2.z);
          float2 aq = f2(0.f), apx = f2(0.f), apy = f2(0.f), apz = f2(0.f), aS = f2(0.f);
          float2 axx = f2(0.f), ayy = f2(0.f), azz = f2(0.f), axy = f2(0.f), ayz = f2(0.f),
                 azx = f2(0.f), acx = f2(0.f), acy = f2(0.f), acz = f2(0.f);
          float2 aGx = f2(0.f), aGy = f2(0.f), aGz = f2(0.f);  // sum of 2 R2 g (with E)
#pragma unroll 4
          for (int p = 0; p < 32; ++p) {
            const float4 ta4 = tg[p][0], tb4 = tg[p][1];
            const float2 dx = __fadd2_rn(make_float2(ta4.x, ta4.y), CX);
            const float2 dy = __fadd2_rn(make_float2(ta4.z, ta4.w), CY);
            const float2 dz = __fadd2_rn(make_float2(tb4.x, tb4.y), CZ);
            const float2 gp = make_float2(tb4.z, tb4.w);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, E2)));
            const float2 R0 = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
            const float2 i2 = __fmul2_rn(R0, R0);
            const float2 R1 = __fmul2_rn(R0, i2);
            // scaled radial factors: T3 = 3 R2, F5 = 5 R3
            const float2 T3 = __fmul2_rn(R1, __fmul2_rn(f2(3.f), i2));
            const float2 F5 = __fmul2_rn(T3, __fmul2_rn(f2(5.f / 3.f), i2));
            const float2 vx = __ffma2_rn(Txx, dx, __ffma2_rn(Txy, dy, __fmul2_rn(Tzx, dz)));
            const float2 vy = __ffma2_rn(Txy, dx, __ffma2_rn(Tyy, dy, __fmul2_rn(Tyz, dz)));
            const float2 vz = __ffma2_rn(Tzx, dx, __ffma2_rn(Tyz, dy, __fmul2_rn(Tzz, dz)));
            const float2 dTd = __ffma2_rn(dx, vx, __ffma2_rn(dy, vy, __fmul2_rn(dz, vz)));
            const float2 nu = __ffma2_rn(NPX, dx, __ffma2_rn(NPY, dy, __ffma2_rn(NPZ, dz, NTR)));
            // ce = q R1 - 3 R2 (p.d + tr) + 5 R3 dTd
            const float2 ce = __ffma2_rn(Q, R1, __ffma2_rn(T3, nu, __fmul2_rn(F5, dTd)));
            const float2 s1 = __fmul2_rn(gp, R1);
            float2 s3 = __fmul2_rn(gp, T3);
            aq = __ffma2_rn(gp, R0, aq);
            aS = __fadd2_rn(aS, s1);
            float2 kd = __fmul2_rn(gp, ce);                        // coefficient of d in cocbar
            float2 kv = __fmul2_rn(f2(-2.f / 3.f), s3);            // of v
            float2 ex_ = f2(0.f), ey_ = f2(0.f), ez_ = f2(0.f);     // -3 R2 g
            float2 ppx = s1;                                        // coefficient of -d in pbar
            if constexpr (kWithE) {
              const float4 tc4 = tg[p][2], td4 = tg[p][3];
              const float2 gxx = make_float2(tc4.x, tc4.y), gyy = make_float2(tc4.z, tc4.w),
                           gzz = make_float2(td4.x, td4.y);
              const float2 ga = __ffma2_rn(gxx, dx, __ffma2_rn(gyy, dy, __fmul2_rn(gzz, dz)));
              const float2 F15 = __fmul2_rn(f2(3.f), F5);
              const float2 F10n = __fmul2_rn(f2(-2.f), F5);
              const float2 S35 = __fmul2_rn(F5, __fmul2_rn(f2(7.f), i2));  // 35 R4
              aq = __ffma2_rn(ga, R1, aq);
              // pbar += R1 g - 3 ga R2 d, kept as -pbar
              const float2 h = __fmul2_rn(ga, T3);  // 3 ga R2
              const float2 nR1 = __fmul2_rn(f2(-1.f), R1);
              apx = __ffma2_rn(nR1, gxx, apx);
              apy = __ffma2_rn(nR1, gyy, apy);
              apz = __ffma2_rn(nR1, gzz, apz);
              ppx = __fadd2_rn(s1, h);
              // Qbar: 15 ga R3 d d - 3 R2 (g d + d g + ga I)
              s3 = __ffma2_rn(F15, ga, s3);
              const float2 nT3 = __fmul2_rn(f2(-1.f), T3);
              ex_ = __fmul2_rn(nT3, gxx);
              ey_ = __fmul2_rn(nT3, gyy);
              ez_ = __fmul2_rn(nT3, gzz);
              aS = __fadd2_rn(aS, h);  // the delta_kl and the p terms share 3 ga R2
              // cocbar: cd d + cg g + 3 R2 ga p - 10 R3 ga v + 2 R2 T g, cg = -ce,
              // cd = ga (3 q R2 - 15 R3 u + 35 R4 dTd) + 3 R2 (g.p) - 10 R3 (g.v);
              // T g is node-constant: the batch sums 2 R2 g (aG) and applies T once
              const float2 gP = __ffma2_rn(gxx, PX, __ffma2_rn(gyy, PY, __fmul2_rn(gzz, PZ)));
              const float2 gv = __ffma2_rn(gxx, vx, __ffma2_rn(gyy, vy, __fmul2_rn(gzz, vz)));
              const float2 inner = __ffma2_rn(Q, T3, __ffma2_rn(F15, nu, __fmul2_rn(S35, dTd)));
              const float2 cd = __ffma2_rn(ga, inner, __ffma2_rn(T3, gP, __fmul2_rn(F10n, gv)));
              kd = __fadd2_rn(kd, cd);
              kv = __ffma2_rn(F10n, ga, kv);
              const float2 R2x2 = __fmul2_rn(f2(2.f / 3.f), T3);
              aGx = __ffma2_rn(R2x2, gxx, aGx);
              aGy = __ffma2_rn(R2x2, gyy, aGy);
              aGz = __ffma2_rn(R2x2, gzz, aGz);
              const float2 nce = __fmul2_rn(f2(-1.f), ce);
              acx = __ffma2_rn(nce, gxx, acx);
              acy = __ffma2_rn(nce, gyy, acy);
              acz = __ffma2_rn(nce, gzz, acz);
            }
            apx = __ffma2_rn(ppx, dx, apx);
            apy = __ffma2_rn(ppx, dy, apy);
            apz = __ffma2_rn(ppx, dz, apz);
            // Qbar's d d terms and (with E) the g d terms:
            //   kl += (s3 d_k + e_k) d_l + e_l d_k,  e = -3 R2 g
            const float2 wx = __ffma2_rn(s3, dx, ex_), wy = __ffma2_rn(s3, dy, ey_),
                         wz = __ffma2_rn(s3, dz, ez_);
            axx = __ffma2_rn(__fadd2_rn(wx, ex_), dx, axx);
            ayy = __ffma2_rn(__fadd2_rn(wy, ey_), dy, ayy);
            azz = __ffma2_rn(__fadd2_rn(wz, ez_), dz, azz);
            axy = __ffma2_rn(wx, dy, __ffma2_rn(ey_, dx, axy));
            ayz = __ffma2_rn(wy, dz, __ffma2_rn(ez_, dy, ayz));
            azx = __ffma2_rn(wz, dx, __ffma2_rn(ex_, dz, azx));
            acx = __ffma2_rn(kd, dx, __ffma2_rn(kv, vx, acx));
            acy = __ffma2_rn(kd, dy, __ffma2_rn(kv, vy, acy));
            acz = __ffma2_rn(kd, dz, __ffma2_rn(kv, vz, acz));
          }
          double* a = A.adj + (int64_t)kNAdj * node;
          // the node-constant factors: the delta_kl terms and R1 p (with E also 3 R2 ga p)
          const double S = (double)aS.x + (double)aS.y;
          adj_add(a + 0, aq);
          adj_add(a + 1, make_float2(-apx.x, -apx.y));
          adj_add(a + 2, make_float2(-apy.x, -apy.y));
          adj_add(a + 3, make_float2(-apz.x, -apz.y));
          if (S != 0.0) {
            atomicAdd(a + 4, (double)axx.x + (double)axx.y - S);
            atomicAdd(a + 5, (double)ayy.x + (double)ayy.y - S);
            atomicAdd(a + 6, (double)azz.x + (double)azz.y - S);
          } else {
            adj_add(a + 4, axx);
            adj_add(a + 5, ayy);
            adj_add(a + 6, azz);
          }
          adj_add(a + 7, axy);
          adj_add(a + 8, ayz);
          adj_add(a + 9, azx);
          double cx = (double)acx.x + (double)acx.y + S * (double)m0.x;
          double cy = (double)acy.x + (double)acy.y + S * (double)m0.y;
          double cz = (double)acz.x + (double)acz.y + S * (double)m0.z;
          if constexpr (kWithE) {
            // + T (sum of 2 R2 g)
            const double Gx = (double)aGx.x + (double)aGx.y, Gy = (double)aGy.x + (double)aGy.y,
                         Gz = (double)aGz.x + (double)aGz.y;
            cx += (double)m0.w * Gx + (double)m1.z * Gy + (double)m2.x * Gz;
            cy += (double)m1.z * Gx + (double)m1.x * Gy + (double)m1.w * Gz;
            cz += (double)m2.x * Gx + (double)m1.w * Gy + (double)m1.y * Gz;
          }
          if (cx != 0.0) atomicAdd(a + 10, cx);
          if (cy != 0.0) atomicAdd(a + 11, cy);
          if (cz != 0.0) atomicAdd(a + 12, cz);
        }
        c_twig += (unsigned)n * (unsigned)nvalid;
        hT = (hT + n) & (kRing - 1);
        nT -= n;
        __syncwarp();
      };
      // leaf records: qbar += gphi R0 (+ g.d R1), cocbar += q [(gphi R1 (+ 3 g.d R2)) d (- R1 g)]
      auto flush_leaves = [&](int n) {
        __syncwarp();
        if (lane < n) {
          const StagedLeafA& r = stl[(hL + lane) & (kRing - 1)];
          const float4 c = r.c;
          const float2 NCX = f2(-c.x), NCY = f2(-c.y), NCZ = f2(-c.z);  // d = r_t - c
          float2 aq = f2(0.f), acx = f2(0.f), acy = f2(0.f), acz = f2(0.f);
          unsigned long long pend = 0ull;  // targets at a zero FP32 offset (bit 2p + half)
#pragma unroll 2
          for (int p = 0; p < 32; ++p) {
            const float4 ta4 = tg[p][0], tb4 = tg[p][1];
            const float2 dx = __fadd2_rn(make_float2(ta4.x, ta4.y), NCX);
            const float2 dy = __fadd2_rn(make_float2(ta4.z, ta4.w), NCY);
            const float2 dz = __fadd2_rn(make_float2(tb4.x, tb4.y), NCZ);
            const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            const bool za = d2.x == 0.f, zb = d2.y == 0.f;
            pend |= (za ? 1ull << (2 * p) : 0ull) | (zb ? 2ull << (2 * p) : 0ull);
            const float2 gp = make_float2(za ? 0.f : tb4.z, zb ? 0.f : tb4.w);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, E2)));
            const float2 R0 = make_float2(r2.x > 0.f ? rsqrt_ftz(r2.x) : 0.f,
                                          r2.y > 0.f ? rsqrt_ftz(r2.y) : 0.f);
            const float2 R1 = __fmul2_rn(R0, __fmul2_rn(R0, R0));
            aq = __ffma2_rn(gp, R0, aq);
            float2 k = __fmul2_rn(gp, R1);
            if constexpr (kWithE) {
              const float4 tc4 = tg[p][2], td4 = tg[p][3];
              const float2 gxx = make_float2(za ? 0.f : tc4.x, zb ? 0.f : tc4.y);
              const float2 gyy = make_float2(za ? 0.f : tc4.z, zb ? 0.f : tc4.w);
              const float2 gzz = make_float2(za ? 0.f : td4.x, zb ? 0.f : td4.y);
              const float2 ga = __ffma2_rn(gxx, dx, __ffma2_rn(gyy, dy, __fmul2_rn(gzz, dz)));
              const float2 R2 = __fmul2_rn(R1, __fmul2_rn(R0, R0));
              aq = __ffma2_rn(ga, R1, aq);
              k = __ffma2_rn(__fmul2_rn(f2(3.f), ga), R2, k);
              const float2 nR1 = __fmul2_rn(f2(-1.f), R1);
              acx = __ffma2_rn(nR1, gxx, acx);
              acy = __ffma2_rn(nR1, gyy, acy);
              acz = __ffma2_rn(nR1, gzz, acz);
            }
            acx = __ffma2_rn(k, dx, acx);
            acy = __ffma2_rn(k, dy, acy);
            acz = __ffma2_rn(k, dz, acz);
          }
          // zero FP32 offsets: the target's own leaf (no interaction, FP64
          // dist2 == 0) or a point closer than FP32 resolves at the group
          // scale, evaluated on the FP64 offset rounded once
          float sq = 0.f, scx = 0.f, scy = 0.f, scz = 0.f;
          while (pend) {
            const int bit = __ffsll((long long)pend) - 1;
            pend &= pend - 1;
            const int64_t t = t0 + (bit >> 1) + 32 * (bit & 1);
            const double ex = (A.tx[t] - vx) - r.x, ey = (A.ty[t] - vy) - r.y,
                         ez = (A.tz[t] - vz) - r.z;
            if (ex == 0.0 && ey == 0.0 && ez == 0.0) continue;
            const float dx = (float)ex, dy = (float)ey, dz = (float)ez;
            const float gp = (float)A.gphi[t];
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, A.eps2)));
            const float R0 = rsqrt_ftz(r2), R1 = R0 * R0 * R0;
            sq = fmaf(gp, R0, sq);
            float k = gp * R1;
            if constexpr (kWithE) {
              const float gx = (float)A.gex[t], gy = (float)A.gey[t], gz = (float)A.gez[t];
              const float ga = fmaf(gx, dx, fmaf(gy, dy, gz * dz));
              sq = fmaf(ga, R1, sq);
              k = fmaf(3.f * ga, R1 * R0 * R0, k);
              scx = fmaf(-R1, gx, scx);
              scy = fmaf(-R1, gy, scy);
              scz = fmaf(-R1, gz, scz);
            }
            scx = fmaf(k, dx, scx);
            scy = fmaf(k, dy, scy);
            scz = fmaf(k, dz, scz);
          }
          double* a = A.adj + (int64_t)kNAdj * r.node;
          const double q = (double)c.w;
          const double vq = (double)aq.x + (double)aq.y + (double)sq;
          if (vq != 0.0) atomicAdd(a + 0, vq);
          const double cx = q * ((double)acx.x + (double)acx.y + (double)scx);
          const double cy = q * ((double)acy.x + (double)acy.y + (double)scy);
          const double cz = q * ((double)acz.x + (double)acz.y + (double)scz);
          if (cx != 0.0) atomicAdd(a + 10, cx);
          if (cy != 0.0) atomicAdd(a + 11, cy);
          if (cz != 0.0) atomicAdd(a + 12, cz);
        }
        c_leaf += (unsigned)n * (unsigned)nvalid;
        hL = (hL + n) & (kRing - 1);
        nL -= n;
        __syncwarp();
      };
      // the traversal and MAC of k_walk_group64 (same decisions, same lists)
      while (top > 0) {
        const int take = top < 32 ? top : 32;
        top -= take;
        const int node = lane < take ? stack[top + lane] : -1;
        __syncwarp();
        bool isleaf = false, accept = false, open = false, amb = false;
        float cx = 0.f, cy = 0.f, cz = 0.f, bl = 0.f;
        double4 a = make_double4(0, 0, 0, 0);
        // the node's level-ordered record and links (k_walk_group64's traversal);
        // the adjoint records are in the same level order
        int4 lk = make_int4(0, 0, 0, 0);
        if (node >= 0) {
          const LevelRecord* rec = A.drec + node;
          a = ld256(&rec->pos);
          lk = rec->link;
          cx = (float)(a.x - gx); cy = (float)(a.y - gy); cz = (float)(a.z - gz);
          if (lk.y & kLeafFlag) {
            isleaf = true;
          } else {
            bl = A.macb ? (float)A.macb[lk.w] : s_bl2[lk.y & 0xff];
            const float dc = sqrtf(cx * cx + cy * cy + cz * cz);
            const float dmin = dc - rg, dmax = dc + rg;
            if (dmin > 0.f && theta2 * (dmin * dmin) > bl) {
              accept = true;
              c_mac += 1;
            } else if (!(theta2 * (dmax * dmax) > bl)) {
              open = true;
              c_mac += 1;
            } else {
              amb = true;
            }
          }
        }
        unsigned am = __ballot_sync(0xffffffffu, amb);
        while (am) {
          const int j = __ffs(am) - 1;
          am &= am - 1;
          const float ux = __shfl_sync(0xffffffffu, cx, j);
          const float uy = __shfl_sync(0xffffffffu, cy, j);
          const float uz = __shfl_sync(0xffffffffu, cz, j);
          const float ub = __shfl_sync(0xffffffffu, bl, j);
          float dx = rxa - ux, dy = rya - uy, dz = rza - uz;
          const bool fa = v0 && !(theta2 * fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > ub);
          dx = rxb - ux; dy = ryb - uy; dz = rzb - uz;
          const bool fb = v1 && !(theta2 * fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > ub);
          const unsigned f0 = __ballot_sync(0xffffffffu, fa);
          const unsigned f1 = __ballot_sync(0xffffffffu, fb);
          if (lane == j) {
            accept = (f0 | f1) == 0;
            open = !accept;
            c_mac += (unsigned)(f0 ? __popc(vm0 & ((2u << (__ffs(f0) - 1)) - 1u))
                                   : __popc(vm0) + (f1 ? __popc(vm1 & ((2u << (__ffs(f1) - 1)) - 1u))
                                                       : __popc(vm1)));
          }
        }
        const unsigned lb = __ballot_sync(0xffffffffu, isleaf);
        const unsigned ab = __ballot_sync(0xffffffffu, accept);
        if (isleaf) {
          StagedLeafA& r = stl[(hL + nL + __popc(lb & lt)) & (kRing - 1)];
          r.c = make_float4(cx, cy, cz, (float)a.w);
          r.x = a.x; r.y = a.y; r.z = a.z;
          r.node = node;
          partner += 1;
        }
        if (accept) {
          StagedTwig& r = stw[(hT + nT + __popc(ab & lt)) & (kRing - 1)];
          r.c = make_float4(-cx, -cy, -cz, __int_as_float(node));
          const float4* m = A.mom32 + kMom32Stride * (int64_t)lk.w;
          cp_async16(&r.m0, m);
          cp_async16(&r.m1, m + 1);
          cp_async16(&r.m2, m + 2);
          partner += lk.z;
        }
        nL += __popc(lb);
        nT += __popc(ab);
        const int npush = open ? min(8, lk.y >> 16) : 0;
        int total;
        const int off = warp_excl_scan(npush, lane, total);
        if (top + total > kStackCap) {
          complete = false;
          break;
        }
        if (npush > 0) {
          int* dst = stack + top + off;
#pragma unroll
          for (int k = 0; k < 8; ++k)
            if (k < npush) dst[k] = lk.x + k;
        }
        top += total;
        __syncwarp();
        if (nT >= 32) flush_twigs(32);
        if (nL >= 32) flush_leaves(32);
      }
      if (nT > 0) flush_twigs(nT);
      if (nL > 0) flush_leaves(nL);
      for (int o = 16; o > 0; o >>= 1) partner += __shfl_xor_sync(0xffffffffu, partner, o);
      if (partner != A.npart) complete = false;
    }
    __syncwarp();
    if (__any_sync(0xffffffffu, !complete) && lane == 0) atomicOr(A.status, ST_INCOMPLETE);
  }
  cp_async_wait_all();
  warp_add3(A.counters, c_leaf, c_twig, c_mac);
}

__global__ void k_reset_mixed(unsigned int* q) { *q = 0; }

}  // namespace

int launch_walk_mixed(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                      double* ex, double* ey, double* ez, double* pot, double* work,
                      const int2* tiles, int64_t ntiles, bool per_target,
                      const int32_t* tflag, const int32_t* pstart, const int32_t* npacks,
                      cudaStream_t s, int slot) {
  MixArgs A;
  A.nt = nt;
  A.tx = tx; A.ty = ty; A.tz = tz;
  A.nc4 = c->nc4.p;
  A.meta = c->meta.p;
  A.mom32 = reinterpret_cast<const float4*>(c->mom32.p);
  A.nleaves = c->nleaves.p;
  A.drec = c->drec.p;
  A.bl2 = c->d_box + 9;
  {
    int rc = prepare_mac(c, &A.macb);
    if (rc) return rc;
  }
  A.vbox = c->d_vbox;
  A.nbox = c->nboxes;
  A.theta2 = (float)c->prm.theta2;
  A.theta2d = c->prm.theta2;
  A.eps2 = (float)c->prm.eps2;
  A.M = (int32_t)c->nnodes;
  A.npart = c->n;
  A.ex = ex; A.ey = ey; A.ez = ez; A.pot = pot; A.work = work;
  A.counters = c->counters.p;
  A.status = c->d_status;
  A.queue = c->walk_queue(slot);
  A.tiles = tiles;
  A.ntiles = ntiles;
  A.fwd = c->fwd.p;
  A.fwdf = c->fwdf.p;
  A.tflag = tflag;
  A.pstart = pstart;
  A.npacks = npacks;
  COUNT_LAUNCH();
  k_reset_mixed<<<1, 1, 0, s>>>(A.queue);
  COUNT_LAUNCH();
  if (per_target) {
    k_walk_target_mixed<<<148 * 8, kMixThreads, 0, s>>>(A);
  } else if (tflag) {
    k_walk_tilepack_mixed<<<148 * 8, kMixThreads, 0, s>>>(A);
  } else {
    // 5 resident blocks per SM (launch bounds: at most 96 registers; the
    // 64-target walk holds 39 KB of shared memory per block); the grid is
    // exactly one wave.  One set of stacks per walk stream.
    const int gblocks = 148 * 5;
    const size_t per = (size_t)gblocks * kWW * kStackCap;
    if (!ensure(c, c->wstack, 2 * per, "walk stacks")) return PEPCG_ERR_OOM;
    if (c->prm.precision == PEPCG_PRECISION_MIXED_STRICT)  // 4 blocks per SM
      k_walk_group64<true><<<148 * 4, kMixThreads, 0, s>>>(A, c->wstack.p + slot * per);
    else if (tiles == nullptr && c->group_size() == 64)
      k_walk_group64<false><<<gblocks, kMixThreads, 0, s>>>(A, c->wstack.p + slot * per);
    else
      k_walk_group_wide<<<gblocks, kMixThreads, 0, s>>>(A, c->wstack.p + slot * per, c->child8.p,
                                                        c->nchild.p);
  }
  return cuda_ok(c, cudaGetLastError(), "mixed walk launch") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

// The adjoint walk of the mixed group walk with 64-target buckets: fills the
// twigs' and leaves' adjoint records (adj, 16 doubles per node, zeroed by the
// caller); the downward pass and the output are adjoint.cu's.
int launch_adjoint_group64(Ctx* c, int64_t nt, const double* tx, const double* ty,
                           const double* tz, const double* gex, const double* gey,
                           const double* gez, const double* gphi, bool with_e, cudaStream_t s) {
  AdjMixArgs A;
  A.nt = nt;
  A.tx = tx; A.ty = ty; A.tz = tz;
  A.gex = gex; A.gey = gey; A.gez = gez; A.gphi = gphi;
  A.nc4 = c->nc4.p;
  A.meta = c->meta.p;
  A.mom32 = reinterpret_cast<const float4*>(c->mom32.p);
  A.nleaves = c->nleaves.p;
  A.drec = c->drec.p;
  A.bl2 = c->d_box + 9;
  {
    int rc = prepare_mac(c, &A.macb);
    if (rc) return rc;
  }
  A.vbox = c->d_vbox;
  A.nbox = c->nboxes;
  A.theta2 = (float)c->prm.theta2;
  A.eps2 = (float)c->prm.eps2;
  A.npart = c->n;
  A.adj = c->adj.p;
  A.counters = c->counters.p;
  A.status = c->d_status;
  A.queue = c->walk_queue();
  const int gblocks = 148 * 4;
  const size_t per = (size_t)gblocks * kWW * kStackCap;
  if (!ensure(c, c->wstack, 2 * per, "walk stacks")) return PEPCG_ERR_OOM;
  COUNT_LAUNCH();
  k_reset_mixed<<<1, 1, 0, s>>>(A.queue);
  COUNT_LAUNCH();
  if (with_e)
    k_adj_group64<true><<<gblocks, kMixThreads, 0, s>>>(A, c->wstack.p);
  else
    k_adj_group64<false><<<gblocks, kMixThreads, 0, s>>>(A, c->wstack.p);
  return cuda_ok(c, cudaGetLastError(), "mixed adjoint launch") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

}  // namespace pepcg
