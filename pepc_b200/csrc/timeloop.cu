// timeloop.cu -- the frontend's time step around the path, on the device, so
// the particles can stay in HBM from one step to the next:
//   push        pepc-mini push_particles (module_helper.f90:205-222):
//               v += dt q/m E, then x += dt v;
//   ext. field  apply_external_field (module_helper.f90:321-334):
//               E_z += ez_ext, pot -= z ez_ext;
//   wrap        constrain_periodic (module_mirror_boxes.f90:177-218): modulo
//               into the box along the axes (principal-axes lattice) or in
//               lattice coordinates through the inverse lattice matrix
//               (inverse3, module_math_tools.f90:114-150);
//   gather      out[i] = in[perm[i]]: carries per-particle state (velocity,
//               mass, ...) into the key order of the last grow, as the
//               reference's domain_decompose moves whole particle records;
//   restore     out[perm[i]] = in[i]: the way back to the input order
//               (domain_restore, module_domains.f90:372-408);
//   energy      the potential energy of pepc-b's diagnostics (potenergy,
//               frontends/pepc-b/module_diagnostics.f90:227-263): the sum of
//               0.5 q phi in FP64, block partials added in block order.
// Compiled with --fmad=false, so every result is the reference expression in
// its order, rounded once per operation.

#include <cmath>

#include "internal.cuh"

namespace pepcg {
namespace {

constexpr int kTL = 256;

inline unsigned grid_of(int64_t n) {
  int64_t b = (n + kTL - 1) / kTL;
  if (b > 148 * 32) b = 148 * 32;
  return (unsigned)(b < 1 ? 1 : b);
}

__global__ void k_push(int64_t n, double dt, const double* __restrict__ q,
                       const double* __restrict__ m, const double* __restrict__ ex,
                       const double* __restrict__ ey, const double* __restrict__ ez, double* vx,
                       double* vy, double* vz, double* x, double* y, double* z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double f = dt * q[i] / m[i];
    const double nvx = vx[i] + f * ex[i], nvy = vy[i] + f * ey[i], nvz = vz[i] + f * ez[i];
    vx[i] = nvx; vy[i] = nvy; vz[i] = nvz;
    x[i] = x[i] + dt * nvx;
    y[i] = y[i] + dt * nvy;
    z[i] = z[i] + dt * nvz;
  }
}

__global__ void k_external_field(int64_t n, double ez_ext, const double* __restrict__ z,
                                 double* ez, double* pot) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    ez[i] = ez[i] + ez_ext;
    pot[i] = pot[i] - z[i] * ez_ext;
  }
}

// Fortran MODULO for reals: the exact remainder with the sign of the divisor
__device__ __forceinline__ double fmodulo(double a, double p) {
  double r = fmod(a, p);
  if (r != 0.0 && ((r < 0.0) != (p < 0.0))) r = r + p;
  return r;
}

struct Wrap {
  double L[3][3], Li[3][3], o[3], walls[3];
  int per[3];
  int simple;
};

__global__ void k_wrap(int64_t n, Wrap w, double* x, double* y, double* z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double c[3] = {x[i], y[i], z[i]};
    if (w.simple) {
      for (int d = 0; d < 3; ++d)
        if (w.per[d]) c[d] = fmodulo(c[d] - w.o[d], w.walls[d]) + w.o[d];
    } else {
      const double v[3] = {c[0] - w.o[0], c[1] - w.o[1], c[2] - w.o[2]};
      double lc[3];
      bool out = false;
      for (int j = 0; j < 3; ++j) {
        lc[j] = (v[0] * w.Li[0][j] + v[1] * w.Li[1][j]) + v[2] * w.Li[2][j];
        if (lc[j] > 1.0 || lc[j] < 0.0) out = true;
      }
      if (out) {
        for (int j = 0; j < 3; ++j) lc[j] = fmodulo(lc[j], 1.0);
        for (int j = 0; j < 3; ++j)
          if (w.per[j]) c[j] = ((lc[0] * w.L[0][j] + lc[1] * w.L[1][j]) + lc[2] * w.L[2][j]) + w.o[j];
      }
    }
    x[i] = c[0]; y[i] = c[1]; z[i] = c[2];
  }
}

__global__ void k_gather(int64_t n, const int32_t* __restrict__ perm, const double* __restrict__ in,
                         double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}

__global__ void k_scatter(int64_t n, const int32_t* __restrict__ perm, const double* __restrict__ in,
                          double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[perm[i]] = in[i];
}

__global__ void k_widen(int64_t n, const int32_t* __restrict__ in, int64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}

// partial sums of (0.5 q) phi (the reference's 0.5 * q(p) * pot(p), left to
// right) over a grid-stride range, one per block
constexpr int kEpotBlocks = 296;
__global__ void __launch_bounds__(kTL) k_epot_partial(int64_t n, const double* __restrict__ q,
                                                      const double* __restrict__ pot,
                                                      double* __restrict__ part) {
  __shared__ double sw[kTL / 32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    s = s + (0.5 * q[i]) * pot[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kTL / 32; ++w) t = t + sw[w];
    part[blockIdx.x] = t;
  }
}

__global__ void k_epot_final(int nb, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double t = 0.0;
  for (int b = 0; b < nb; ++b) t = t + part[b];
  *out = t;
}

}  // namespace

int potential_energy_device(Ctx* c, int64_t n, const double* q, const double* pot,
                            double* epot) {
  cudaStream_t s = c->stream;
  double* part = c->d_part;  // 6 * 512 doubles: kEpotBlocks partials and the total
  COUNT_LAUNCH();
  k_epot_partial<<<kEpotBlocks, kTL, 0, s>>>(n, q, pot, part);
  COUNT_LAUNCH();
  k_epot_final<<<1, 32, 0, s>>>(kEpotBlocks, part, part + kEpotBlocks);
  if (!cuda_ok(c, cudaGetLastError(), "potential energy") ||
      !cuda_ok(c, cudaMemcpyAsync(epot, part + kEpotBlocks, sizeof(double),
                                  cudaMemcpyDeviceToHost, s), "potential energy") ||
      !cuda_ok(c, cudaStreamSynchronize(s), "potential energy"))
    return PEPCG_ERR_CUDA;
  return PEPCG_OK;
}

int push_device(Ctx* c, int64_t n, double dt, const double* q, const double* m, const double* ex,
                const double* ey, const double* ez, double* vx, double* vy, double* vz, double* x,
                double* y, double* z) {
  COUNT_LAUNCH();
  k_push<<<grid_of(n), kTL, 0, c->stream>>>(n, dt, q, m, ex, ey, ez, vx, vy, vz, x, y, z);
  return cuda_ok(c, cudaGetLastError(), "push") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int external_field_device(Ctx* c, int64_t n, double ez_ext, const double* z, double* ez,
                          double* pot) {
  COUNT_LAUNCH();
  k_external_field<<<grid_of(n), kTL, 0, c->stream>>>(n, ez_ext, z, ez, pot);
  return cuda_ok(c, cudaGetLastError(), "external field") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int wrap_device(Ctx* c, int64_t n, double* x, double* y, double* z) {
  const pepcg_params& p = c->prm;
  Wrap w;
  for (int j = 0; j < 3; ++j) {
    w.L[0][j] = p.t_lattice_1[j];
    w.L[1][j] = p.t_lattice_2[j];
    w.L[2][j] = p.t_lattice_3[j];
    w.o[j] = p.lattice_origin[j];
    w.per[j] = p.periodicity[j] != 0;
  }
  w.walls[0] = p.t_lattice_1[0];
  w.walls[1] = p.t_lattice_2[1];
  w.walls[2] = p.t_lattice_3[2];
  // system_uses_principal_axes (module_mirror_boxes.f90:231-242)
  w.simple = p.t_lattice_1[0] > 0.0 && p.t_lattice_1[1] == 0.0 && p.t_lattice_1[2] == 0.0 &&
             p.t_lattice_2[0] == 0.0 && p.t_lattice_2[1] > 0.0 && p.t_lattice_2[2] == 0.0 &&
             p.t_lattice_3[0] == 0.0 && p.t_lattice_3[1] == 0.0 && p.t_lattice_3[2] > 0.0;
  // inverse3: Cramer's rule, the 2x2 determinants in the reference's order
  auto m = [&](int i, int j) { return w.L[i - 1][j - 1]; };
  const double det = m(1, 1) * m(2, 2) * m(3, 3) + m(1, 2) * m(2, 3) * m(3, 1) +
                              m(1, 3) * m(2, 1) * m(3, 2) - m(1, 3) * m(2, 2) * m(3, 1) -
                              m(1, 2) * m(2, 1) * m(3, 3) - m(1, 1) * m(2, 3) * m(3, 2);
  if (det == 0.0) {
    c->err = "pepcg_constrain_periodic: the lattice vectors are linearly dependent";
    return PEPCG_ERR_BAD_ARG;
  }
  auto d2 = [](double a, double b, double cc, double d) { return a * d - b * cc; };
  w.Li[0][0] = d2(m(2, 2), m(3, 2), m(2, 3), m(3, 3)) / det;
  w.Li[1][0] = d2(m(2, 3), m(3, 3), m(2, 1), m(3, 1)) / det;
  w.Li[2][0] = d2(m(2, 1), m(3, 1), m(2, 2), m(3, 2)) / det;
  w.Li[0][1] = d2(m(1, 3), m(3, 3), m(1, 2), m(3, 2)) / det;
  w.Li[1][1] = d2(m(1, 1), m(3, 1), m(1, 3), m(3, 3)) / det;
  w.Li[2][1] = d2(m(1, 2), m(3, 2), m(1, 1), m(3, 1)) / det;
  w.Li[0][2] = d2(m(1, 2), m(2, 2), m(1, 3), m(2, 3)) / det;
  w.Li[1][2] = d2(m(1, 3), m(2, 3), m(1, 1), m(2, 1)) / det;
  w.Li[2][2] = d2(m(1, 1), m(2, 1), m(1, 2), m(2, 2)) / det;
  COUNT_LAUNCH();
  k_wrap<<<grid_of(n), kTL, 0, c->stream>>>(n, w, x, y, z);
  return cuda_ok(c, cudaGetLastError(), "constrain periodic") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int gather_device(Ctx* c, const double* in, double* out) {
  COUNT_LAUNCH();
  k_gather<<<grid_of(c->n), kTL, 0, c->stream>>>(c->n, c->perm.p, in, out);
  return cuda_ok(c, cudaGetLastError(), "gather") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int restore_device(Ctx* c, const double* in, double* out) {
  COUNT_LAUNCH();
  k_scatter<<<grid_of(c->n), kTL, 0, c->stream>>>(c->n, c->perm.p, in, out);
  return cuda_ok(c, cudaGetLastError(), "restore") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int widen_perm_device(Ctx* c, int64_t* out, cudaStream_t st, const int32_t* src) {
  COUNT_LAUNCH();
  k_widen<<<grid_of(c->n), kTL, 0, st ? st : c->stream>>>(c->n, src ? src : c->perm.p, out);
  return cuda_ok(c, cudaGetLastError(), "perm") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

}  // namespace pepcg
