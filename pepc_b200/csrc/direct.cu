// direct.cu -- FP64 direct sum on sampled targets (utils/module_directsum.f90:34-172):
// every key-ordered particle acts on each target through every near-field
// box (central box last); the target itself is skipped in the central box
// (:119-124); the lattice term follows when the context is periodic.
// Each block handles kTB targets and streams all sources once; partial sums
// are combined by a block reduction (summation order differs from the
// reference's sequential loop, so results agree to rounding, not bitwise).
// Compiled with --fmad=false.

#include <cmath>

#include "internal.cuh"

namespace pepcg {
namespace {

constexpr int kTB = 8;
constexpr int kDThreads = 256;

template <int kLaw>
__global__ void __launch_bounds__(kDThreads)
k_direct(int64_t ntest, const int64_t* __restrict__ tidx, int64_t n, const double* __restrict__ x,
         const double* __restrict__ y, const double* __restrict__ z, const double* __restrict__ q,
         const double* __restrict__ vbox, int nbox, double eps2, double kinv, double sqrtpi,
         double* __restrict__ ex, double* __restrict__ ey, double* __restrict__ ez,
         double* __restrict__ pot) {
  __shared__ double s_vb[3 * 125];
  __shared__ double red[kDThreads / 32][kTB * 4];
  for (int i = threadIdx.x; i < 3 * nbox; i += blockDim.x) s_vb[i] = vbox[i];
  __syncthreads();
  const int64_t t0 = (int64_t)blockIdx.x * kTB;
  int64_t tj[kTB];
  double tx[kTB], ty[kTB], tz[kTB], tq[kTB];
  double acc[kTB][4];
#pragma unroll
  for (int k = 0; k < kTB; ++k) {
    int64_t t = t0 + k < ntest ? t0 + k : ntest - 1;
    tj[k] = t0 + k < ntest ? tidx[t] : -2;
    int64_t jj = tidx[t];
    tx[k] = x[jj];
    ty[k] = y[jj];
    tz[k] = z[jj];
    tq[k] = q[jj];
    acc[k][0] = acc[k][1] = acc[k][2] = acc[k][3] = 0.0;
  }
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
    const double xs = x[j], ys = y[j], zs = z[j], qs = q[j];
    for (int ib = 0; ib < nbox; ++ib) {
      const double vx = s_vb[3 * ib], vy = s_vb[3 * ib + 1], vz = s_vb[3 * ib + 2];
      const bool central = (ib == nbox - 1);
#pragma unroll
      for (int k = 0; k < kTB; ++k) {
        if (central && tj[k] == j) continue;
        const double dx = (tx[k] - vx) - xs, dy = (ty[k] - vy) - ys, dz = (tz[k] - vz) - zs;
        const double dist2 = (dx * dx + dy * dy) + dz * dz;
        double fx, fy, fz, fp;
        law_leaf64<kLaw>(qs, dx, dy, dz, dist2, eps2, fx, fy, fz, fp,
                         KelbgArgs{tq[k], kinv, sqrtpi});
        acc[k][0] += fx;
        acc[k][1] += fy;
        acc[k][2] += fz;
        acc[k][3] += fp;
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kTB; ++k)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double v = acc[k][c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][4 * k + c] = v;
    }
  __syncthreads();
  if (threadIdx.x < kTB * 4) {
    double v = 0.0;
    for (int w = 0; w < kDThreads / 32; ++w) v += red[w][threadIdx.x];
    const int k = threadIdx.x / 4, c = threadIdx.x % 4;
    const int64_t t = t0 + k;
    if (t < ntest) {
      double* out = c == 0 ? ex : c == 1 ? ey : c == 2 ? ez : pot;
      out[t] = v;
    }
  }
}

__global__ void k_gather_pos(int64_t nt, const int64_t* __restrict__ tidx, const double* __restrict__ x,
                             const double* __restrict__ y, const double* __restrict__ z,
                             double* __restrict__ o) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nt;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = tidx[i];
    o[i] = x[j];
    o[nt + i] = y[j];
    o[2 * nt + i] = z[j];
  }
}

}  // namespace

int direct_device(Ctx* c, int64_t ntest, const int64_t* d_tidx, double* ex, double* ey,
                  double* ez, double* pot) {
  cudaStream_t s = c->stream;
  const int64_t nb = (ntest + kTB - 1) / kTB;
  COUNT_LAUNCH();
  const int law = c->prm.force_law;
  auto kern = law == 2 ? k_direct<2> : law == 4 ? k_direct<4> : law == 5 ? k_direct<5> : k_direct<3>;
  kern<<<(unsigned)nb, kDThreads, 0, s>>>(ntest, d_tidx, c->n, c->x.p, c->y.p, c->z.p, c->q.p,
                                          c->d_vbox, c->nboxes, c->prm.eps2,
                                          c->prm.kelbg_invsqrttemp, std::sqrt(std::acos(-1.0)), ex,
                                          ey, ez, pot);
  if (!cuda_ok(c, cudaGetLastError(), "direct launch")) return PEPCG_ERR_CUDA;
  if (c->far_field) {
    double* pos = nullptr;
    if (!cuda_ok(c, cudaMallocAsync((void**)&pos, 3 * ntest * sizeof(double), s), "direct pos"))
      return PEPCG_ERR_OOM;
    COUNT_LAUNCH();
    k_gather_pos<<<148, 256, 0, s>>>(ntest, d_tidx, c->x.p, c->y.p, c->z.p, pos);
    int rc = lattice_add(c, ntest, pos, pos + ntest, pos + 2 * ntest, ex, ey, ez, pot, false);
    cudaFreeAsync(pos, s);
    if (rc) return rc;
  }
  return PEPCG_OK;
}

}  // namespace pepcg
