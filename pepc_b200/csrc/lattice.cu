// lattice.cu -- periodic far-lattice term of the Coulomb backend
// (interaction_specific/coulomb/module_fmm_framework.f90) on the device.
//
//  prepare  (fmm_framework_prepare, :100-126): lattice coefficients MLattice by
//           the iteration of calc_lattice_coefficients (:154-213).  For a
//           unit-cube lattice the reference loads a table that was produced by
//           that same iteration at Lmax_multipole = 50 (:253-259); running it
//           at 50 here reproduces the table's entries (to ~1e-14), the first
//           Lmax_taylor = 40 orders are kept, and the entries the table does
//           not list (odd l, m not a multiple of 4) are zero as there.
//  timestep (fmm_framework_timestep, :132-149): box dipole and quadrupole
//           trace, the central box's multipole expansion omega_tilde (l <= 20,
//           fictitious charges included) and mu_cent = M2L(MLattice, omega).
//  add      (fmm_sum_lattice_force, :766-826): per target, O(l <= 20) at the
//           target, L2L to l <= 1, E and phi, then the extrinsic correction.
//  adjoint  (no reference counterpart): the transpose of add and timestep for
//           L = sum_t dL/dphi_t phi_t + dL/dE_t . E_t, giving dL/dq, dL/dx of
//           the particles: targets -> dL/dmu -> dL/domega (M2L transposed) ->
//           particles through O_lm(x - center) and its gradient, plus the
//           fictitious charges' and the Redlack terms' chains through the box
//           dipole and quadrupole trace.
// Expansions use the flat layout tblinv(l, m) = l(l+1)/2 + m, m >= 0.
// Compiled with --fmad=false.

#include <cmath>
#include <vector>

#include "internal.cuh"

namespace pepcg {
namespace {

constexpr int kLM = 20;                    // Lmax_multipole
constexpr int kLT = 40;                    // Lmax_taylor
constexpr int kLenM = 231;
constexpr int kLenT = 861;
constexpr int kLMTable = 50;               // unit-cube table order
constexpr int kMaxIter = 32;

__device__ __forceinline__ int tblinv(int l, int m) { return l * (l + 1) / 2 + m; }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// tbl, :838-854
__device__ __forceinline__ double2 tbl(const double2* A, int l, int m, int lmax) {
  if (l > lmax || abs(m) > l) return make_double2(0.0, 0.0);
  double2 t = A[tblinv(l, abs(m))];
  if (m < 0) {
    double s = (m & 1) ? -1.0 : 1.0;
    t = make_double2(s * t.x, -s * t.y);
  }
  return t;
}

// LegendreP, :1196-1242
__device__ double legendre_p(int l, int m, double x) {
  double pll = 0.0, pmm = 1.0;
  if (m > 0) {
    double somx2 = sqrt((1.0 - x) * (1.0 + x));
    double fact = 1.0;
    for (int i = 1; i <= m; ++i) {
      pmm = (-pmm * fact) * somx2;
      fact = fact + 2.0;
    }
  }
  double r;
  if (l == m) {
    r = pmm;
  } else {
    double pmmp1 = (x * (2.0 * m + 1.0)) * pmm;
    if (l == m + 1) {
      r = pmmp1;
    } else {
      for (int ll = m + 2; ll <= l; ++ll) {
        pll = ((x * (2.0 * ll - 1.0)) * pmmp1 - ((double)(ll + m) - 1.0) * pmm) / (double)(ll - m);
        pmm = pmmp1;
        pmmp1 = pll;
      }
      r = pll;
    }
  }
  return ((m & 1) ? -1.0 : 1.0) * r;
}

// cartesian_to_spherical, :1083-1103 -> (r, cos theta, phi)
__device__ __forceinline__ void cart2sph(double cx, double cy, double cz, double s[3]) {
  s[0] = sqrt((cx * cx + cy * cy) + cz * cz);
  s[1] = (s[0] == 0.0) ? 1.0 : cz / s[0];
  s[2] = (cx == 0.0 && cy == 0.0) ? 0.0 : atan2(cy, cx);
}

// OMultipole, :695-714 (fact = factorial table)
__device__ __forceinline__ double2 omultipole(int l, int m, const double s[3], const double* fact) {
  double ph = (double)m * s[2];
  double sn, cs;
  sincos(ph, &sn, &cs);
  double pt = legendre_p(l, m, s[1]) / fact[l + m];
  double a = (s[0] > 0.0 || l > 0) ? pow(s[0], (double)l) * pt : pt;
  return make_double2(a * cs, a * -sn);
}

// MTaylor, :720-733
__device__ __forceinline__ double2 mtaylor(int l, int m, const double s[3], const double* fact) {
  double ph = (double)m * s[2];
  double sn, cs;
  sincos(ph, &sn, &cs);
  double p2 = legendre_p(l, m, s[1]) * fact[l - m];
  double a = (1.0 / pow(s[0], (double)(l + 1))) * p2;
  return make_double2(a * cs, a * sn);
}

// sort_abs, :1321-1367 (heap sort by magnitude) on a strided global slice
__device__ void sort_abs(double* a, int n) {
  auto sift = [&](int l, int r) {
    double v = a[l - 1];
    int jold = l, j = l + l;
    for (;;) {
      if (j > r) break;
      if (j < r && fabs(a[j - 1]) < fabs(a[j])) j = j + 1;
      if (fabs(v) >= fabs(a[j - 1])) break;
      a[jold - 1] = a[j - 1];
      jold = j;
      j = j + j;
    }
    a[jold - 1] = v;
  };
  for (int i = n / 2; i >= 1; --i) sift(i, n);
  for (int i = n; i >= 2; --i) {
    double t = a[0];
    a[0] = a[i - 1];
    a[i - 1] = t;
    sift(1, i - 1);
  }
}

// MstarFunc, :1005-1036: one thread per (l, m), l <= lm
__global__ void k_mstar(int lm, int nb, const double* __restrict__ vbox, const double* fact,
                        double* scratch, double2* __restrict__ mstar) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int len = lm * (lm + 1) / 2 + lm + 1;
  if (idx >= len) return;
  int l = (int)((sqrt(8.0 * idx + 1.0) - 1.0) / 2.0);
  while (l * (l + 1) / 2 > idx) --l;
  while ((l + 1) * (l + 2) / 2 <= idx) ++l;
  int m = idx - l * (l + 1) / 2;
  double* rp = scratch + (int64_t)idx * 2 * nb;
  double* ip = rp + nb;
  for (int i = 0; i < nb; ++i) {
    double s[3];
    cart2sph(-vbox[3 * i], -vbox[3 * i + 1], -vbox[3 * i + 2], s);
    double2 t = omultipole(l, m, s, fact);
    rp[i] = t.x;
    ip[i] = t.y;
  }
  sort_abs(rp, nb);
  sort_abs(ip, nb);
  double r = 0.0, im = 0.0;
  for (int i = 0; i < nb; ++i) {
    r = r + rp[i];
    im = im + ip[i];
  }
  mstar[idx] = make_double2(r, im);
}

// LstarFunc, :1042-1077: one thread per (l, m), l <= lt
__global__ void k_lstar(int lt, int nb, int ws, const double* __restrict__ vbox, const double* fact,
                        double* scratch, double2* __restrict__ lstar) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int len = lt * (lt + 1) / 2 + lt + 1;
  if (idx >= len) return;
  int l = (int)((sqrt(8.0 * idx + 1.0) - 1.0) / 2.0);
  while (l * (l + 1) / 2 > idx) --l;
  while ((l + 1) * (l + 2) / 2 <= idx) ++l;
  int m = idx - l * (l + 1) / 2;
  const int cnt = nb * (nb - 1);
  double* rp = scratch + (int64_t)idx * 2 * cnt;
  double* ip = rp + cnt;
  int k = 0;
  const double f = (double)(2 * ws + 1);
  for (int i = 0; i < nb - 1; ++i)
    for (int ii = 0; ii < nb; ++ii) {
      double s[3];
      cart2sph(f * vbox[3 * i] + vbox[3 * ii], f * vbox[3 * i + 1] + vbox[3 * ii + 1],
               f * vbox[3 * i + 2] + vbox[3 * ii + 2], s);
      double2 t = mtaylor(l, m, s, fact);
      rp[k] = t.x;
      ip[k] = t.y;
      ++k;
    }
  sort_abs(rp, cnt);
  sort_abs(ip, cnt);
  double r = 0.0, im = 0.0;
  for (int i = 0; i < cnt; ++i) {
    r = r + rp[i];
    im = im + ip[i];
  }
  lstar[idx] = make_double2(r, im);
}

// one step of calc_lattice_coefficients: ML_new = M2L(UL(ML), Mstar) + Lstar
// (UL, :982-999; M2L, :912-937); scp[l] = (2 ws + 1)**(l + 1)
__global__ void k_lattice_iter(int lt, int lm, const double2* __restrict__ ML,
                               const double2* __restrict__ mstar, const double2* __restrict__ lstar,
                               const double* __restrict__ scp, double2* __restrict__ out) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int len = lt * (lt + 1) / 2 + lt + 1;
  if (idx >= len) return;
  int l = (int)((sqrt(8.0 * idx + 1.0) - 1.0) / 2.0);
  while (l * (l + 1) / 2 > idx) --l;
  while ((l + 1) * (l + 2) / 2 <= idx) ++l;
  int m = idx - l * (l + 1) / 2;
  double2 t = make_double2(0.0, 0.0);
  for (int j = 0; j <= lt; ++j) {
    const double sg = (j & 1) ? -1.0 : 1.0;
    for (int k = -j; k <= j; ++k) {
      const int ll = j + l, mm = k + m;
      double2 a = make_double2(0.0, 0.0);
      if (ll <= lt && abs(mm) <= ll) {
        double2 v = ML[tblinv(ll, abs(mm))];
        const double d = scp[ll];
        v = make_double2(v.x / d, v.y / d);  // UL
        if (mm < 0) {
          const double s = (mm & 1) ? -1.0 : 1.0;
          v = make_double2(s * v.x, -s * v.y);
        }
        a = v;
      }
      double2 b = tbl(mstar, j, k, lm);
      t = cadd(t, cmul(make_double2(sg * a.x, sg * a.y), b));
    }
  }
  out[idx] = cadd(t, lstar[idx]);
}

// keep the first Lmax_taylor orders of a table of order lt.  For the unit
// cube the reference starts from MLattice = 0 and loads only the entries of
// its table (fmm_framework_prepare, :112-115; load_lattice_coefficients,
// :260-508): l even and m a multiple of 4, as real numbers.  Every other entry
// stays zero there -- among them (1, 0) and (1, 1), which the iteration leaves
// at O(1) values (the conditionally convergent dipole sum) and which would
// otherwise couple the box dipole into phi -- so the same pattern is applied.
__global__ void k_truncate(const double2* __restrict__ src, double2* __restrict__ dst,
                           int unit_cube_table) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= kLenT) return;
  double2 v = src[idx];
  if (unit_cube_table) {
    int l = 0;
    while ((l + 1) * (l + 2) / 2 <= idx) ++l;
    const int m = idx - l * (l + 1) / 2;
    v = ((l & 1) == 0 && (m & 3) == 0) ? make_double2(v.x, 0.0) : make_double2(0.0, 0.0);
  }
  dst[idx] = v;
}

// box dipole and quadrupole trace (calc_box_dipole, :605-630): block partials
__global__ void k_box_dipole(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, const double* __restrict__ q,
                             double cx, double cy, double cz, double* __restrict__ part) {
  double a[4] = {0, 0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double r0 = x[i] - cx, r1 = y[i] - cy, r2 = z[i] - cz;
    a[0] = a[0] + q[i] * r0;
    a[1] = a[1] + q[i] * r1;
    a[2] = a[2] + q[i] * r2;
    a[3] = a[3] + q[i] * ((r0 * r0 + r1 * r1) + r2 * r2);
  }
  __shared__ double sm[4][8];
  for (int c = 0; c < 4; ++c) {
    double v = a[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[c][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int w = 0; w < 8; ++w) v += sm[threadIdx.x][w];
    part[4 * blockIdx.x + threadIdx.x] = v;
  }
}

// omega_tilde partials (calc_omega_tilde, :514-596).  Lane m (< 21) of each
// warp takes the order m of every harmonic of its particles: LegendreP's
// recurrence (:1196-1242) runs once up through l = 20, giving P_l^m for every
// l >= m in the same operations as a separate call per l; r^l is carried by
// multiplication and e^{-i m phi} comes from one sincos.  Each block sums a
// contiguous chunk of particles (warp partials added in shared memory).
constexpr int kOmChunk = 1024;
constexpr int kOmWarps = 8;
__global__ void __launch_bounds__(256) k_omega_partial(int64_t n, const double* __restrict__ x,
                                                       const double* __restrict__ y,
                                                       const double* __restrict__ z,
                                                       const double* __restrict__ q, double cx,
                                                       double cy, double cz, const double* fact,
                                                       double2* __restrict__ part) {
  __shared__ double2 s_acc[kOmWarps][kLenM];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m = lane;
  const int64_t base = (int64_t)blockIdx.x * kOmChunk;
  const int cnt = (int)min((int64_t)kOmChunk, n - base);
  double2 acc[kLM + 1];
#pragma unroll
  for (int l = 0; l <= kLM; ++l) acc[l] = make_double2(0.0, 0.0);
  if (m <= kLM) {
    for (int i = w; i < cnt; i += kOmWarps) {
      double sph[3];
      cart2sph(x[base + i] - cx, y[base + i] - cy, z[base + i] - cz, sph);
      const double qi = q[base + i];
      const double xc = sph[1];
      double sn, cs;
      sincos((double)m * sph[2], &sn, &cs);
      const double sg = (m & 1) ? -1.0 : 1.0;
      double pmm = 1.0;
      if (m > 0) {
        const double somx2 = sqrt((1.0 - xc) * (1.0 + xc));
        double f = 1.0;
        for (int k = 1; k <= m; ++k) {
          pmm = (-pmm * f) * somx2;
          f = f + 2.0;
        }
      }
      double pmmp1 = 0.0, rl = 1.0;
#pragma unroll
      for (int l = 0; l <= kLM; ++l) {
        if (l >= m) {
          double P;
          if (l == m) {
            P = pmm;
          } else if (l == m + 1) {
            pmmp1 = (xc * (2.0 * m + 1.0)) * pmm;
            P = pmmp1;
          } else {
            const double pll =
                ((xc * (2.0 * l - 1.0)) * pmmp1 - ((double)(l + m) - 1.0) * pmm) / (double)(l - m);
            pmm = pmmp1;
            pmmp1 = pll;
            P = pll;
          }
          const double pt = (sg * P) / fact[l + m];
          const double amp = (sph[0] > 0.0 || l > 0) ? rl * pt : pt;
          acc[l] = cadd(acc[l], make_double2(qi * (amp * cs), qi * (amp * -sn)));
        }
        rl = rl * sph[0];
      }
    }
  }
#pragma unroll
  for (int l = 0; l <= kLM; ++l)
    if (m <= l) s_acc[w][tblinv(l, m)] = acc[l];
  __syncthreads();
  for (int idx = threadIdx.x; idx < kLenM; idx += blockDim.x) {
    double2 t = s_acc[0][idx];
    for (int ww = 1; ww < kOmWarps; ++ww) t = cadd(t, s_acc[ww][idx]);
    part[(int64_t)blockIdx.x * kLenM + idx] = t;
  }
}

// sum the partials in block order, add the fictitious charges (:536-559),
// remove a net monopole (:570-573), then mu_cent = M2L(MLattice, omega)
__global__ void k_omega_final(int nparts, const double2* __restrict__ part, const double* aux,
                              double cx, double cy, double cz, const double* fact,
                              double2* __restrict__ omega, uint32_t* status) {
  const int idx = threadIdx.x;
  __shared__ double s_fict[4][4];
  __shared__ int s_nf;
  if (idx == 0) {
    s_nf = (int)aux[4];
    for (int p = 0; p < s_nf; ++p)
      for (int k = 0; k < 4; ++k) s_fict[p][k] = aux[8 + 4 * p + k];
  }
  __syncthreads();
  if (idx >= kLenM) return;
  int l = 0;
  while ((l + 1) * (l + 2) / 2 <= idx) ++l;
  const int m = idx - l * (l + 1) / 2;
  double2 acc = make_double2(0.0, 0.0);
  for (int b = 0; b < nparts; ++b) acc = cadd(acc, part[(int64_t)b * kLenM + idx]);
  for (int p = 0; p < s_nf; ++p) {
    double s[3];
    cart2sph(s_fict[p][0] - cx, s_fict[p][1] - cy, s_fict[p][2] - cz, s);
    double2 o = omultipole(l, m, s, fact);
    acc = cadd(acc, make_double2(s_fict[p][3] * o.x, s_fict[p][3] * o.y));
  }
  if (idx == 0 && hypot(acc.x, acc.y) > 0.0) {
    acc = make_double2(0.0, 0.0);
    atomicOr(status, ST_NOT_NEUTRAL);
  }
  omega[idx] = acc;
}

__global__ void k_mu_cent(const double2* __restrict__ ML, const double2* __restrict__ omega,
                          double2* __restrict__ mu) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= kLenT) return;
  int l = 0;
  while ((l + 1) * (l + 2) / 2 <= idx) ++l;
  int m = idx - l * (l + 1) / 2;
  double2 t = make_double2(0.0, 0.0);
  for (int j = 0; j <= kLT; ++j) {
    const double sg = (j & 1) ? -1.0 : 1.0;
    for (int k = -j; k <= j; ++k) {
      double2 a = tbl(ML, j + l, k + m, kLT);
      t = cadd(t, cmul(make_double2(sg * a.x, sg * a.y), tbl(omega, j, k, kLM)));
    }
  }
  mu[idx] = t;
}

// fictitious charges from the box dipole (single thread; :540-552)
__global__ void k_fict(int nbp, const double* __restrict__ part, double* aux, int p0, int p1,
                       int p2, const double* lat, const double* origin, int corr) {
  if (threadIdx.x != 0) return;
  double a[4] = {0, 0, 0, 0};
  for (int b = 0; b < nbp; ++b)
    for (int c = 0; c < 4; ++c) a[c] += part[4 * b + c];
  for (int c = 0; c < 4; ++c) aux[c] = a[c];
  int nf = 0;
  if (corr == 2) {
    int per[3] = {p0, p1, p2};
    double sum = 0.0;
    for (int p = 0; p < 3; ++p) {
      if (!per[p]) continue;
      const double* L = lat + 3 * p;
      for (int d = 0; d < 3; ++d) aux[8 + 4 * nf + d] = origin[d] + L[d];
      aux[8 + 4 * nf + 3] = -a[p] / sqrt((L[0] * L[0] + L[1] * L[1]) + L[2] * L[2]);
      ++nf;
    }
    for (int p = 0; p < nf; ++p) sum = sum + aux[8 + 4 * p + 3];
    for (int d = 0; d < 3; ++d) aux[8 + 4 * nf + d] = origin[d];
    aux[8 + 4 * nf + 3] = -sum;
    ++nf;
  }
  aux[4] = nf;
}

// fmm_sum_lattice_force per target (:766-826)
__global__ void __launch_bounds__(128) k_lattice_force(
    int64_t nt, const double* __restrict__ tx, const double* __restrict__ ty,
    const double* __restrict__ tz, const double2* __restrict__ mu, const double* __restrict__ aux,
    const double* __restrict__ vbox, int nbox, double cx, double cy, double cz, double volume,
    int corr, const double* fact, double* ex, double* ey, double* ez, double* pot, int overwrite) {
  __shared__ double2 s_mu[kLenM];  // only j <= Lmax_multipole entries are read by L2L
  __shared__ double s_aux[32];
  __shared__ double s_vb[3 * 125];
  __shared__ double s_fact[2 * kLM + 1];
  for (int i = threadIdx.x; i < kLenM; i += blockDim.x) s_mu[i] = mu[i];
  for (int i = threadIdx.x; i < 32; i += blockDim.x) s_aux[i] = aux[i];
  for (int i = threadIdx.x; i < 3 * nbox; i += blockDim.x) s_vb[i] = vbox[i];
  for (int i = threadIdx.x; i <= 2 * kLM; i += blockDim.x) s_fact[i] = fact[i];
  __syncthreads();
  const double pi = acos(-1.0);
  const double prefact = (2.0 * pi) / (3.0 * volume);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt;
       t += (int64_t)gridDim.x * blockDim.x) {
    const double px = tx[t], py = ty[t], pz = tz[t];
    const double R0 = px - cx, R1 = py - cy, R2 = pz - cz;
    double s[3];
    cart2sph(R0, R1, R2, s);
    // O_R(a, b) at the target (OMultipole, :695-714) times mu, L2L to l <= 1
    // (:943-976 with max_l = 1): output (l, m') collects O_R(a, b) mu(a + l,
    // b + m') over |b| <= a <= 20.  The harmonics are generated order by
    // order: for each m, one sincos, LegendreP's recurrence through a = 20
    // and r^a by multiplication, and O_R(a, -m) = (-1)^m conj(O_R(a, m)).
    double2 ms[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int m = 0; m <= kLM; ++m) {
      double sn, cs;
      sincos((double)m * s[2], &sn, &cs);
      const double sg = (m & 1) ? -1.0 : 1.0;
      const double xc = s[1];
      double pmm = 1.0;
      if (m > 0) {
        const double somx2 = sqrt((1.0 - xc) * (1.0 + xc));
        double f = 1.0;
        for (int k = 1; k <= m; ++k) {
          pmm = (-pmm * f) * somx2;
          f = f + 2.0;
        }
      }
      double rl = 1.0;
      for (int k = 0; k < m; ++k) rl = rl * s[0];
      double pmmp1 = 0.0;
      for (int a = m; a <= kLM; ++a) {
        double P;
        if (a == m) {
          P = pmm;
        } else if (a == m + 1) {
          pmmp1 = (xc * (2.0 * m + 1.0)) * pmm;
          P = pmmp1;
        } else {
          const double pll =
              ((xc * (2.0 * a - 1.0)) * pmmp1 - ((double)(a + m) - 1.0) * pmm) / (double)(a - m);
          pmm = pmmp1;
          pmmp1 = pll;
          P = pll;
        }
        const double pt = (sg * P) / s_fact[a + m];
        const double amp = (s[0] > 0.0 || a > 0) ? rl * pt : pt;
        rl = rl * s[0];
        const double2 o = make_double2(amp * cs, amp * -sn);
        ms[0] = cadd(ms[0], cmul(o, tbl(s_mu, a, m, kLM)));
        ms[1] = cadd(ms[1], cmul(o, tbl(s_mu, a + 1, m, kLM)));
        ms[2] = cadd(ms[2], cmul(o, tbl(s_mu, a + 1, m + 1, kLM)));
        if (m > 0) {
          const double2 on = make_double2(sg * o.x, -sg * o.y);
          ms[0] = cadd(ms[0], cmul(on, tbl(s_mu, a, -m, kLM)));
          ms[1] = cadd(ms[1], cmul(on, tbl(s_mu, a + 1, -m, kLM)));
          ms[2] = cadd(ms[2], cmul(on, tbl(s_mu, a + 1, -m + 1, kLM)));
        }
      }
    }
    double e0 = -ms[2].x, e1 = -ms[2].y, e2 = -ms[1].x, ph = ms[0].x;
    if (corr == 1) {
      e0 = e0 + (2.0 * prefact) * s_aux[0];
      e1 = e1 + (2.0 * prefact) * s_aux[1];
      e2 = e2 + (2.0 * prefact) * s_aux[2];
      double rd = (R0 * s_aux[0] + R1 * s_aux[1]) + R2 * s_aux[2];
      ph = (ph - (2.0 * prefact) * rd) + prefact * s_aux[3];
    } else if (corr == 2) {
      const int nf = (int)s_aux[4];
      for (int p = 0; p < nf; ++p) {
        const double fx = s_aux[8 + 4 * p], fy = s_aux[9 + 4 * p], fz = s_aux[10 + 4 * p];
        const double fq = s_aux[11 + 4 * p];
        for (int ib = 0; ib < nbox; ++ib) {
          const double d0 = (px - s_vb[3 * ib]) - fx, d1 = (py - s_vb[3 * ib + 1]) - fy,
                       d2 = (pz - s_vb[3 * ib + 2]) - fz;
          double gx, gy, gz, gp;
          force_leaf64(fq, d0, d1, d2, (d0 * d0 + d1 * d1) + d2 * d2, gx, gy, gz, gp);
          e0 = e0 + gx;
          e1 = e1 + gy;
          e2 = e2 + gz;
          ph = ph + gp;
        }
      }
    }
    if (overwrite) {
      ex[t] = e0; ey[t] = e1; ez[t] = e2; pot[t] = ph;
    } else {
      ex[t] += e0; ey[t] += e1; ez[t] += e2; pot[t] += ph;
    }
  }
}

// ---- adjoint of the lattice term ----
//
// With c00 = dL/dphi, c11 = -dL/dEx + i dL/dEy and c10 = -dL/dEz, one
// target contributes L_t = Re sum_{j, k} A(j, k) mu(j, k) over |k| <= j <= 20,
// A(j, k) = c00 O(j, k) + c11 O(j-1, k-1) + c10 O(j-1, k) (the L2L rows
// l <= 1).  Folding k < 0 onto k > 0 by mu(j, -m) = (-1)^m conj(mu(j, m)) and
// O(j, -m) = (-1)^m conj(O(j, m)) gives L_t = Re sum_{m >= 0} G(j, m) mu(j, m):
//   G(j, 0) = c00 O(j, 0) + c10 O(j-1, 0) - c11 conj(O(j-1, 1))
//   G(j, m) = 2 c00 O(j, m) + 2 c10 O(j-1, m) + c11 O(j-1, m-1)
//             - conj(c11) O(j-1, m+1)                          (m > 0)
// Lane m of a warp generates O(j, m) for j = 0..20 by LegendreP's recurrence
// (as the omega kernel) and takes O(j-1, m -+ 1) from lanes m -+ 1.  The
// extrinsic correction's adjoints ride along in xa: the fictitious charges'
// direct terms dL/dq_f (0..3), and for the Redlack form dL/d(dipole) (4..6)
// and dL/d(trace) (7).
constexpr int kLatAdjChunk = 1024;
__global__ void __launch_bounds__(256) k_latadj_targets(
    int64_t nt, const double* __restrict__ tx, const double* __restrict__ ty,
    const double* __restrict__ tz, const double* __restrict__ gex, const double* __restrict__ gey,
    const double* __restrict__ gez, const double* __restrict__ gphi, double cx, double cy,
    double cz, double prefact, int corr, const double* __restrict__ aux,
    const double* __restrict__ vbox, int nbox, const double* __restrict__ fact,
    double2* __restrict__ part, double* __restrict__ xpart) {
  __shared__ double2 s_acc[kOmWarps][kLenM];
  __shared__ double s_x[kOmWarps][8];
  __shared__ double s_aux[32];
  __shared__ double s_vb[3 * 125];
  __shared__ double s_fact[2 * kLM + 1];
  for (int i = threadIdx.x; i < 32; i += blockDim.x) s_aux[i] = aux[i];
  for (int i = threadIdx.x; i < 3 * nbox; i += blockDim.x) s_vb[i] = vbox[i];
  for (int i = threadIdx.x; i <= 2 * kLM; i += blockDim.x) s_fact[i] = fact[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m = lane;
  const int64_t base = (int64_t)blockIdx.x * kLatAdjChunk;
  const int cnt = (int)min((int64_t)kLatAdjChunk, nt - base);
  const int nf = (corr == 2) ? (int)s_aux[4] : 0;
  const int npair = nf * nbox;
  double2 acc[kLM + 1];
#pragma unroll
  for (int l = 0; l <= kLM; ++l) acc[l] = make_double2(0.0, 0.0);
  double xa[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = w; i < cnt; i += kOmWarps) {
    const int64_t t = base + i;
    const double px = tx[t], py = ty[t], pz = tz[t];
    const double gp = gphi[t], g0 = gex[t], g1 = gey[t], g2 = gez[t];
    double sph[3];
    cart2sph(px - cx, py - cy, pz - cz, sph);
    const double2 c11 = make_double2(-g0, g1);
    const double c10 = -g2;
    const double xc = sph[1];
    double sn = 0.0, cs = 1.0;
    double pmm = 1.0;
    if (m <= kLM) {
      sincos((double)m * sph[2], &sn, &cs);
      if (m > 0) {
        const double somx2 = sqrt((1.0 - xc) * (1.0 + xc));
        double f = 1.0;
        for (int k = 1; k <= m; ++k) {
          pmm = (-pmm * f) * somx2;
          f = f + 2.0;
        }
      }
    }
    const double sg = (m & 1) ? -1.0 : 1.0;
    double pmmp1 = 0.0, rl = 1.0;
    double2 prev = make_double2(0.0, 0.0);  // O(j - 1, m)
#pragma unroll
    for (int j = 0; j <= kLM; ++j) {
      double2 o = make_double2(0.0, 0.0);
      if (j >= m) {
        double P;
        if (j == m) {
          P = pmm;
        } else if (j == m + 1) {
          pmmp1 = (xc * (2.0 * m + 1.0)) * pmm;
          P = pmmp1;
        } else {
          const double pll =
              ((xc * (2.0 * j - 1.0)) * pmmp1 - ((double)(j + m) - 1.0) * pmm) / (double)(j - m);
          pmm = pmmp1;
          pmmp1 = pll;
          P = pll;
        }
        const double pt = (sg * P) / s_fact[j + m];
        const double amp = (sph[0] > 0.0 || j > 0) ? rl * pt : pt;
        o = make_double2(amp * cs, amp * -sn);
      }
      rl = rl * sph[0];
      double2 lo, hi;  // O(j - 1, m - 1) and O(j - 1, m + 1)
      lo.x = __shfl_up_sync(0xffffffffu, prev.x, 1);
      lo.y = __shfl_up_sync(0xffffffffu, prev.y, 1);
      hi.x = __shfl_down_sync(0xffffffffu, prev.x, 1);
      hi.y = __shfl_down_sync(0xffffffffu, prev.y, 1);
      if (m == 31) hi = make_double2(0.0, 0.0);
      const double2 hic = make_double2(hi.x, -hi.y);
      double2 g;
      if (m == 0) {
        const double2 a = cmul(c11, hic);
        g = make_double2((gp * o.x + c10 * prev.x) - a.x, (gp * o.y + c10 * prev.y) - a.y);
      } else {
        const double2 a = cmul(c11, lo);
        const double2 b = cmul(make_double2(c11.x, -c11.y), hi);
        g = make_double2(((2.0 * gp) * o.x + (2.0 * c10) * prev.x) + (a.x - b.x),
                         ((2.0 * gp) * o.y + (2.0 * c10) * prev.y) + (a.y - b.y));
      }
      acc[j] = cadd(acc[j], g);
      prev = o;
    }
    if (corr == 1 && lane == 0) {
      const double R[3] = {px - cx, py - cy, pz - cz};
      const double ge[3] = {g0, g1, g2};
      for (int d = 0; d < 3; ++d) xa[4 + d] += (2.0 * prefact) * ge[d] - ((2.0 * prefact) * gp) * R[d];
      xa[7] += prefact * gp;
    }
    for (int k = lane; k < npair; k += 32) {
      const int p = k / nbox, ib = k - p * nbox;
      const double d0 = (px - s_vb[3 * ib]) - s_aux[8 + 4 * p];
      const double d1 = (py - s_vb[3 * ib + 1]) - s_aux[9 + 4 * p];
      const double d2 = (pz - s_vb[3 * ib + 2]) - s_aux[10 + 4 * p];
      const double rd = 1.0 / sqrt((d0 * d0 + d1 * d1) + d2 * d2);
      const double v = gp * rd + ((rd * rd) * rd) * ((g0 * d0 + g1 * d1) + g2 * d2);
      if (p == 0) xa[0] += v;
      else if (p == 1) xa[1] += v;
      else if (p == 2) xa[2] += v;
      else xa[3] += v;
    }
  }
#pragma unroll
  for (int l = 0; l <= kLM; ++l)
    if (m <= l) s_acc[w][tblinv(l, m)] = acc[l];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double v = xa[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) s_x[w][k] = v;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < kLenM; idx += blockDim.x) {
    double2 t = s_acc[0][idx];
    for (int ww = 1; ww < kOmWarps; ++ww) t = cadd(t, s_acc[ww][idx]);
    part[(int64_t)blockIdx.x * kLenM + idx] = t;
  }
  if (threadIdx.x < 8) {
    double v = s_x[0][threadIdx.x];
    for (int ww = 1; ww < kOmWarps; ++ww) v += s_x[ww][threadIdx.x];
    xpart[(int64_t)blockIdx.x * 8 + threadIdx.x] = v;
  }
}

struct LatAdjGeom {
  int per[3];
  double len[3];  // |t_lattice_p|
  double cx, cy, cz;
  int corr;
};

// One block: G = sum of the partials (block order); dL/domega = the M2L
// transpose of G, B(j, k) = (-1)^j sum_{l, m >= 0} G(l, m) ML(j + l, k + m),
// folded onto k >= 0, and zero at (0, 0).  Then
// the fictitious charges: dL/dq_f = the direct terms + Re sum dL/domega O(x_f
// - c), and q_p = -d_p / |L_p|, q_last = -sum q_p give dL/d(dipole).  The
// output coef holds dL/domega and the gradient tables Dx, Dy, Dz with
// Re sum_{a, b >= 0} D(a, b) O(a, b) = d/dx Re sum dL/domega(l, m) O(l, m),
// from the ladder relations d/dz O(l, m) = O(l-1, m) and (d/dx +- i d/dy)
// O(l, m) = +-O(l-1, m-+1):
//   Dx(a, b) = (W(a+1, b+1) - W(a+1, b-1) - [b = 1] conj(W(a+1, 0))) / 2
//   Dy(a, b) = -i (W(a+1, b+1) + W(a+1, b-1) + [b = 1] conj(W(a+1, 0))) / 2
//   Dz(a, b) = W(a+1, b)        (W(a+1, -1) read as 0), then dL/d(dipole)
// and dL/d(trace) in coef[4 kLenM ..].
__global__ void __launch_bounds__(256) k_latadj_final(int nparts, const double2* __restrict__ part,
                                                      const double* __restrict__ xpart,
                                                      const double2* __restrict__ ML,
                                                      const double* __restrict__ aux,
                                                      LatAdjGeom geo, const double* fact,
                                                      double2* __restrict__ coef) {
  __shared__ double2 s_G[kLenM], s_W[kLenM];
  __shared__ double s_X[8], s_qf[4];
  const int idx = threadIdx.x;
  if (idx < kLenM) {
    double2 t = make_double2(0.0, 0.0);
    for (int b = 0; b < nparts; ++b) t = cadd(t, part[(int64_t)b * kLenM + idx]);
    s_G[idx] = t;
  }
  if (idx < 8) {
    double v = 0.0;
    for (int b = 0; b < nparts; ++b) v += xpart[(int64_t)b * 8 + idx];
    s_X[idx] = v;
  }
  __syncthreads();
  int j = 0, m = 0;
  if (idx < kLenM) {
    while ((j + 1) * (j + 2) / 2 <= idx) ++j;
    m = idx - j * (j + 1) / 2;
    const double sj = (j & 1) ? -1.0 : 1.0;
    double2 b = make_double2(0.0, 0.0), bn = make_double2(0.0, 0.0);
    for (int l = 0; l <= kLM; ++l)
      for (int mm = 0; mm <= l; ++mm) {
        const double2 g = s_G[tblinv(l, mm)];
        const double2 a = tbl(ML, j + l, m + mm, kLT);
        b = cadd(b, cmul(g, make_double2(sj * a.x, sj * a.y)));
        if (m > 0) {
          const double2 an = tbl(ML, j + l, mm - m, kLT);
          bn = cadd(bn, cmul(g, make_double2(sj * an.x, sj * an.y)));
        }
      }
    if (m > 0) {
      const double s = (m & 1) ? -1.0 : 1.0;
      b = cadd(b, make_double2(s * bn.x, -s * bn.y));
    }
    // omega(0, 0) never reaches mu (removed, or exactly zero with every
    // change of a charge making it removed): its adjoint is zero, which also
    // keeps the divergent ML(0, 0) (~1e32 in the unit-cube table) out of the
    // fictitious charges' difference below
    if (idx == 0) b = make_double2(0.0, 0.0);
    s_W[idx] = b;
    coef[idx] = b;
  }
  __syncthreads();
  const int nf = (geo.corr == 2) ? (int)aux[4] : 0;
  if (idx < nf) {
    double s[3];
    cart2sph(aux[8 + 4 * idx] - geo.cx, aux[9 + 4 * idx] - geo.cy, aux[10 + 4 * idx] - geo.cz, s);
    double v = s_X[idx];
    for (int l = 0; l <= kLM; ++l)
      for (int mm = 0; mm <= l; ++mm) {
        const double2 o = omultipole(l, mm, s, fact), wv = s_W[tblinv(l, mm)];
        v += wv.x * o.x - wv.y * o.y;
      }
    s_qf[idx] = v;
  }
  __syncthreads();
  if (idx == 0) {
    double db[3] = {0.0, 0.0, 0.0}, tb = 0.0;
    if (geo.corr == 1) {
      for (int d = 0; d < 3; ++d) db[d] = s_X[4 + d];
      tb = s_X[7];
    } else if (geo.corr == 2) {
      const double qlast = s_qf[nf - 1];
      int ip = 0;
      for (int p = 0; p < 3; ++p) {
        if (!geo.per[p]) continue;
        db[p] = (qlast - s_qf[ip]) / geo.len[p];
        ++ip;
      }
    }
    coef[4 * kLenM] = make_double2(db[0], db[1]);
    coef[4 * kLenM + 1] = make_double2(db[2], tb);
  }
  if (idx < kLenM) {
    const int a = j, bb = m;
    double2 dxv = make_double2(0.0, 0.0), dyv = dxv, dzv = dxv;
    if (a < kLM) {
      const double2 up = s_W[tblinv(a + 1, bb + 1)];
      const double2 dn = (bb >= 1) ? s_W[tblinv(a + 1, bb - 1)] : make_double2(0.0, 0.0);
      double2 ex = make_double2(0.0, 0.0);
      if (bb == 1) ex = make_double2(s_W[tblinv(a + 1, 0)].x, -s_W[tblinv(a + 1, 0)].y);
      const double2 sx = make_double2((up.x - dn.x) - ex.x, (up.y - dn.y) - ex.y);
      const double2 sy = make_double2((up.x + dn.x) + ex.x, (up.y + dn.y) + ex.y);
      dxv = make_double2(0.5 * sx.x, 0.5 * sx.y);
      dyv = make_double2(0.5 * sy.y, -0.5 * sy.x);  // -i sy / 2
      dzv = s_W[tblinv(a + 1, bb)];
    }
    coef[kLenM + idx] = dxv;
    coef[2 * kLenM + idx] = dyv;
    coef[3 * kLenM + idx] = dzv;
  }
}

// per particle (key order): dL/dq = Re sum W O(x - c) + dipole-bar . R +
// trace-bar |R|^2, dL/dx = q (Re sum D O + dipole-bar + 2 trace-bar R), added
// at the caller's original index perm[i]
__global__ void __launch_bounds__(128) k_latadj_particles(
    int64_t n, const double* __restrict__ x, const double* __restrict__ y,
    const double* __restrict__ z, const double* __restrict__ q, const int32_t* __restrict__ perm,
    const double2* __restrict__ coef, double cx, double cy, double cz,
    const double* __restrict__ fact, double* dq, double* dx, double* dy, double* dz) {
  __shared__ double2 s_c[4 * kLenM + 2];
  __shared__ double s_fact[2 * kLM + 1];
  for (int i = threadIdx.x; i < 4 * kLenM + 2; i += blockDim.x) s_c[i] = coef[i];
  for (int i = threadIdx.x; i <= 2 * kLM; i += blockDim.x) s_fact[i] = fact[i];
  __syncthreads();
  const double db0 = s_c[4 * kLenM].x, db1 = s_c[4 * kLenM].y, db2 = s_c[4 * kLenM + 1].x;
  const double tb = s_c[4 * kLenM + 1].y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double R0 = x[i] - cx, R1 = y[i] - cy, R2 = z[i] - cz;
    double s[3];
    cart2sph(R0, R1, R2, s);
    double gq = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
    for (int m = 0; m <= kLM; ++m) {
      double sn, cs;
      sincos((double)m * s[2], &sn, &cs);
      const double sg = (m & 1) ? -1.0 : 1.0;
      const double xc = s[1];
      double pmm = 1.0;
      if (m > 0) {
        const double somx2 = sqrt((1.0 - xc) * (1.0 + xc));
        double f = 1.0;
        for (int k = 1; k <= m; ++k) {
          pmm = (-pmm * f) * somx2;
          f = f + 2.0;
        }
      }
      double rl = 1.0;
      for (int k = 0; k < m; ++k) rl = rl * s[0];
      double pmmp1 = 0.0;
      for (int a = m; a <= kLM; ++a) {
        double P;
        if (a == m) {
          P = pmm;
        } else if (a == m + 1) {
          pmmp1 = (xc * (2.0 * m + 1.0)) * pmm;
          P = pmmp1;
        } else {
          const double pll =
              ((xc * (2.0 * a - 1.0)) * pmmp1 - ((double)(a + m) - 1.0) * pmm) / (double)(a - m);
          pmm = pmmp1;
          pmmp1 = pll;
          P = pll;
        }
        const double pt = (sg * P) / s_fact[a + m];
        const double amp = (s[0] > 0.0 || a > 0) ? rl * pt : pt;
        rl = rl * s[0];
        const double ox = amp * cs, oy = amp * -sn;
        const int t = tblinv(a, m);
        const double2 wv = s_c[t], ax = s_c[kLenM + t], ay = s_c[2 * kLenM + t],
                      az = s_c[3 * kLenM + t];
        gq += wv.x * ox - wv.y * oy;
        g0 += ax.x * ox - ax.y * oy;
        g1 += ay.x * ox - ay.y * oy;
        g2 += az.x * ox - az.y * oy;
      }
    }
    gq += ((db0 * R0 + db1 * R1) + db2 * R2) + tb * ((R0 * R0 + R1 * R1) + R2 * R2);
    const double qi = q[i];
    const int64_t o = perm[i];
    dq[o] += gq;
    dx[o] += qi * ((g0 + db0) + (2.0 * tb) * R0);
    dy[o] += qi * ((g1 + db1) + (2.0 * tb) * R1);
    dz[o] += qi * ((g2 + db2) + (2.0 * tb) * R2);
  }
}

double host_factorial(int n) {  // factorial, :1247-1314 (the exact values to 24!, gamma above)
  static const double f[25] = {1.0, 1.0, 2.0, 6.0, 24.0, 120.0, 720.0, 5040.0, 40320.0,
                               362880.0, 3628800.0, 39916800.0, 479001600.0, 6227020800.0,
                               87178291200.0, 1307674368000.0, 20922789888000.0,
                               355687428096000.0, 6402373705728000.0, 121645100408832000.0,
                               2432902008176640000.0, 51090942171709440000.0,
                               1124000727777607680000.0, 25852016738884976640000.0,
                               620448401733239439360000.0};
  if (n <= 24) return f[n];
  return std::tgamma((double)(n + 1));
}

bool unit_cube(const pepcg_params& p) {  // system_is_unit_cube, module_mirror_boxes.f90:248-255
  auto nsq = [](const double* v) { return (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]; };
  bool axes = p.t_lattice_1[0] > 0 && p.t_lattice_1[1] == 0 && p.t_lattice_1[2] == 0 &&
              p.t_lattice_2[0] == 0 && p.t_lattice_2[1] > 0 && p.t_lattice_2[2] == 0 &&
              p.t_lattice_3[0] == 0 && p.t_lattice_3[1] == 0 && p.t_lattice_3[2] > 0;
  return axes && nsq(p.t_lattice_1) == 1.0 && nsq(p.t_lattice_2) == 1.0 && nsq(p.t_lattice_3) == 1.0;
}

}  // namespace

int lattice_prepare(Ctx* c) {
  const pepcg_params& p = c->prm;
  cudaStream_t s = c->stream;
  const int lm = unit_cube(p) ? kLMTable : kLM;
  const int lt = 2 * lm;
  const int lenm = lm * (lm + 1) / 2 + lm + 1, lent = lt * (lt + 1) / 2 + lt + 1;
  const int nb = c->nboxes, ws = p.mirror_box_layers;
  // factorials (exact to 24!, gamma above, as the reference) and (2 ws + 1)**(l + 1)
  std::vector<double> hf(2 * lt + 2), hs(lt + 1);
  for (int i = 0; i < (int)hf.size(); ++i) hf[i] = host_factorial(i);
  for (int l = 0; l <= lt; ++l) hs[l] = std::pow((double)(2 * ws + 1), (double)(l + 1));
  double2 *mstar = nullptr, *lstar = nullptr, *ml0 = nullptr, *ml1 = nullptr;
  double *scratch = nullptr, *d_scp = nullptr;
  const int64_t cnt = (int64_t)nb * (nb - 1);
  const size_t scratch_n = (size_t)lent * 2 * (cnt > nb ? cnt : nb);
  bool ok = cuda_ok(c, cudaMalloc((void**)&c->d_factorial, hf.size() * 8), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&c->d_mlattice, kLenT * 16), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&c->d_omega, kLenM * 16), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&c->d_mu, kLenT * 16), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&c->d_fmm_aux, 64 * 8), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&mstar, lenm * 16), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&lstar, lent * 16), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&ml0, lent * 16), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&ml1, lent * 16), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&d_scp, (lt + 1) * 8), "fmm") &&
            cuda_ok(c, cudaMalloc((void**)&scratch, scratch_n * 8), "fmm scratch");
  if (ok) {
    cudaMemcpyAsync(c->d_factorial, hf.data(), hf.size() * 8, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_scp, hs.data(), hs.size() * 8, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(c->d_fmm_aux, 0, 64 * 8, s);
    COUNT_LAUNCH();
    k_mstar<<<(lenm + 63) / 64, 64, 0, s>>>(lm, nb, c->d_vbox, c->d_factorial, scratch, mstar);
    COUNT_LAUNCH();
    k_lstar<<<(lent + 63) / 64, 64, 0, s>>>(lt, nb, ws, c->d_vbox, c->d_factorial, scratch, lstar);
    cudaMemcpyAsync(ml0, lstar, lent * 16, cudaMemcpyDeviceToDevice, s);
    for (int it = 0; it < kMaxIter; ++it) {
      COUNT_LAUNCH();
      k_lattice_iter<<<(lent + 127) / 128, 128, 0, s>>>(lt, lm, ml0, mstar, lstar, d_scp, ml1);
      std::swap(ml0, ml1);
    }
    COUNT_LAUNCH();
    k_truncate<<<(kLenT + 127) / 128, 128, 0, s>>>(ml0, c->d_mlattice, lm == kLMTable ? 1 : 0);
    ok = cuda_ok(c, cudaGetLastError(), "lattice coefficients") &&
         cuda_ok(c, cudaStreamSynchronize(s), "lattice coefficients");
  }
  for (void* q : {(void*)mstar, (void*)lstar, (void*)ml0, (void*)ml1, (void*)scratch, (void*)d_scp})
    if (q) cudaFree(q);
  return ok ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int lattice_timestep(Ctx* c) {
  const pepcg_params& p = c->prm;
  cudaStream_t s = c->stream;
  const double cx = 0.5 * ((p.t_lattice_1[0] + p.t_lattice_2[0]) + p.t_lattice_3[0]) + p.lattice_origin[0];
  const double cy = 0.5 * ((p.t_lattice_1[1] + p.t_lattice_2[1]) + p.t_lattice_3[1]) + p.lattice_origin[1];
  const double cz = 0.5 * ((p.t_lattice_1[2] + p.t_lattice_2[2]) + p.t_lattice_3[2]) + p.lattice_origin[2];
  const int64_t n = c->n;
  const int nbp = 148;
  const int64_t nom = (n + kOmChunk - 1) / kOmChunk;
  double* part = nullptr;
  double2* opart = nullptr;
  double* d_lat = nullptr;
  bool ok = cuda_ok(c, cudaMallocAsync((void**)&part, 4 * nbp * 8, s), "fmm") &&
            cuda_ok(c, cudaMallocAsync((void**)&opart, nom * kLenM * 16, s), "fmm") &&
            cuda_ok(c, cudaMallocAsync((void**)&d_lat, 12 * 8, s), "fmm");
  if (!ok) return PEPCG_ERR_OOM;
  double lat[12];
  for (int d = 0; d < 3; ++d) {
    lat[d] = p.t_lattice_1[d];
    lat[3 + d] = p.t_lattice_2[d];
    lat[6 + d] = p.t_lattice_3[d];
    lat[9 + d] = p.lattice_origin[d];
  }
  cudaMemcpyAsync(d_lat, lat, 12 * 8, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(c->d_status, 0, 4, s);
  COUNT_LAUNCH();
  k_box_dipole<<<nbp, 256, 0, s>>>(n, c->x.p, c->y.p, c->z.p, c->q.p, cx, cy, cz, part);
  COUNT_LAUNCH();
  k_fict<<<1, 32, 0, s>>>(nbp, part, c->d_fmm_aux, p.periodicity[0], p.periodicity[1],
                         p.periodicity[2], d_lat, d_lat + 9, p.fmm_extrinsic_correction);
  COUNT_LAUNCH();
  k_omega_partial<<<(unsigned)nom, 256, 0, s>>>(n, c->x.p, c->y.p, c->z.p, c->q.p, cx, cy, cz,
                                                c->d_factorial, opart);
  COUNT_LAUNCH();
  k_omega_final<<<1, 256, 0, s>>>((int)nom, opart, c->d_fmm_aux, cx, cy, cz, c->d_factorial,
                                  c->d_omega, c->d_status);
  COUNT_LAUNCH();
  k_mu_cent<<<(kLenT + 127) / 128, 128, 0, s>>>(c->d_mlattice, c->d_omega, c->d_mu);
  uint32_t st = 0;
  ok = cuda_ok(c, cudaGetLastError(), "lattice timestep") &&
       cuda_ok(c, cudaMemcpyAsync(&st, c->d_status, 4, cudaMemcpyDeviceToHost, s), "status");
  cudaFreeAsync(part, s);
  cudaFreeAsync(opart, s);
  cudaFreeAsync(d_lat, s);
  ok = ok && cuda_ok(c, cudaStreamSynchronize(s), "lattice timestep");
  if (!ok) return PEPCG_ERR_CUDA;
  return st ? status_to_code(c, st) : PEPCG_OK;
}

int lattice_add(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                double* ex, double* ey, double* ez, double* pot, bool overwrite) {
  const pepcg_params& p = c->prm;
  cudaStream_t s = c->stream;
  const double cx = 0.5 * ((p.t_lattice_1[0] + p.t_lattice_2[0]) + p.t_lattice_3[0]) + p.lattice_origin[0];
  const double cy = 0.5 * ((p.t_lattice_1[1] + p.t_lattice_2[1]) + p.t_lattice_3[1]) + p.lattice_origin[1];
  const double cz = 0.5 * ((p.t_lattice_1[2] + p.t_lattice_2[2]) + p.t_lattice_3[2]) + p.lattice_origin[2];
  const double* a = p.t_lattice_1;
  const double* b = p.t_lattice_2;
  const double* cc = p.t_lattice_3;
  double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  const double volume = std::fabs((cr[0] * cc[0] + cr[1] * cc[1]) + cr[2] * cc[2]);
  unsigned blocks = (unsigned)((nt + 127) / 128);
  if (blocks > 148 * 16) blocks = 148 * 16;
  COUNT_LAUNCH();
  k_lattice_force<<<blocks, 128, 0, s>>>(nt, tx, ty, tz, c->d_mu, c->d_fmm_aux, c->d_vbox, c->nboxes,
                                         cx, cy, cz, volume, p.fmm_extrinsic_correction,
                                         c->d_factorial, ex, ey, ez, pot, overwrite ? 1 : 0);
  return cuda_ok(c, cudaGetLastError(), "lattice force") ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int lattice_adjoint(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                    const double* gex, const double* gey, const double* gez, const double* gphi,
                    double* dq, double* dx, double* dy, double* dz) {
  const pepcg_params& p = c->prm;
  cudaStream_t s = c->stream;
  LatAdjGeom geo;
  geo.cx = 0.5 * ((p.t_lattice_1[0] + p.t_lattice_2[0]) + p.t_lattice_3[0]) + p.lattice_origin[0];
  geo.cy = 0.5 * ((p.t_lattice_1[1] + p.t_lattice_2[1]) + p.t_lattice_3[1]) + p.lattice_origin[1];
  geo.cz = 0.5 * ((p.t_lattice_1[2] + p.t_lattice_2[2]) + p.t_lattice_3[2]) + p.lattice_origin[2];
  const double* lv[3] = {p.t_lattice_1, p.t_lattice_2, p.t_lattice_3};
  for (int d = 0; d < 3; ++d) {
    geo.per[d] = p.periodicity[d];
    geo.len[d] = std::sqrt((lv[d][0] * lv[d][0] + lv[d][1] * lv[d][1]) + lv[d][2] * lv[d][2]);
  }
  geo.corr = p.fmm_extrinsic_correction;
  const double* a = p.t_lattice_1;
  const double* b = p.t_lattice_2;
  const double* cc = p.t_lattice_3;
  double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  const double volume = std::fabs((cr[0] * cc[0] + cr[1] * cc[1]) + cr[2] * cc[2]);
  const double prefact = (2.0 * std::acos(-1.0)) / (3.0 * volume);
  const int64_t nparts = nt > 0 ? (nt + kLatAdjChunk - 1) / kLatAdjChunk : 1;
  double2* part = nullptr;
  double* xpart = nullptr;
  double2* coef = nullptr;
  bool ok = cuda_ok(c, cudaMallocAsync((void**)&part, nparts * kLenM * 16, s), "lattice adjoint") &&
            cuda_ok(c, cudaMallocAsync((void**)&xpart, nparts * 8 * 8, s), "lattice adjoint") &&
            cuda_ok(c, cudaMallocAsync((void**)&coef, (4 * kLenM + 2) * 16, s), "lattice adjoint");
  if (!ok) {
    for (void* v : {(void*)part, (void*)xpart, (void*)coef})
      if (v) cudaFreeAsync(v, s);
    return PEPCG_ERR_OOM;
  }
  if (nt > 0) {
    COUNT_LAUNCH();
    k_latadj_targets<<<(unsigned)nparts, 256, 0, s>>>(nt, tx, ty, tz, gex, gey, gez, gphi, geo.cx,
                                                      geo.cy, geo.cz, prefact, geo.corr,
                                                      c->d_fmm_aux, c->d_vbox, c->nboxes,
                                                      c->d_factorial, part, xpart);
  } else {
    cudaMemsetAsync(part, 0, kLenM * 16, s);
    cudaMemsetAsync(xpart, 0, 8 * 8, s);
  }
  COUNT_LAUNCH();
  k_latadj_final<<<1, 256, 0, s>>>((int)nparts, part, xpart, c->d_mlattice, c->d_fmm_aux, geo,
                                   c->d_factorial, coef);
  const int64_t n = c->n;
  unsigned blocks = (unsigned)((n + 127) / 128);
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks == 0) blocks = 1;
  COUNT_LAUNCH();
  k_latadj_particles<<<blocks, 128, 0, s>>>(n, c->x.p, c->y.p, c->z.p, c->q.p, c->perm.p, coef,
                                            geo.cx, geo.cy, geo.cz, c->d_factorial, dq, dx, dy,
                                            dz);
  ok = cuda_ok(c, cudaGetLastError(), "lattice adjoint");
  cudaFreeAsync(part, s);
  cudaFreeAsync(xpart, s);
  cudaFreeAsync(coef, s);
  return ok ? PEPCG_OK : PEPCG_ERR_CUDA;
}

}  // namespace pepcg
