// pepc_oracle_fmm.cpp -- CPU FP64 restatement of PEPC's periodic far-lattice
// term (interaction_specific/coulomb/module_fmm_framework.f90).
//
// TEST INFRASTRUCTURE ONLY (parity checker, see pepc_oracle.cpp).
//
// Expansions use the reference's flat (l, m >= 0) table layout
// tblinv(l, m) = l(l+1)/2 + m (0-based here), Lmax_multipole = 20 and
// Lmax_taylor = 40 (module_fmm_framework.f90:70-77).  chop() is a no-op in the
// reference (chop_arrays = .false., :62) and is omitted.

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "pepc_oracle.h"

namespace {

constexpr int kLmaxM = 20;                 // Lmax_multipole, :70
constexpr int kLmaxT = 2 * kLmaxM;         // Lmax_taylor, :71
constexpr int kMaxIter = 32;               // :72
constexpr int kLenM = kLmaxM * (kLmaxM + 1) / 2 + kLmaxM + 1;  // 231
constexpr int kLenT = kLmaxT * (kLmaxT + 1) / 2 + kLmaxT + 1;  // 861

struct C {
  double re, im;
};
inline C cadd(C a, C b) { return {a.re + b.re, a.im + b.im}; }
inline C cmul(C a, C b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C cscale(double s, C a) { return {s * a.re, s * a.im}; }

inline int tblinv(int l, int m) { return l * (l + 1) / 2 + m; }  // :865-875 (0-based)

// tbl, :838-854: symmetric access for negative m, zero outside the table
inline C tbl(const C* A, int l, int m, int lmax) {
  if (l > lmax || std::abs(m) > l) return {0.0, 0.0};
  C t = A[tblinv(l, std::abs(m))];
  if (m < 0) {
    double s = (m % 2 == 0) ? 1.0 : -1.0;  // (-one)**m
    t = {s * t.re, -s * t.im};            // (-1)^m conjg
  }
  return t;
}

// factorial, :1247-1314 (exact table to 24, gamma above)
double factorial(int n) {
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

// LegendreP, :1196-1242 (Numerical Recipes recurrence, times (-1)^m)
double legendre_p(int l, int m, double x) {
  double pll = 0.0, pmm = 1.0;
  if (m > 0) {
    double somx2 = std::sqrt((1.0 - x) * (1.0 + x));
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
  return ((m % 2 == 0) ? 1.0 : -1.0) * r;
}

// Ptilda / P2tilda, :659-689 (only m >= 0 is used by the callers below)
inline double ptilda(int l, int m, double x) { return legendre_p(l, m, x) / factorial(l + m); }
inline double p2tilda(int l, int m, double x) { return legendre_p(l, m, x) * factorial(l - m); }

// cartesian_to_spherical, :1083-1103 -> (r, cos(theta), phi)
std::array<double, 3> cart2sph(const double c[3]) {
  std::array<double, 3> s;
  s[0] = std::sqrt((c[0] * c[0] + c[1] * c[1]) + c[2] * c[2]);
  s[1] = (s[0] == 0.0) ? 1.0 : c[2] / s[0];
  s[2] = (c[0] == 0.0 && c[1] == 0.0) ? 0.0 : std::atan2(c[1], c[0]);
  return s;
}

// OMultipole, :695-714
C omultipole(int l, int m, const std::array<double, 3>& s) {
  double ph = (double)m * s[2];
  C e = {std::cos(ph), -std::sin(ph)};  // exp(-i m phi)
  double a;
  if (s[0] > 0.0 || l > 0) a = std::pow(s[0], (double)l) * ptilda(l, m, s[1]);
  else a = ptilda(l, m, s[1]);
  return cscale(a, e);
}

// MTaylor, :720-733
C mtaylor(int l, int m, const std::array<double, 3>& s) {
  double ph = (double)m * s[2];
  C e = {std::cos(ph), std::sin(ph)};  // exp(+i m phi)
  double a = (1.0 / std::pow(s[0], (double)(l + 1))) * p2tilda(l, m, s[1]);
  return cscale(a, e);
}

// M2L, :912-937
void m2l(const C* Mb, const C* Oa, C* out) {
  for (int l = 0; l <= kLmaxT; ++l)
    for (int m = 0; m <= l; ++m) {
      C t = {0.0, 0.0};
      for (int j = 0; j <= kLmaxT; ++j) {
        double sg = (j % 2 == 0) ? 1.0 : -1.0;
        for (int k = -j; k <= j; ++k)
          t = cadd(t, cmul(cscale(sg, tbl(Mb, j + l, k + m, kLmaxT)), tbl(Oa, j, k, kLmaxM)));
      }
      out[tblinv(l, m)] = t;
    }
}

// L2L, :943-976 (only the terms up to max_l are formed)
void l2l(const C* Ob, const C* Mr, int maxl, C* out) {
  for (int l = 0; l <= maxl; ++l)
    for (int m = 0; m <= l; ++m) {
      C t = {0.0, 0.0};
      for (int j = l; j <= kLmaxM; ++j)
        for (int k = -j; k <= j; ++k)
          t = cadd(t, cmul(tbl(Ob, j - l, k - m, kLmaxM), tbl(Mr, j, k, kLmaxT)));
      out[tblinv(l, m)] = t;
    }
}

// sort_abs, :1321-1367 (heap sort by |value|, Numerical Recipes f90)
void sort_abs(std::vector<double>& a) {
  int n = (int)a.size();
  auto sift = [&](int l, int r) {  // 1-based l, r
    double v = a[l - 1];
    int jold = l, j = l + l;
    for (;;) {
      if (j > r) break;
      if (j < r && std::fabs(a[j - 1]) < std::fabs(a[j])) j = j + 1;
      if (std::fabs(v) >= std::fabs(a[j - 1])) break;
      a[jold - 1] = a[j - 1];
      jold = j;
      j = j + j;
    }
    a[jold - 1] = v;
  };
  for (int i = n / 2; i >= 1; --i) sift(i, n);
  for (int i = n; i >= 2; --i) {
    std::swap(a[0], a[i - 1]);
    sift(1, i - 1);
  }
}

}  // namespace

struct OrcFmm {
  orc_params p;
  std::vector<std::array<int, 3>> boxes;
  double lattice[3][3];
  double center[3];
  double volume;
  int ws;
  std::vector<C> mlattice, omega, mu;
  double box_dipole[3] = {0, 0, 0}, quad_trace = 0;
  int nfict = 0;
  double fict_pos[4][3], fict_q[4];

  void lvect(const std::array<int, 3>& ijk, double v[3]) const {
    for (int d = 0; d < 3; ++d)
      v[d] = ((double)ijk[0] * p.t_lattice_1[d] + (double)ijk[1] * p.t_lattice_2[d]) +
             (double)ijk[2] * p.t_lattice_3[d];
  }
};

// neighbour_boxes_prepare order (module_mirror_boxes.f90:99-156)
static std::vector<std::array<int, 3>> fmm_boxes(const orc_params& p) {
  int sw[3];
  for (int d = 0; d < 3; ++d) sw[d] = p.periodicity[d] ? p.mirror_box_layers : 0;
  std::vector<std::array<int, 3>> nb;
  for (int i = -sw[0]; i <= -1; ++i)
    for (int j = -sw[1]; j <= sw[1]; ++j)
      for (int k = -sw[2]; k <= sw[2]; ++k) {
        nb.push_back({i, j, k});
        nb.push_back({-i, -j, -k});
      }
  for (int j = -sw[1]; j <= -1; ++j)
    for (int k = -sw[2]; k <= sw[2]; ++k) {
      nb.push_back({0, j, k});
      nb.push_back({0, -j, -k});
    }
  for (int k = -sw[2]; k <= -1; ++k) {
    nb.push_back({0, 0, k});
    nb.push_back({0, 0, -k});
  }
  nb.push_back({0, 0, 0});
  return nb;
}

// calc_lattice_coefficients, module_fmm_framework.f90:154-213
static void calc_lattice_coefficients(const OrcFmm& f, std::vector<C>& ML) {
  std::vector<C> Mstar(kLenM, {0, 0}), Lstar(kLenT, {0, 0});
  const int nb = (int)f.boxes.size();
  for (int l = 0; l <= kLmaxM; ++l)  // MstarFunc, :1005-1036
    for (int m = 0; m <= l; ++m) {
      std::vector<double> rp(nb), ip(nb);
      for (int i = 0; i < nb; ++i) {
        double v[3];
        f.lvect(f.boxes[i], v);
        double nv[3] = {-v[0], -v[1], -v[2]};
        C t = omultipole(l, m, cart2sph(nv));
        rp[i] = t.re;
        ip[i] = t.im;
      }
      sort_abs(rp);
      sort_abs(ip);
      double r = 0, im = 0;
      for (int i = 0; i < nb; ++i) { r = r + rp[i]; im = im + ip[i]; }
      Mstar[tblinv(l, m)] = {r, im};
    }
  for (int l = 0; l <= kLmaxT; ++l)  // LstarFunc, :1042-1077
    for (int m = 0; m <= l; ++m) {
      std::vector<double> rp, ip;
      rp.reserve(nb * (nb - 1));
      ip.reserve(nb * (nb - 1));
      for (int i = 0; i < nb - 1; ++i)
        for (int ii = 0; ii < nb; ++ii) {
          double a[3], b[3], s[3];
          f.lvect(f.boxes[i], a);
          f.lvect(f.boxes[ii], b);
          for (int d = 0; d < 3; ++d) s[d] = (double)(2 * f.ws + 1) * a[d] + b[d];
          C t = mtaylor(l, m, cart2sph(s));
          rp.push_back(t.re);
          ip.push_back(t.im);
        }
      sort_abs(rp);
      sort_abs(ip);
      double r = 0, im = 0;
      for (size_t i = 0; i < rp.size(); ++i) { r = r + rp[i]; im = im + ip[i]; }
      Lstar[tblinv(l, m)] = {r, im};
    }
  ML = Lstar;
  std::vector<C> U(kLenT), T(kLenT);
  const double sc = (double)(2 * f.ws + 1);
  for (int it = 0; it < kMaxIter; ++it) {
    for (int l = 0; l <= kLmaxT; ++l)  // UL, :982-999
      for (int m = 0; m <= l; ++m) {
        double d = std::pow(sc, (double)(l + 1));
        U[tblinv(l, m)] = {ML[tblinv(l, m)].re / d, ML[tblinv(l, m)].im / d};
      }
    m2l(U.data(), Mstar.data(), T.data());
    for (int i = 0; i < kLenT; ++i) ML[i] = cadd(T[i], Lstar[i]);
  }
}

OrcFmm* orc_fmm_create(const orc_params& p) {
  OrcFmm* f = new OrcFmm;
  f->p = p;
  f->boxes = fmm_boxes(p);
  for (int d = 0; d < 3; ++d) {
    f->lattice[0][d] = p.t_lattice_1[d];
    f->lattice[1][d] = p.t_lattice_2[d];
    f->lattice[2][d] = p.t_lattice_3[d];
    // LatticeCenter, module_mirror_boxes.f90:106
    f->center[d] = 0.5 * ((p.t_lattice_1[d] + p.t_lattice_2[d]) + p.t_lattice_3[d]) +
                   p.lattice_origin[d];
  }
  // unit_box_volume, module_mirror_boxes.f90:153
  const double* a = p.t_lattice_1;
  const double* b = p.t_lattice_2;
  const double* c = p.t_lattice_3;
  double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  f->volume = std::fabs((cr[0] * c[0] + cr[1] * c[1]) + cr[2] * c[2]);
  f->ws = p.mirror_box_layers;
  f->mlattice.assign(kLenT, {0, 0});
  calc_lattice_coefficients(*f, f->mlattice);
  f->omega.assign(kLenM, {0, 0});
  f->mu.assign(kLenT, {0, 0});
  return f;
}

void orc_fmm_destroy(OrcFmm* f) { delete f; }

// fmm_framework_timestep, :132-149 -> calc_box_dipole (:605-630),
// calc_omega_tilde (:514-596), calc_mu_cent (:636-649)
void orc_fmm_timestep(OrcFmm* f, int64_t n, const double* x, const double* y, const double* z,
                      const double* q) {
  const int corr = f->p.fmm_extrinsic_correction;
  for (int d = 0; d < 3; ++d) f->box_dipole[d] = 0.0;
  f->quad_trace = 0.0;
  if (corr == 1 || corr == 2) {
    for (int64_t i = 0; i < n; ++i) {
      double r[3] = {x[i] - f->center[0], y[i] - f->center[1], z[i] - f->center[2]};
      for (int d = 0; d < 3; ++d) f->box_dipole[d] = f->box_dipole[d] + q[i] * r[d];
      f->quad_trace = f->quad_trace + q[i] * ((r[0] * r[0] + r[1] * r[1]) + r[2] * r[2]);
    }
  }
  std::vector<C>& om = f->omega;
  om.assign(kLenM, {0, 0});
  auto addparticle = [&](const double R[3], double qq) {
    double rr[3] = {R[0] - f->center[0], R[1] - f->center[1], R[2] - f->center[2]};
    auto s = cart2sph(rr);
    for (int l = 0; l <= kLmaxM; ++l)
      for (int m = 0; m <= l; ++m) om[tblinv(l, m)] = cadd(om[tblinv(l, m)], cscale(qq, omultipole(l, m, s)));
  };
  for (int64_t i = 0; i < n; ++i) {
    double R[3] = {x[i], y[i], z[i]};
    addparticle(R, q[i]);
  }
  f->nfict = 0;
  if (corr == 2) {  // fictitious charges (Kudin & Scuseria), :536-559
    for (int pp = 0; pp < 3; ++pp) {
      if (!f->p.periodicity[pp]) continue;
      const double* L = f->lattice[pp];
      for (int d = 0; d < 3; ++d) f->fict_pos[f->nfict][d] = f->p.lattice_origin[d] + L[d];
      f->fict_q[f->nfict] = -f->box_dipole[pp] / std::sqrt((L[0] * L[0] + L[1] * L[1]) + L[2] * L[2]);
      ++f->nfict;
    }
    double s = 0.0;
    for (int i = 0; i < f->nfict; ++i) s = s + f->fict_q[i];
    for (int d = 0; d < 3; ++d) f->fict_pos[f->nfict][d] = f->p.lattice_origin[d];
    f->fict_q[f->nfict] = -s;
    ++f->nfict;
    for (int i = 0; i < f->nfict; ++i) addparticle(f->fict_pos[i], f->fict_q[i]);
  }
  // a non-neutral box has its monopole removed, :570-573
  if (std::hypot(om[0].re, om[0].im) > 0.0) om[0] = {0.0, 0.0};
  m2l(f->mlattice.data(), om.data(), f->mu.data());
}

// fmm_sum_lattice_force, :766-826
void orc_fmm_sum_lattice_force(const OrcFmm* f, const double pos[3], double e[3], double* phi) {
  const double pi = std::acos(-1.0);
  const double prefact = (2.0 * pi) / (3.0 * f->volume);
  double R[3] = {pos[0] - f->center[0], pos[1] - f->center[1], pos[2] - f->center[2]};
  auto s = cart2sph(R);
  C OR[kLenM];
  for (int l = 0; l <= kLmaxM; ++l)
    for (int m = 0; m <= l; ++m) OR[tblinv(l, m)] = omultipole(l, m, s);
  C mus[3];
  l2l(OR, f->mu.data(), 1, mus);
  e[0] = -mus[tblinv(1, 1)].re;
  e[1] = -mus[tblinv(1, 1)].im;
  e[2] = -mus[tblinv(1, 0)].re;
  double ph = mus[tblinv(0, 0)].re;
  const int corr = f->p.fmm_extrinsic_correction;
  if (corr == 1) {
    for (int d = 0; d < 3; ++d) e[d] = e[d] + (2.0 * prefact) * f->box_dipole[d];
    double rd = (R[0] * f->box_dipole[0] + R[1] * f->box_dipole[1]) + R[2] * f->box_dipole[2];
    ph = (ph - (2.0 * prefact) * rd) + prefact * f->quad_trace;
  } else if (corr == 2) {
    for (int pp = 0; pp < f->nfict; ++pp) {
      for (const auto& bx : f->boxes) {
        double v[3], d[3];
        f->lvect(bx, v);
        for (int k = 0; k < 3; ++k) d[k] = (pos[k] - v[k]) - f->fict_pos[pp][k];
        double dist2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
        // calc_force_coulomb_3D_direct, module_coulomb_kernels.f90:242-257
        double r = std::sqrt(dist2);
        double rd = 1.0 / r;
        double rd3q = ((f->fict_q[pp] * rd) * rd) * rd;
        ph = ph + f->fict_q[pp] * rd;
        for (int k = 0; k < 3; ++k) e[k] = e[k] + rd3q * d[k];
      }
    }
  }
  *phi = ph;
}

void orc_fmm_set_mlattice(OrcFmm* f, const double* re_im) {
  for (int i = 0; i < kLenT; ++i) f->mlattice[i] = {re_im[2 * i], re_im[2 * i + 1]};
}

extern "C" {
// Lattice coefficients (MLattice) for inspection: 861 complex values as
// interleaved (re, im), layout tblinv(l, m).
void orc_fmm_lattice_coefficients(const orc_params* p, double* out) {
  OrcFmm* f = orc_fmm_create(*p);
  for (int i = 0; i < kLenT; ++i) {
    out[2 * i] = f->mlattice[i].re;
    out[2 * i + 1] = f->mlattice[i].im;
  }
  orc_fmm_destroy(f);
}
}
