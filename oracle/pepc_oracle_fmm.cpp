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

// ---------------------------------------------------------------------------
// Adjoint of the lattice term (no reference counterpart: the reference has no
// differentiation).  L = sum_t gphi_t phi_lat(t) + gE_t . E_lat(t); returns
// dL/dq and dL/dx of the n particles (x, y, z, q as given, the grown order).
// The chain: targets -> mu (transpose of L2L to l <= 1) -> omega (transpose of
// M2L) -> particles through O_lm(x - center), the fictitious charges (through
// the box dipole) and the Redlack terms.  The derivative of O_lm is taken by
// forward-mode dual numbers through omultipole's own operations, independently
// of any ladder relation between the harmonics.
// ---------------------------------------------------------------------------
namespace {
struct Dn {  // dual number v + d eps
  double v, d;
};
inline Dn operator+(Dn a, Dn b) { return {a.v + b.v, a.d + b.d}; }
inline Dn operator-(Dn a, Dn b) { return {a.v - b.v, a.d - b.d}; }
inline Dn operator*(Dn a, Dn b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dn operator/(Dn a, Dn b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dn dsc(double s, Dn a) { return {s * a.v, s * a.d}; }
inline Dn dsqrt(Dn a) {
  double r = std::sqrt(a.v);
  return {r, r > 0.0 ? a.d / (2.0 * r) : 0.0};
}

// legendre_p with a dual argument
Dn legendre_p_d(int l, int m, Dn x) {
  Dn pll = {0.0, 0.0}, pmm = {1.0, 0.0};
  if (m > 0) {
    Dn somx2 = dsqrt(( Dn{1.0, 0.0} - x) * (Dn{1.0, 0.0} + x));
    double fact = 1.0;
    for (int i = 1; i <= m; ++i) {
      pmm = dsc(-fact, pmm) * somx2;
      fact = fact + 2.0;
    }
  }
  Dn r;
  if (l == m) {
    r = pmm;
  } else {
    Dn pmmp1 = dsc(2.0 * m + 1.0, x * pmm);
    if (l == m + 1) {
      r = pmmp1;
    } else {
      for (int ll = m + 2; ll <= l; ++ll) {
        pll = dsc(1.0 / (double)(ll - m),
                  dsc(2.0 * ll - 1.0, x * pmmp1) - dsc((double)(ll + m) - 1.0, pmm));
        pmm = pmmp1;
        pmmp1 = pll;
      }
      r = pll;
    }
  }
  return dsc((m % 2 == 0) ? 1.0 : -1.0, r);
}

// d O_lm(c) / d c_k, by dual numbers through cart2sph and omultipole
C omultipole_deriv(int l, int m, const double c[3], int k) {
  Dn X[3];
  for (int d = 0; d < 3; ++d) X[d] = {c[d], d == k ? 1.0 : 0.0};
  Dn r = dsqrt((X[0] * X[0] + X[1] * X[1]) + X[2] * X[2]);
  Dn ct = r.v == 0.0 ? Dn{1.0, 0.0} : X[2] / r;
  // phi = atan2(y, x): d phi = (x dy - y dx) / (x^2 + y^2)
  Dn ph = {0.0, 0.0};
  if (!(c[0] == 0.0 && c[1] == 0.0)) {
    ph.v = std::atan2(c[1], c[0]);
    ph.d = (X[0].v * X[1].d - X[1].v * X[0].d) / (X[0].v * X[0].v + X[1].v * X[1].v);
  }
  Dn rl = {1.0, 0.0};
  for (int i = 0; i < l; ++i) rl = rl * r;
  Dn a = dsc(1.0 / factorial(l + m), rl * legendre_p_d(l, m, ct));
  // a exp(-i m phi)
  const double cs = std::cos(m * ph.v), sn = std::sin(m * ph.v);
  const double dcs = -m * sn * ph.d, dsn = m * cs * ph.d;
  return {a.d * cs + a.v * dcs, -(a.d * sn + a.v * dsn)};
}
}  // namespace

void orc_fmm_adjoint(const OrcFmm* f, int64_t nt, const double* tx, const double* ty,
                     const double* tz, const double* gex, const double* gey, const double* gez,
                     const double* gphi, int64_t n, const double* x, const double* y,
                     const double* z, const double* q, double* dq, double* dx, double* dy,
                     double* dz) {
  const double pi = std::acos(-1.0);
  const double prefact = (2.0 * pi) / (3.0 * f->volume);
  const int corr = f->p.fmm_extrinsic_correction;
  // 1. dL/dmu (l <= Lmax_multipole), as G with L = Re sum_{l, m >= 0} G(l, m) mu(l, m),
  //    accumulated over (l, k) with k of either sign and folded afterwards
  const int W = 2 * kLmaxM + 1;
  std::vector<C> A((kLmaxM + 1) * W, {0.0, 0.0});  // A(j, k), k in [-j, j]
  auto Aat = [&](int j, int k) -> C& { return A[j * W + (k + kLmaxM)]; };
  double dbar[3] = {0.0, 0.0, 0.0}, tbar = 0.0;
  std::vector<double> qfbar(f->nfict, 0.0);
  for (int64_t t = 0; t < nt; ++t) {
    const double pos[3] = {tx[t], ty[t], tz[t]};
    double R[3] = {pos[0] - f->center[0], pos[1] - f->center[1], pos[2] - f->center[2]};
    auto s = cart2sph(R);
    // L_t = Re[gphi mus(0,0) + (-gEx + i gEy) mus(1,1) - gEz mus(1,0)],
    // mus(l, m) = sum_{j, k} O_R(j - l, k - m) mu(j, k)  (L2L, :943-976)
    const C c00 = {gphi[t], 0.0}, c11 = {-gex[t], gey[t]}, c10 = {-gez[t], 0.0};
    C OR[kLenM];
    for (int l = 0; l <= kLmaxM; ++l)
      for (int m = 0; m <= l; ++m) OR[tblinv(l, m)] = omultipole(l, m, s);
    for (int j = 0; j <= kLmaxM; ++j)
      for (int k = -j; k <= j; ++k) {
        C acc = cmul(c00, tbl(OR, j, k, kLmaxM));
        if (j >= 1) {
          acc = cadd(acc, cmul(c11, tbl(OR, j - 1, k - 1, kLmaxM)));
          acc = cadd(acc, cmul(c10, tbl(OR, j - 1, k, kLmaxM)));
        }
        Aat(j, k) = cadd(Aat(j, k), acc);
      }
    if (corr == 1) {
      for (int d = 0; d < 3; ++d) dbar[d] += (2.0 * prefact) * (d == 0 ? gex[t] : d == 1 ? gey[t] : gez[t]);
      for (int d = 0; d < 3; ++d) dbar[d] -= (2.0 * prefact) * gphi[t] * R[d];
      tbar += prefact * gphi[t];
    } else if (corr == 2) {
      for (int pp = 0; pp < f->nfict; ++pp)
        for (const auto& bx : f->boxes) {
          double v[3], dd[3];
          f->lvect(bx, v);
          for (int k = 0; k < 3; ++k) dd[k] = (pos[k] - v[k]) - f->fict_pos[pp][k];
          double r = std::sqrt((dd[0] * dd[0] + dd[1] * dd[1]) + dd[2] * dd[2]);
          double rd = 1.0 / r, rd3 = rd * rd * rd;
          qfbar[pp] += gphi[t] * rd + rd3 * ((gex[t] * dd[0] + gey[t] * dd[1]) + gez[t] * dd[2]);
        }
    }
  }
  // fold k < 0: mu(j, -m) = (-1)^m conj(mu(j, m))
  std::vector<C> G(kLenM, {0.0, 0.0});
  for (int j = 0; j <= kLmaxM; ++j)
    for (int m = 0; m <= j; ++m) {
      C g = Aat(j, m);
      if (m > 0) {
        C a = Aat(j, -m);
        double sg = (m % 2 == 0) ? 1.0 : -1.0;
        g = cadd(g, C{sg * a.re, -sg * a.im});
      }
      G[tblinv(j, m)] = g;
    }
  // 2. dL/domega: mu(l, m) = sum_{j, k} (-1)^j ML(j + l, k + m) omega(j, k) (M2L, :912-937)
  std::vector<C> Ob(kLenM, {0.0, 0.0});
  for (int j = 0; j <= kLmaxM; ++j)
    for (int m = 0; m <= j; ++m) {
      C b = {0.0, 0.0}, bn = {0.0, 0.0};  // B(j, m) and B(j, -m)
      const double sj = (j % 2 == 0) ? 1.0 : -1.0;
      for (int l = 0; l <= kLmaxM; ++l)
        for (int mm = 0; mm <= l; ++mm) {
          b = cadd(b, cmul(G[tblinv(l, mm)], cscale(sj, tbl(f->mlattice.data(), j + l, m + mm, kLmaxT))));
          if (m > 0)
            bn = cadd(bn, cmul(G[tblinv(l, mm)], cscale(sj, tbl(f->mlattice.data(), j + l, -m + mm, kLmaxT))));
        }
      if (m > 0) {
        double sg = (m % 2 == 0) ? 1.0 : -1.0;
        b = cadd(b, C{sg * bn.re, -sg * bn.im});
      }
      Ob[tblinv(j, m)] = b;
    }
  // omega(0, 0) never reaches mu: the forward removes it, or it is exactly
  // zero and any change of a charge makes it nonzero and removed.  Its
  // adjoint is therefore zero, which also keeps the divergent ML(0, 0) (of
  // order 1e32 in the unit-cube table) out of every sum below
  Ob[0] = {0.0, 0.0};
  // 3. fictitious charges: q_f from the box dipole (:536-559)
  if (corr == 2) {
    for (int pp = 0; pp < f->nfict; ++pp) {
      double rr[3] = {f->fict_pos[pp][0] - f->center[0], f->fict_pos[pp][1] - f->center[1],
                      f->fict_pos[pp][2] - f->center[2]};
      auto s = cart2sph(rr);
      for (int l = 0; l <= kLmaxM; ++l)
        for (int m = 0; m <= l; ++m) {
          C o = omultipole(l, m, s), w = Ob[tblinv(l, m)];
          qfbar[pp] += w.re * o.re - w.im * o.im;
        }
    }
    const double qlast = qfbar[f->nfict - 1];
    int ip = 0;
    for (int pp = 0; pp < 3; ++pp) {
      if (!f->p.periodicity[pp]) continue;
      const double* L = f->lattice[pp];
      const double len = std::sqrt((L[0] * L[0] + L[1] * L[1]) + L[2] * L[2]);
      dbar[pp] += (qlast - qfbar[ip]) / len;
      ++ip;
    }
  }
  // 4. the particles
  for (int64_t i = 0; i < n; ++i) {
    const double R[3] = {x[i] - f->center[0], y[i] - f->center[1], z[i] - f->center[2]};
    auto s = cart2sph(R);
    double gq = 0.0, gx[3] = {0.0, 0.0, 0.0};
    for (int l = 0; l <= kLmaxM; ++l)
      for (int m = 0; m <= l; ++m) {
        const C w = Ob[tblinv(l, m)];
        const C o = omultipole(l, m, s);
        gq += w.re * o.re - w.im * o.im;
        for (int k = 0; k < 3; ++k) {
          const C od = omultipole_deriv(l, m, R, k);
          gx[k] += w.re * od.re - w.im * od.im;
        }
      }
    if (corr == 1 || corr == 2) {
      gq += (dbar[0] * R[0] + dbar[1] * R[1]) + dbar[2] * R[2];
      for (int k = 0; k < 3; ++k) gx[k] += dbar[k];
    }
    if (corr == 1) {
      gq += tbar * ((R[0] * R[0] + R[1] * R[1]) + R[2] * R[2]);
      for (int k = 0; k < 3; ++k) gx[k] += 2.0 * tbar * R[k];
    }
    dq[i] = gq;
    dx[i] = q[i] * gx[0];
    dy[i] = q[i] * gx[1];
    dz[i] = q[i] * gx[2];
  }
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
