// pepc_oracle.cpp -- CPU FP64 restatement of PEPC's tree-code force evaluation.
//
// TEST INFRASTRUCTURE ONLY: this is the parity checker for libpepcg (the CUDA
// library).  It is loaded by the tests, the smoke check and the CPU-baseline
// leg of the benchmark, never by the product path.
//
// Every routine restates the reference (ALaDyn/pepc, Fortran 2003) and cites
// the file:line it follows.  Paths are relative to the reference's src/ tree.
// Build with -ffp-contract=off: the operation order below is the contract.

#include "pepc_oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace {

constexpr int kMaxLevel = 20;  // treevars.f90:55 -> (64-2)/3 = 20 for idim = 3
constexpr int64_t kNodeInvalid = -1;

// ---------------------------------------------------------------------------
// Box (treecode/lpepcsrc/module_box.f90:48-93)
// ---------------------------------------------------------------------------
struct Box {
  double min[3], max[3], size[3];
};

Box box_create(int64_t n, const double* x, const double* y, const double* z, bool cubic) {
  Box b;
  const double* c[3] = {x, y, z};
  for (int d = 0; d < 3; ++d) {
    double lo = c[d][0], hi = c[d][0];
    for (int64_t i = 1; i < n; ++i) {
      lo = std::min(lo, c[d][i]);
      hi = std::max(hi, c[d][i]);
    }
    b.min[d] = lo;
    b.max[d] = hi;
  }
  if (cubic) {  // module_box.f90:71-74
    double lo = std::min(b.min[0], std::min(b.min[1], b.min[2]));
    double hi = std::max(b.max[0], std::max(b.max[1], b.max[2]));
    for (int d = 0; d < 3; ++d) { b.min[d] = lo; b.max[d] = hi; }
  }
  // module_box.f90:81-84: safety margin of boxsize/10000 on both sides
  for (int d = 0; d < 3; ++d) {
    double s = b.max[d] - b.min[d];
    b.min[d] = b.min[d] - s / 10000.0;
    b.max[d] = b.max[d] + s / 10000.0;
    b.size[d] = b.max[d] - b.min[d];
  }
  return b;
}

// ---------------------------------------------------------------------------
// Keys (treecode/lpepcsrc/module_spacefilling.f90)
// ---------------------------------------------------------------------------
// coord_to_intcoord_with_refinement_length, module_spacefilling.f90:207-219:
// s = boxsize / 2**maxlevel (:238), ic = int((x - boxmin) / s)  (truncation)
inline void coord_to_intcoord(const Box& b, const double s[3], double x, double y, double z,
                              int64_t ic[3]) {
  ic[0] = (int64_t)((x - b.min[0]) / s[0]);
  ic[1] = (int64_t)((y - b.min[1]) / s[1]);
  ic[2] = (int64_t)((z - b.min[2]) / s[2]);
}

// intcoord_to_key_hilbert3D, module_spacefilling.f90:380-440 (Kamata et al.)
const int kCI3[8] = {0, 1, 3, 2, 7, 6, 4, 5};          // :389
const int kG3x[8] = {5, 6, 0, 5, 5, 0, 6, 5};          // :390, G3(:,0) exchange
const int kG3r[8] = {0, 0, 0, 5, 0, 0, 6, 5};          // :390, G3(:,1) reverse

int64_t intcoord_to_key_hilbert3d(const int64_t ic_in[3]) {
  int64_t it[3] = {ic_in[0], ic_in[1], ic_in[2]};
  int64_t key = 1;  // placeholder bit, :402
  for (int i = kMaxLevel - 1; i >= 0; --i) {
    int64_t cval = 0;
    for (int j = 3; j >= 1; --j) {  // :409-412, cval = z<<2 | y<<1 | x
      cval = (cval << 1) | ((it[j - 1] >> i) & 1);
      it[j - 1] &= ~(int64_t(1) << i);
    }
    int h = kCI3[cval];
    int exch = kG3x[h], rev = kG3r[h];
    key = (key << 3) | h;  // :420
    if (exch == 5) std::swap(it[0], it[2]);       // :425-428
    else if (exch == 6) std::swap(it[1], it[2]);  // :429-432
    for (int j = 1; j <= 3; ++j)                  // :436-438
      if ((rev >> (j - 1)) & 1) it[j - 1] = (~it[j - 1]) & ((int64_t(1) << i) - 1);
  }
  return key;
}

// 3D Morton (Z) curve: bit interleave with the same digit convention as the
// Hilbert cell value (z<<2 | y<<1 | x), generalising intcoord_to_key_morton1D
// (module_spacefilling.f90:291-308).  Not in the reference for idim = 3.
int64_t intcoord_to_key_morton3d(const int64_t ic[3]) {
  int64_t key = 1;
  for (int i = kMaxLevel - 1; i >= 0; --i) {
    int64_t cval = (((ic[2] >> i) & 1) << 2) | (((ic[1] >> i) & 1) << 1) | ((ic[0] >> i) & 1);
    key = (key << 3) | cval;
  }
  return key;
}

// level_from_key, module_spacefilling.f90:47-57
inline int level_from_key(int64_t key) {
  return (63 - __builtin_clzll((unsigned long long)key)) / 3;
}

// key_to_intcoord_hilbert, module_spacefilling.f90:501-565
void key_to_intcoord_hilbert(int64_t key, int64_t ic[3]) {
  static const int C3[8] = {0, 1, 3, 2, 6, 7, 5, 4};  // :515
  int lev = level_from_key(key);
  ic[0] = ic[1] = ic[2] = 0;
  for (int i = 0; i < lev; ++i) {
    int h = (int)((key >> (3 * i)) & 7);
    int cval = C3[h], rev = kG3r[h], exch = kG3x[h];
    if (i > 0) {
      for (int j = 1; j <= 3; ++j)
        if ((rev >> (j - 1)) & 1) ic[j - 1] = (~ic[j - 1]) & ((int64_t(1) << i) - 1);
      for (int j = 1; j <= 2; ++j) {
        if (!((exch >> (j - 1)) & 1)) continue;
        for (int k = j + 1; k <= 3; ++k)
          if ((exch >> (k - 1)) & 1) std::swap(ic[j - 1], ic[k - 1]);
      }
    }
    for (int j = 1; j <= 3; ++j) ic[j - 1] |= (int64_t)((cval >> (j - 1)) & 1) << i;
  }
  for (int j = 0; j < 3; ++j) ic[j] <<= (kMaxLevel - lev);
}

void key_to_intcoord_morton3d(int64_t key, int64_t ic[3]) {
  int lev = level_from_key(key);
  ic[0] = ic[1] = ic[2] = 0;
  for (int i = 0; i < lev; ++i)
    for (int j = 0; j < 3; ++j) ic[j] |= ((key >> (3 * i + j)) & 1) << i;
  for (int j = 0; j < 3; ++j) ic[j] <<= (kMaxLevel - lev);
}

// key_to_coord, module_spacefilling.f90:445-471
void key_to_coord(const Box& b, int64_t key, int curve, double x[3]) {
  int64_t ic[3];
  if (curve == 1) key_to_intcoord_morton3d(key, ic);
  else key_to_intcoord_hilbert(key, ic);
  for (int d = 0; d < 3; ++d) {
    double s = b.size[d] / (double)(int64_t(1) << kMaxLevel);
    x[d] = ((double)ic[d] + 0.5) * s + b.min[d];
  }
}

// ---------------------------------------------------------------------------
// Local key sort: restatement of the SL library's in-place MSD radix sort
// (treecode/sl_pepc/src/core/sort_radix.c:33-119 rs_rec_ip, :122-151
// sort_radix_ip; width 10 and insertion threshold 256 from
// src/include/sl_tune_intern.h:22,30; insertion kernel sort_insert.c:14-37).
// The element is (key, index); the reference also carries the work weight,
// which does not influence the order.
// ---------------------------------------------------------------------------
void insert_sort_bmask(int64_t* k, int64_t* ix, int64_t n, uint64_t bmask) {
  for (int64_t i = 1; i < n; ++i) {
    if ((uint64_t(k[i]) & bmask) < (uint64_t(k[i - 1]) & bmask)) {
      int64_t j = i - 1;
      int64_t tk = k[i], ti = ix[i];
      do {
        k[j + 1] = k[j];
        ix[j + 1] = ix[j];
        if (--j < 0) break;
      } while ((uint64_t(tk) & bmask) < (uint64_t(k[j]) & bmask));
      k[j + 1] = tk;
      ix[j + 1] = ti;
    }
  }
}

void rs_rec_ip(int64_t* k, int64_t* ix, int64_t n, int rhigh, int rlow, int rwidth) {
  const int width = std::min(rwidth, rhigh - rlow + 1);
  rhigh -= width - 1;
  const int64_t ncls = int64_t(1) << width;
  const int64_t mask = ncls - 1;
  std::vector<int64_t> c(ncls, 0), parts(ncls);
  auto cls = [&](int64_t key) { return (key >> rhigh) & mask; };
  for (int64_t i = 0; i < n; ++i) ++c[cls(k[i])];
  parts[0] = 0;
  for (int64_t i = 1; i < ncls; ++i) parts[i] = parts[i - 1] + c[i - 1];
  int64_t end = 0;
  for (int64_t i = 0; i < ncls; ++i) {
    end += c[i];
    int64_t xi = parts[i];
    while (xi < end) {
      int64_t j = cls(k[xi]);
      while (j != i) {
        int64_t kk = cls(k[parts[j]]);
        if (kk != j) {
          std::swap(k[xi], k[parts[j]]);
          std::swap(ix[xi], ix[parts[j]]);
        }
        ++parts[j];
        j = kk;
      }
      ++xi;
    }
  }
  --rhigh;
  if (rhigh >= rlow) {
    uint64_t bmask = 0;
    if (rhigh - rlow + 1 <= 63) bmask = uint64_t(1) << (rhigh - rlow + 1);
    bmask = (bmask - 1) << rlow;
    int64_t off = 0;
    for (int64_t i = 0; i < ncls; ++i) {
      if (c[i] > 256) rs_rec_ip(k + off, ix + off, c[i], rhigh, rlow, rwidth);
      else if (c[i] > 1) insert_sort_bmask(k + off, ix + off, c[i], bmask);
      off += c[i];
    }
  }
}

// ---------------------------------------------------------------------------
// Coulomb backend (interaction_specific/coulomb/)
// Moment record layout = t_tree_node_interaction_data
// (module_interaction_specific_types_XYZQVM.f90:47-57):
//   0..2 coc, 3 charge, 4 abs_charge, 5..7 dip, 8..10 quad, 11 xyquad,
//   12 yzquad, 13 zxquad, 14 bmax
// ---------------------------------------------------------------------------
enum { M_COCX = 0, M_COCY, M_COCZ, M_Q, M_ABSQ, M_DX, M_DY, M_DZ, M_QXX, M_QYY, M_QZZ,
       M_XY, M_YZ, M_ZX, M_BMAX, M_N };

// multipole_from_particle, coulomb/module_interaction_specific.f90:67-79
void multipole_from_particle(const double pos[3], double q, double* m) {
  m[M_COCX] = pos[0]; m[M_COCY] = pos[1]; m[M_COCZ] = pos[2];
  m[M_Q] = q;
  m[M_ABSQ] = std::fabs(q);
  for (int i = M_DX; i < M_N; ++i) m[i] = 0.0;
}

// shift_multipoles_up, coulomb/module_interaction_specific.f90:84-140
void shift_multipoles_up(double* p, const double* const* ch, int nc) {
  double charge = 0.0, absq = 0.0;
  for (int j = 0; j < nc; ++j) charge = charge + ch[j][M_Q];   // :96
  for (int j = 0; j < nc; ++j) absq = absq + ch[j][M_ABSQ];    // :97
  double coc[3] = {0.0, 0.0, 0.0};
  if (absq != 0.0) {  // :102-108
    for (int j = 0; j < nc; ++j)
      for (int d = 0; d < 3; ++d) coc[d] = coc[d] + ch[j][M_COCX + d] * ch[j][M_ABSQ];
    for (int d = 0; d < 3; ++d) coc[d] = coc[d] / absq;
  } else {  // :110-116, geometric mean of the children
    for (int j = 0; j < nc; ++j)
      for (int d = 0; d < 3; ++d) coc[d] = coc[d] + ch[j][M_COCX + d];
    for (int d = 0; d < 3; ++d) coc[d] = coc[d] / (double)nc;
  }
  double dip[3] = {0, 0, 0}, quad[3] = {0, 0, 0}, xy = 0, yz = 0, zx = 0;
  for (int j = 0; j < nc; ++j) {  // :125-137
    const double* c = ch[j];
    double s[3];
    for (int d = 0; d < 3; ++d) s[d] = coc[d] - c[M_COCX + d];
    for (int d = 0; d < 3; ++d) dip[d] = (dip[d] + c[M_DX + d]) + c[M_Q] * s[d];
    for (int d = 0; d < 3; ++d)
      quad[d] = ((quad[d] + c[M_QXX + d]) + c[M_DX + d] * s[d]) + (0.5 * c[M_Q]) * (s[d] * s[d]);
    xy = (((xy + c[M_XY]) + c[M_DX] * s[1]) + c[M_DY] * s[0]) + (c[M_Q] * s[0]) * s[1];
    yz = (((yz + c[M_YZ]) + c[M_DY] * s[2]) + c[M_DZ] * s[1]) + (c[M_Q] * s[1]) * s[2];
    zx = (((zx + c[M_ZX]) + c[M_DZ] * s[0]) + c[M_DX] * s[2]) + (c[M_Q] * s[2]) * s[0];
  }
  double bmax = 0.0;  // :139
  for (int j = 0; j < nc; ++j) {
    const double* c = ch[j];
    double a = coc[0] - c[M_COCX], b = coc[1] - c[M_COCY], d = coc[2] - c[M_COCZ];
    double v = std::sqrt((a * a + b * b) + d * d) + c[M_BMAX];
    if (j == 0 || v > bmax) bmax = v;
  }
  p[M_COCX] = coc[0]; p[M_COCY] = coc[1]; p[M_COCZ] = coc[2];
  p[M_Q] = charge; p[M_ABSQ] = absq;
  p[M_DX] = dip[0]; p[M_DY] = dip[1]; p[M_DZ] = dip[2];
  p[M_QXX] = quad[0]; p[M_QYY] = quad[1]; p[M_QZZ] = quad[2];
  p[M_XY] = xy; p[M_YZ] = yz; p[M_ZX] = zx; p[M_BMAX] = bmax;
}

// calc_force_coulomb_3D_direct, coulomb/module_coulomb_kernels.f90:242-257
inline void force_leaf(const double* t, const double d[3], double dist2, double e[3],
                       double& phi) {
  double r = std::sqrt(dist2);
  double rd = 1.0 / r;
  double rd3charge = ((t[M_Q] * rd) * rd) * rd;
  phi = t[M_Q] * rd;
  e[0] = rd3charge * d[0];
  e[1] = rd3charge * d[1];
  e[2] = rd3charge * d[2];
}

// calc_force_coulomb_3D, coulomb/module_coulomb_kernels.f90:60-145
inline void force_twig(const double* t, const double d[3], double dist2, double e[3],
                       double& phi) {
  const double dx = d[0], dy = d[1], dz = d[2];
  const double r = std::sqrt(dist2);
  const double rd = 1.0 / r;
  const double rd2 = rd * rd;
  const double rd3 = rd * rd2;
  const double rd5 = rd3 * rd2;
  const double rd7 = rd5 * rd2;
  const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
  const double fdx = ((3.0 * dx2) * rd5) - rd3;
  const double fdy = ((3.0 * dy2) * rd5) - rd3;
  const double fdz = ((3.0 * dz2) * rd5) - rd3;
  const double fdxy = ((3.0 * dx) * dy) * rd5;
  const double fdyz = ((3.0 * dy) * dz) * rd5;
  const double fdxz = ((3.0 * dx) * dz) * rd5;
  const double m2rd5 = 2.0 * rd5;
  const double m5rd7 = 5.0 * rd7;
  const double pre1 = ((m5rd7 * dx) * dy) * dz;
  const double pre2x = (m5rd7 * dx2) - rd5;
  const double pre2y = (m5rd7 * dy2) - rd5;
  const double pre2z = (m5rd7 * dz2) - rd5;
  const double preQx = pre2x * t[M_QXX];
  const double preQy = pre2y * t[M_QYY];
  const double preQz = pre2z * t[M_QZZ];
  phi = (((((((t[M_Q] * rd) - (((dx * t[M_DX]) + (dy * t[M_DY])) + (dz * t[M_DZ])) * rd3)
            + fdx * t[M_QXX]) + fdy * t[M_QYY]) + fdz * t[M_QZZ]) + fdxy * t[M_XY])
         + fdyz * t[M_YZ]) + fdxz * t[M_ZX];
  e[0] = (((t[M_Q] * dx) * rd3) - (((fdx * t[M_DX]) + (fdxy * t[M_DY])) + (fdxz * t[M_DZ])))
         + 3.0 * ((((dx * ((((pre2x - m2rd5) * t[M_QXX]) + preQy) + preQz))
                    + ((dy * pre2x) * t[M_XY])) + ((dz * pre2x) * t[M_ZX])) + (pre1 * t[M_YZ]));
  e[1] = (((t[M_Q] * dy) * rd3) - (((fdy * t[M_DY]) + (fdxy * t[M_DX])) + (fdyz * t[M_DZ])))
         + 3.0 * ((((dy * ((((pre2y - m2rd5) * t[M_QYY]) + preQx) + preQz))
                    + ((dx * pre2y) * t[M_XY])) + ((dz * pre2y) * t[M_YZ])) + (pre1 * t[M_ZX]));
  e[2] = (((t[M_Q] * dz) * rd3) - (((fdz * t[M_DZ]) + (fdyz * t[M_DY])) + (fdxz * t[M_DX])))
         + 3.0 * ((((dz * ((((pre2z - m2rd5) * t[M_QZZ]) + preQy) + preQx))
                    + ((dx * pre2z) * t[M_ZX])) + ((dy * pre2z) * t[M_YZ])) + (pre1 * t[M_XY]));
}

// The 2D Coulomb and Lennard-Jones kernels are templates on the scalar type:
// double for the walk, std::complex<double> for the complex-step derivative of
// the adjoint (orc_traverse_adjoint with force_law 2 or 4).  rv() is the real
// part, for the one comparison (calc_force_LJ's cutoff).
inline double rv(double x) { return x; }
inline double rv(const std::complex<double>& x) { return x.real(); }

// calc_force_coulomb_2D_direct, coulomb/module_coulomb_kernels.f90:267-279
// (d2 = dx^2 + dy^2 + eps2)
template <class T>
inline void force_leaf_2d(const double* t, const T d[3], T d2, T e[3], T& phi) {
  using std::log;
  phi = -((0.5 * t[M_Q]) * log(d2));
  const T rd2charge = t[M_Q] / d2;
  e[0] = rd2charge * d[0];
  e[1] = rd2charge * d[1];
  e[2] = 0.0;
}

// calc_force_coulomb_2D, coulomb/module_coulomb_kernels.f90:155-195
template <class T>
inline void force_twig_2d(const double* t, const T d[3], T d2, T e[3], T& phi) {
  using std::log;
  const T dx = d[0], dy = d[1];
  const T rd2 = 1.0 / d2, rd4 = rd2 * rd2, rd6 = rd4 * rd2;
  const T dx2 = dx * dx, dy2 = dy * dy, dx3 = dx2 * dx, dy3 = dy2 * dy;
  const double q = t[M_Q], p1 = t[M_DX], p2 = t[M_DY];
  const double q1 = t[M_QXX], q2 = t[M_QYY], qxy = t[M_XY];
  phi = ((((-((0.5 * q) * log(d2))) - ((dx * p1) + (dy * p2)) * rd2) +
          q1 * (((2.0 * dx2) * rd4) - rd2)) +
         q2 * (((2.0 * dy2) * rd4) - rd2)) +
        (((2.0 * qxy) * dx) * dy) * rd4;
  e[0] = (((((q * dx) * rd2 - p1 * (((2.0 * dx2) * rd4) - rd2)) - (((p2 * 2.0) * dx) * dy) * rd4) +
           q1 * (((8.0 * dx3) * rd6) - ((6.0 * dx) * rd4))) +
          q2 * ((((8.0 * dx) * dy2) * rd6) - ((2.0 * dx) * rd4))) +
         qxy * ((((8.0 * dx2) * dy) * rd6) - ((2.0 * dy) * rd4));
  e[1] = (((((q * dy) * rd2 - p2 * (((2.0 * dy2) * rd4) - rd2)) - (((p1 * 2.0) * dx) * dy) * rd4) +
           q2 * (((8.0 * dy3) * rd6) - ((6.0 * dy) * rd4))) +
          q1 * ((((8.0 * dy) * dx2) * rd6) - ((2.0 * dy) * rd4))) +
         qxy * ((((8.0 * dy2) * dx) * rd6) - ((2.0 * dx) * rd4));
  e[2] = 0.0;
}

// calc_force_LJ, coulomb/module_coulomb_kernels.f90:204-235 (r2 unsoftened,
// aii2 = eps2; the same for leaves and twigs)
template <class T>
inline void force_lj(const T d[3], T r2, double aii2, T e[3], T& phi) {
  using std::sqrt;
  const double epsc2 = 0.8 * aii2;
  const T aii2_r2 = (rv(r2) > epsc2) ? T(aii2 / r2) : T(aii2 / epsc2);
  const T aii4_r4 = aii2_r2 * aii2_r2;
  const T flj = 2.0 * (aii4_r4 * aii4_r4) - aii4_r4;
  phi = 0.0;
  const T r = sqrt(r2);
  const T fljrd = flj / r;
  e[0] = d[0] * fljrd;
  e[1] = d[1] * fljrd;
  e[2] = d[2] * fljrd;
}

// calc_force_per_interaction_with_leaf / _with_twig
// (coulomb/module_interaction_specific.f90:314-387): the force law's kernel
// for an unsoftened |delta|^2
// calc_force_kelbg_3D_direct, coulomb/module_coulomb_kernels.f90:286-325
// (tq: the target's charge; dist2 unsoftened)
inline void force_kelbg(double tq, const double* t, const double d[3], double dist2, double kinv,
                        double e[3], double& phi) {
  const double q = t[M_Q];
  double lambda;
  if (tq * q < 0.0) lambda = 1.00027227 * kinv;      // e-i
  else if (q > 0.0) lambda = 0.03300355 * kinv;      // i-i
  else lambda = 1.41421356 * kinv;                   // e-e
  const double sqrtpi = std::sqrt(std::acos(-1.0));
  const double r = std::sqrt(dist2);
  const double rd = 1.0 / r;
  const double rd3 = (rd * rd) * rd;
  const double rol = r / lambda;
  const double ome = 1.0 - std::exp(-(rol * rol));
  phi = (q * rd) * (ome + (sqrtpi * rol) * (1.0 - std::erf(rol)));
  const double fprefac = (q * rd3) * ome;
  e[0] = fprefac * d[0];
  e[1] = fprefac * d[1];
  e[2] = fprefac * d[2];
}

inline void law_leaf(int law, const double* t, const double d[3], double dist2, double eps2,
                     double e[3], double& phi, double tq = 0.0, double kinv = 0.0) {
  switch (law) {
    case 2:
      force_leaf_2d(t, d, (d[0] * d[0] + d[1] * d[1]) + eps2, e, phi);
      break;
    case 4:
      force_lj(d, dist2, eps2, e, phi);
      break;
    case 5:
      force_kelbg(tq, t, d, dist2, kinv, e, phi);
      break;
    default:
      force_leaf(t, d, dist2 + eps2, e, phi);
  }
}
inline void law_twig(int law, const double* t, const double d[3], double dist2, double eps2,
                     double e[3], double& phi) {
  switch (law) {
    case 2:
      force_twig_2d(t, d, (d[0] * d[0] + d[1] * d[1]) + eps2, e, phi);
      break;
    case 4:
      force_lj(d, dist2, eps2, e, phi);
      break;
    case 5:  // multipole expansion with Coulomb, unsoftened (specific.f90:375-378)
      force_twig(t, d, dist2, e, phi);
      break;
    default:
      force_twig(t, d, dist2 + eps2, e, phi);
  }
}

// ---------------------------------------------------------------------------
// Mirror boxes (treecode/lpepcsrc/module_mirror_boxes.f90:73-156)
// ---------------------------------------------------------------------------
std::vector<std::array<int, 3>> neighbour_boxes(const orc_params& p) {
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
  nb.push_back({0, 0, 0});  // central box last, :151
  return nb;
}

// lattice_vect, module_mirror_boxes.f90:73-79 (integer * real promotes to FP64)
void lattice_vect(const orc_params& p, const std::array<int, 3>& ijk, double v[3]) {
  for (int d = 0; d < 3; ++d)
    v[d] = ((double)ijk[0] * p.t_lattice_1[d] + (double)ijk[1] * p.t_lattice_2[d])
           + (double)ijk[2] * p.t_lattice_3[d];
}

}  // namespace

// forward declarations of the periodic lattice term (pepc_oracle_fmm.cpp)
struct OrcFmm;
OrcFmm* orc_fmm_create(const orc_params& p);
void orc_fmm_destroy(OrcFmm* f);
void orc_fmm_timestep(OrcFmm* f, int64_t n, const double* x, const double* y, const double* z,
                      const double* q);
void orc_fmm_sum_lattice_force(const OrcFmm* f, const double pos[3], double e[3], double* phi);
void orc_fmm_set_mlattice(OrcFmm* f, const double* re_im);
void orc_fmm_adjoint(const OrcFmm* f, int64_t nt, const double* tx, const double* ty,
                     const double* tz, const double* gex, const double* gey, const double* gez,
                     const double* gphi, int64_t n, const double* x, const double* y,
                     const double* z, const double* q, double* dq, double* dx, double* dy,
                     double* dz);

// ---------------------------------------------------------------------------
// Whole-path context
// ---------------------------------------------------------------------------
struct Node {
  int64_t key;
  int32_t level;
  int64_t leaves, descendants;
  int64_t parent, first_child, next_sibling;
  int64_t particle;  // leaf: key-ordered particle index; twig: -1
  double m[M_N];
};

struct orc_ctx {
  orc_params p;
  Box box;
  int64_t n = 0;
  std::vector<int64_t> keys, perm;
  std::vector<double> x, y, z, q;
  std::vector<Node> nodes;
  int64_t root = kNodeInvalid;
  double boxlength2[kMaxLevel + 1];
  int64_t n_interactions = 0, n_mac = 0;
  OrcFmm* fmm = nullptr;
  bool periodic_far() const {
    return (p.periodicity[0] || p.periodicity[1] || p.periodicity[2]) &&
           p.include_far_field_if_periodic;
  }
};

// mac (coulomb/module_interaction_specific.f90:256-275): Barnes-Hut, Bmax
// (min(bmax^2, 3 boxlength2)), or no acceptance at all (the N^2 code)
static bool mac_pass(const orc_ctx* c, const Node& nd, double dist2) {
  const double bl2 = c->boxlength2[nd.level];
  switch (c->p.mac_select) {
    case 0:
      return c->p.theta2 * dist2 > bl2;
    case 1:
      return c->p.theta2 * dist2 > std::min(nd.m[M_BMAX] * nd.m[M_BMAX], 3.0 * bl2);
    default:
      return false;
  }
}


namespace {

// tree_node_create_from_particle, module_tree_grow.f90:702-734
int64_t make_leaf(orc_ctx* c, int64_t k, int64_t ip) {
  Node nd{};
  nd.key = k;
  nd.level = level_from_key(k);
  nd.leaves = 1;
  nd.descendants = 0;
  nd.parent = nd.first_child = nd.next_sibling = kNodeInvalid;
  nd.particle = ip;
  double pos[3] = {c->x[ip], c->y[ip], c->z[ip]};
  multipole_from_particle(pos, c->q[ip], nd.m);
  c->nodes.push_back(nd);
  return (int64_t)c->nodes.size() - 1;
}

// tree_node_update_from_children, module_tree_grow.f90:762-821 (+ connect, module_tree.f90:409-433)
void update_from_children(orc_ctx* c, int64_t pi, const std::vector<int64_t>& ch) {
  Node& p = c->nodes[pi];
  p.leaves = 0;
  p.descendants = (int64_t)ch.size();
  const double* cm[8];
  for (size_t i = 0; i < ch.size(); ++i) {
    p.leaves += c->nodes[ch[i]].leaves;
    p.descendants += c->nodes[ch[i]].descendants;
    cm[i] = c->nodes[ch[i]].m;
  }
  shift_multipoles_up(p.m, cm, (int)ch.size());
  p.first_child = ch[0];
  for (size_t i = 0; i < ch.size(); ++i) {
    c->nodes[ch[i]].parent = pi;
    c->nodes[ch[i]].next_sibling = (i + 1 < ch.size()) ? ch[i + 1] : kNodeInvalid;
  }
}

// insert_helper, module_tree_grow.f90:623-696 (node indices in insertion order)
int64_t insert_helper(orc_ctx* c, int64_t k, int l, int64_t& cur, int& err) {
  const int64_t n = c->n;
  auto is_anc = [&](int64_t kp) { return k == (kp >> (3 * (kMaxLevel - l))); };
  bool first = cur < n && is_anc(c->keys[cur]);
  bool second = cur + 1 < n && is_anc(c->keys[cur + 1]);
  if (!first && !second) return kNodeInvalid;
  if (first && !second) {
    int64_t nd = make_leaf(c, k, cur);
    ++cur;
    return nd;
  }
  if (l >= kMaxLevel) {  // :671-675, "no more levels"
    err = -2;
    return kNodeInvalid;
  }
  Node tw{};
  tw.key = k;
  tw.level = l;
  tw.particle = -1;
  tw.parent = tw.first_child = tw.next_sibling = kNodeInvalid;
  c->nodes.push_back(tw);
  int64_t me = (int64_t)c->nodes.size() - 1;
  std::vector<int64_t> ch;
  for (int ic = 0; ic < 8; ++ic) {
    int64_t cn = insert_helper(c, (k << 3) + ic, l + 1, cur, err);
    if (err) return kNodeInvalid;
    if (cn != kNodeInvalid) ch.push_back(cn);
  }
  update_from_children(c, me, ch);
  return me;
}

struct Counters {
  int64_t inter = 0, mac = 0;
};

// any(abs(delta) >= spatial_interaction_cutoff): the node is skipped
// (module_tree_walk_pthreads.f90:622,639, module_tree_walk_simple.f90:330,377)
inline bool cut_off(const orc_ctx* c, const double d[3]) {
  const double* sc = c->p.spatial_interaction_cutoff;
  return std::fabs(d[0]) >= sc[0] || std::fabs(d[1]) >= sc[1] || std::fabs(d[2]) >= sc[2];
}

// walk_single_particle, treecode/lpepcsrc/module_tree_walk_pthreads.f90:558-765.
// At one rank every child is local, so the defer list only ever holds the
// root (:601 parses it once and pushes the root's children); the todo list is
// a LIFO stack.  Returns the number of partner leaves (completeness check :452).
int64_t walk_pthreads(const orc_ctx* c, const double xt[3], const double vbox[3], double e[3],
                      double& pot, double& work, Counters& cnt, std::vector<int64_t>& todo,
                      double tq) {
  const double shifted[3] = {xt[0] - vbox[0], xt[1] - vbox[1], xt[2] - vbox[2]};  // :595
  int64_t partner = 0;
  todo.clear();
  for (int64_t ch = c->nodes[c->root].first_child; ch != kNodeInvalid;
       ch = c->nodes[ch].next_sibling)
    todo.push_back(ch);
  const double eps2 = c->p.eps2;
  while (!todo.empty()) {
    int64_t ni = todo.back();
    todo.pop_back();
    const Node& nd = c->nodes[ni];
    double d[3] = {shifted[0] - nd.m[M_COCX], shifted[1] - nd.m[M_COCY],
                   shifted[2] - nd.m[M_COCZ]};  // :614
    double dist2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];  // :615
    if (nd.descendants == 0) {  // leaf, :617-631
      partner += 1;
      work += 1.0;
      if (cut_off(c, d)) continue;  // :622, after the work count
      if (dist2 > 0.0) {
        double ee[3], ph;
        law_leaf(c->p.force_law, nd.m, d, dist2, eps2, ee, ph, tq, c->p.kelbg_invsqrttemp);  // specific.f90:327-343
        e[0] += ee[0]; e[1] += ee[1]; e[2] += ee[2];
        pot += ph;
      }
      cnt.inter += 1;
    } else {
      cnt.mac += 1;
      if (mac_pass(c, nd, dist2)) {  // mac, :635 / specific.f90:256-275
        partner += nd.leaves;
        if (cut_off(c, d)) continue;  // :639, before the work count
        double ee[3], ph;
        law_twig(c->p.force_law, nd.m, d, dist2, eps2, ee, ph);  // specific.f90:368-380
        e[0] += ee[0]; e[1] += ee[1]; e[2] += ee[2];
        pot += ph;
        cnt.inter += 1;
        work += 1.0;
      } else {  // resolve: push all children, first .. last (:660-725)
        for (int64_t ch = nd.first_child; ch != kNodeInvalid; ch = c->nodes[ch].next_sibling)
          todo.push_back(ch);
      }
    }
  }
  return partner;
}

// tree_walk_single_aux, treecode/lpepcsrc/module_tree_walk_simple.f90:301-384
void walk_simple_aux(const orc_ctx* c, int64_t ni, int np, const double (*xs)[3],
                     const double vbox[3], double (*e)[3], double* pot, double* work,
                     int64_t& partner, Counters& cnt, const double* tqs) {
  const Node& nd = c->nodes[ni];
  const double eps2 = c->p.eps2;
  double d[64][3], d2[64];
  if (nd.descendants == 0) {
    partner += 1;
    for (int ip = 0; ip < np; ++ip) {
      for (int k = 0; k < 3; ++k) d[ip][k] = (xs[ip][k] - vbox[k]) - nd.m[M_COCX + k];
      if (cut_off(c, d[ip])) continue;  // :330, before the work count
      d2[ip] = (d[ip][0] * d[ip][0] + d[ip][1] * d[ip][1]) + d[ip][2] * d[ip][2];
      cnt.inter += 1;
      work[ip] += 1.0;
      if (d2[ip] > 0.0) {
        double ee[3], ph;
        law_leaf(c->p.force_law, nd.m, d[ip], d2[ip], eps2, ee, ph, tqs[ip], c->p.kelbg_invsqrttemp);
        e[ip][0] += ee[0]; e[ip][1] += ee[1]; e[ip][2] += ee[2];
        pot[ip] += ph;
      }
    }
    return;
  }
  for (int ip = 0; ip < np; ++ip) {
    cnt.mac += 1;
    for (int k = 0; k < 3; ++k) d[ip][k] = (xs[ip][k] - vbox[k]) - nd.m[M_COCX + k];
    d2[ip] = (d[ip][0] * d[ip][0] + d[ip][1] * d[ip][1]) + d[ip][2] * d[ip][2];
    if (!mac_pass(c, nd, d2[ip])) {  // MAC fails for this target: resolve
      for (int64_t ch = nd.first_child; ch != kNodeInvalid; ch = c->nodes[ch].next_sibling)
        walk_simple_aux(c, ch, np, xs, vbox, e, pot, work, partner, cnt, tqs);
      return;
    }
  }
  partner += nd.leaves;  // MAC OK for the whole tile: interact
  for (int ip = 0; ip < np; ++ip) {
    if (cut_off(c, d[ip])) continue;  // :377
    cnt.inter += 1;
    work[ip] += 1.0;
    double ee[3], ph;
    law_twig(c->p.force_law, nd.m, d[ip], d2[ip], eps2, ee, ph);
    e[ip][0] += ee[0]; e[ip][1] += ee[1]; e[ip][2] += ee[2];
    pot[ip] += ph;
  }
}

// tree_walk_init_aux, module_tree_walk_simple.f90:168-211: recursive split of
// the key-ordered targets into tiles of at most tile_size.
void make_tiles(const int64_t* keys, int64_t lo, int64_t hi, int64_t k, int l, int ts,
                std::vector<std::pair<int64_t, int64_t>>& tiles, int& err) {
  int64_t np = hi - lo;
  if (np == 0) return;
  if (np <= ts) {
    tiles.push_back({lo, hi});
    return;
  }
  if (l >= kMaxLevel) {
    err = -2;
    return;
  }
  int64_t ps = lo;
  for (int ic = 0; ic < 8; ++ic) {
    int64_t ck = (k << 3) + ic;
    int64_t pe = ps;
    while (pe < hi && (keys[pe] >> (3 * (kMaxLevel - (l + 1)))) == ck) ++pe;
    make_tiles(keys, ps, pe, ck, l + 1, ts, tiles, err);
    if (err) return;
    ps = pe;
  }
}

template <class F>
void parallel_for(int64_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 64) {
    for (int64_t i = 0; i < n; ++i) f(i, 0);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t)
    th.emplace_back([&, t] {
      for (;;) {
        int64_t i0 = next.fetch_add(64);
        if (i0 >= n) break;
        int64_t i1 = std::min(n, i0 + 64);
        for (int64_t i = i0; i < i1; ++i) f(i, t);
      }
    });
  for (auto& t : th) t.join();
}


// ---------------------------------------------------------------------------
// Adjoint of the walk (checker for pepcg_traverse_adjoint; the reference has
// no adjoint).  Writing the twig potential as
//   phi = q D0 + p_k D1_k + sum_{kl in xx,yy,zz,xy,yz,zx} Q_kl D2_kl
// with D the Cartesian derivative tensors of 1/r (r^2 = |d|^2 + eps^2) --
// which is exactly calc_force_coulomb_3D (module_coulomb_kernels.f90:60-145)
// -- one target-node pair with dL/dphi = gphi, dL/dE = gE contributes
//   qbar += gphi D0 - gE.D1,  pbar_k += gphi D1_k - gE_i D2_ik,
//   Qbar_kl += gphi D2_kl - gE_i D3_ikl,  cocbar += gphi E + H gE
// (E = -grad phi, H = the Hessian of phi).  The interaction lists are held
// fixed (the MAC and the keys are piecewise constant).
// ---------------------------------------------------------------------------
struct Tens {
  double d[3], R[5];
  void set(const double dd[3], double eps2) {
    d[0] = dd[0]; d[1] = dd[1]; d[2] = dd[2];
    const double r2 = ((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]) + eps2;
    const double r0 = 1.0 / std::sqrt(r2);
    const double r02 = r0 * r0;
    R[0] = r0;
    R[1] = R[0] * r02;
    R[2] = R[1] * r02;
    R[3] = R[2] * r02;
    R[4] = R[3] * r02;
  }
  static double dl(int i, int j) { return i == j ? 1.0 : 0.0; }
  double D1(int i) const { return -d[i] * R[1]; }
  double D2(int i, int j) const { return 3.0 * d[i] * d[j] * R[2] - dl(i, j) * R[1]; }
  double D3(int i, int j, int k) const {
    return -15.0 * d[i] * d[j] * d[k] * R[3] +
           3.0 * R[2] * (dl(i, j) * d[k] + dl(i, k) * d[j] + dl(j, k) * d[i]);
  }
  double D4(int i, int j, int k, int l) const {
    return 105.0 * d[i] * d[j] * d[k] * d[l] * R[4] -
           15.0 * R[3] *
               (dl(i, j) * d[k] * d[l] + dl(i, k) * d[j] * d[l] + dl(i, l) * d[j] * d[k] +
                dl(j, k) * d[i] * d[l] + dl(j, l) * d[i] * d[k] + dl(k, l) * d[i] * d[j]) +
           3.0 * R[2] * (dl(i, j) * dl(k, l) + dl(i, k) * dl(j, l) + dl(i, l) * dl(j, k));
  }
};

const int kQK[6] = {0, 1, 2, 0, 1, 2};  // moment order xx yy zz xy yz zx
const int kQL[6] = {0, 1, 2, 1, 2, 0};

struct Adj {
  double q = 0, p[3] = {0, 0, 0}, Q[6] = {0, 0, 0, 0, 0, 0}, c[3] = {0, 0, 0}, A = 0;
};

void twig_adjoint(const double* m, const double d[3], double eps2, double gphi, const double gE[3],
                  Adj& a) {
  Tens T;
  T.set(d, eps2);
  const double q = m[M_Q];
  const double p[3] = {m[M_DX], m[M_DY], m[M_DZ]};
  const double Q[6] = {m[M_QXX], m[M_QYY], m[M_QZZ], m[M_XY], m[M_YZ], m[M_ZX]};
  a.q += gphi * T.R[0];
  for (int i = 0; i < 3; ++i) a.q -= gE[i] * T.D1(i);
  for (int k = 0; k < 3; ++k) {
    double v = gphi * T.D1(k);
    for (int i = 0; i < 3; ++i) v -= gE[i] * T.D2(i, k);
    a.p[k] += v;
  }
  for (int s = 0; s < 6; ++s) {
    double v = gphi * T.D2(kQK[s], kQL[s]);
    for (int i = 0; i < 3; ++i) v -= gE[i] * T.D3(i, kQK[s], kQL[s]);
    a.Q[s] += v;
  }
  for (int j = 0; j < 3; ++j) {
    double E = q * T.D1(j);
    for (int k = 0; k < 3; ++k) E += p[k] * T.D2(j, k);
    for (int s = 0; s < 6; ++s) E += Q[s] * T.D3(j, kQK[s], kQL[s]);
    E = -E;
    double hg = 0.0;
    for (int i = 0; i < 3; ++i) {
      double H = q * T.D2(i, j);
      for (int k = 0; k < 3; ++k) H += p[k] * T.D3(i, j, k);
      for (int s = 0; s < 6; ++s) H += Q[s] * T.D4(i, j, kQK[s], kQL[s]);
      hg += H * gE[i];
    }
    a.c[j] += gphi * E + hg;
  }
}

void leaf_adjoint(double q, const double d[3], double eps2, double gphi, const double gE[3],
                  Adj& a) {
  Tens T;
  T.set(d, eps2);
  a.q += gphi * T.R[0];
  for (int i = 0; i < 3; ++i) a.q -= gE[i] * T.D1(i);
  for (int j = 0; j < 3; ++j) {
    const double E = -q * T.D1(j);
    double hg = 0.0;
    for (int i = 0; i < 3; ++i) hg += q * T.D2(i, j) * gE[i];
    a.c[j] += gphi * E + hg;
  }
}

// Adjoint of one interaction for force_law 2 (2D Coulomb) and 4 (Lennard-
// Jones), where no closed form is written out.  The 2D fields are linear in
// the node's charge and moments, so dL/dq and dL/dm are L of the unit moments;
// the Lennard-Jones fields depend on neither.  The offset derivative is the
// complex step, dL/dd_j = Im L(d + i h e_j) / h with h = 1e-40, exact to
// rounding for these analytic expressions (law_leaf / law_twig's arguments,
// evaluated by the same kernels on complex offsets).
void law_adjoint(int law, bool leaf, const double* m, const double d[3], double eps2, double gphi,
                 const double gE[3], Adj& a) {
  using Cx = std::complex<double>;
  auto Lreal = [&](const double* t) {
    double e[3], ph;
    const double dist2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
    if (leaf) law_leaf(law, t, d, dist2, eps2, e, ph);
    else law_twig(law, t, d, dist2, eps2, e, ph);
    return gphi * ph + ((gE[0] * e[0] + gE[1] * e[1]) + gE[2] * e[2]);
  };
  if (law == 2) {
    double t[M_N];
    for (int k = 0; k < M_N; ++k) t[k] = 0.0;
    t[M_Q] = 1.0;
    a.q += Lreal(t);
    if (!leaf) {
      t[M_Q] = 0.0;
      for (int k = 0; k < 3; ++k) {
        t[M_DX + k] = 1.0;
        a.p[k] += Lreal(t);
        t[M_DX + k] = 0.0;
      }
      const int qs[6] = {M_QXX, M_QYY, M_QZZ, M_XY, M_YZ, M_ZX};
      for (int k = 0; k < 6; ++k) {
        t[qs[k]] = 1.0;
        a.Q[k] += Lreal(t);
        t[qs[k]] = 0.0;
      }
    }
  }
  const double h = 1e-40;
  for (int j = 0; j < 3; ++j) {
    Cx dc[3] = {Cx(d[0], 0.0), Cx(d[1], 0.0), Cx(d[2], 0.0)};
    dc[j] = Cx(d[j], h);
    Cx e[3], ph;
    if (law == 2) {
      const Cx d2 = (dc[0] * dc[0] + dc[1] * dc[1]) + eps2;
      if (leaf) force_leaf_2d(m, dc, d2, e, ph);
      else force_twig_2d(m, dc, d2, e, ph);
    } else {
      force_lj(dc, (dc[0] * dc[0] + dc[1] * dc[1]) + dc[2] * dc[2], eps2, e, ph);
    }
    const Cx L = gphi * ph + ((gE[0] * e[0] + gE[1] * e[1]) + gE[2] * e[2]);
    a.c[j] -= L.imag() / h;  // d = target - node centre
  }
}

// the interaction adjoint of the context's force law (3: closed forms above)
void any_leaf_adjoint(int law, const double* m, const double d[3], double eps2, double gphi,
                      const double gE[3], Adj& a) {
  if (law == 3) leaf_adjoint(m[M_Q], d, eps2, gphi, gE, a);
  else law_adjoint(law, true, m, d, eps2, gphi, gE, a);
}
void any_twig_adjoint(int law, const double* m, const double d[3], double eps2, double gphi,
                      const double gE[3], Adj& a) {
  if (law == 3) twig_adjoint(m, d, eps2, gphi, gE, a);
  else law_adjoint(law, false, m, d, eps2, gphi, gE, a);
}

inline double sgn(double v) { return (double)((v > 0.0) - (v < 0.0)); }

// transpose of shift_multipoles_up (coulomb/module_interaction_specific.f90:84-140)
// for one parent: adds to the children's adjoints (children in key order)
void shift_up_adjoint(const double* par, const double* const* ch, int nc, const Adj& pa, Adj* ca) {
  const double A = par[M_ABSQ];
  double s[8][3];
  for (int c = 0; c < nc; ++c)
    for (int d = 0; d < 3; ++d) s[c][d] = par[M_COCX + d] - ch[c][M_COCX + d];
  double cocbar[3] = {pa.c[0], pa.c[1], pa.c[2]};
  for (int c = 0; c < nc; ++c) {
    const double* m = ch[c];
    const double qc = m[M_Q];
    const double pc[3] = {m[M_DX], m[M_DY], m[M_DZ]};
    const double* sc = s[c];
    double sbar[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i) sbar[i] += pa.p[i] * qc;                        // dip
    for (int i = 0; i < 3; ++i) sbar[i] += pa.Q[i] * (pc[i] + qc * sc[i]);      // quad diag
    sbar[0] += pa.Q[3] * (pc[1] + qc * sc[1]); sbar[1] += pa.Q[3] * (pc[0] + qc * sc[0]);  // xy
    sbar[1] += pa.Q[4] * (pc[2] + qc * sc[2]); sbar[2] += pa.Q[4] * (pc[1] + qc * sc[1]);  // yz
    sbar[2] += pa.Q[5] * (pc[0] + qc * sc[0]); sbar[0] += pa.Q[5] * (pc[2] + qc * sc[2]);  // zx
    Adj& a = ca[c];
    a.q += pa.q;
    for (int i = 0; i < 3; ++i) a.q += pa.p[i] * sc[i] + pa.Q[i] * 0.5 * sc[i] * sc[i];
    a.q += pa.Q[3] * sc[0] * sc[1] + pa.Q[4] * sc[1] * sc[2] + pa.Q[5] * sc[2] * sc[0];
    for (int i = 0; i < 3; ++i) a.p[i] += pa.p[i] + pa.Q[i] * sc[i];
    a.p[0] += pa.Q[3] * sc[1] + pa.Q[5] * sc[2];
    a.p[1] += pa.Q[3] * sc[0] + pa.Q[4] * sc[2];
    a.p[2] += pa.Q[4] * sc[1] + pa.Q[5] * sc[0];
    for (int k = 0; k < 6; ++k) a.Q[k] += pa.Q[k];
    for (int i = 0; i < 3; ++i) {
      a.c[i] -= sbar[i];  // s_c = coc - coc_c
      cocbar[i] += sbar[i];
    }
    a.A += pa.A;  // abs_charge = sum of the children's abs_charge
  }
  for (int c = 0; c < nc; ++c) {
    Adj& a = ca[c];
    if (A != 0.0) {
      const double w = ch[c][M_ABSQ] / A;
      double g = 0.0;
      for (int i = 0; i < 3; ++i) {
        a.c[i] += cocbar[i] * w;
        g += cocbar[i] * (ch[c][M_COCX + i] - par[M_COCX + i]);
      }
      a.A += g / A;
    } else {
      for (int i = 0; i < 3; ++i) a.c[i] += cocbar[i] / (double)nc;
    }
  }
}

}  // namespace

extern "C" {

void orc_params_default(orc_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->theta2 = 0.36;   // coulomb/module_interaction_specific.f90:38
  p->eps2 = 0.0;      // :39
  p->curve = 0;
  p->walk = 0;
  p->tile_size = 16;  // module_tree_walk_simple.f90:40
  p->mirror_box_layers = 1;             // module_mirror_boxes.f90:38
  p->include_far_field_if_periodic = 1; // coulomb/...specific.f90:37
  p->fmm_extrinsic_correction = 2;      // module_fmm_framework.f90:49
  p->t_lattice_1[0] = 1.0;
  p->t_lattice_2[1] = 1.0;
  p->t_lattice_3[2] = 1.0;
  p->num_threads = 1;
  p->force_law = 3;   // coulomb/module_interaction_specific.f90:35
  for (int k = 0; k < 3; ++k)  // huge(0._kind_physics), module_mirror_boxes.f90:52
    p->spatial_interaction_cutoff[k] = std::numeric_limits<double>::max();
}

void orc_box_create(int64_t n, const double* x, const double* y, const double* z,
                    int32_t force_cubic, double box9[9]) {
  Box b = box_create(n, x, y, z, force_cubic != 0);
  for (int d = 0; d < 3; ++d) {
    box9[d] = b.min[d];
    box9[3 + d] = b.max[d];
    box9[6 + d] = b.size[d];
  }
}

void orc_compute_keys(int64_t n, const double* x, const double* y, const double* z,
                      const double boxmin[3], const double boxsize[3], int32_t curve,
                      int64_t* keys) {
  Box b{};
  for (int d = 0; d < 3; ++d) { b.min[d] = boxmin[d]; b.size[d] = boxsize[d]; }
  double s[3];
  for (int d = 0; d < 3; ++d) s[d] = b.size[d] / (double)(int64_t(1) << kMaxLevel);
  for (int64_t i = 0; i < n; ++i) {
    int64_t ic[3];
    coord_to_intcoord(b, s, x[i], y[i], z[i], ic);
    keys[i] = curve == 1 ? intcoord_to_key_morton3d(ic) : intcoord_to_key_hilbert3d(ic);
  }
}

void orc_key_to_coord(int64_t key, const double boxmin[3], const double boxsize[3],
                      int32_t curve, double xout[3]) {
  Box b{};
  for (int d = 0; d < 3; ++d) { b.min[d] = boxmin[d]; b.size[d] = boxsize[d]; }
  key_to_coord(b, key, curve, xout);
}

void orc_sort_radix(int64_t n, int64_t* keys, int64_t* idx) {
  if (n < 2) return;
  rs_rec_ip(keys, idx, n, 63, 0, 10);
}

void orc_multipole_from_particle(const double pos[3], double q, double mp[15]) {
  multipole_from_particle(pos, q, mp);
}

void orc_shift_multipoles_up(double parent[15], const double* children, int32_t nchild) {
  const double* cm[8];
  for (int i = 0; i < nchild && i < 8; ++i) cm[i] = children + 15 * i;
  shift_multipoles_up(parent, cm, std::min(nchild, 8));
}

void orc_force_leaf(const double node[15], const double delta[3], double dist2, double e[3],
                    double* phi) {
  force_leaf(node, delta, dist2, e, *phi);
}

void orc_force_twig(const double node[15], const double delta[3], double dist2, double e[3],
                    double* phi) {
  force_twig(node, delta, dist2, e, *phi);
}

// par_rand, frontends/pepc-mini/module_helper.f90:592-658 (L'Ecuyer with
// Bays-Durham shuffle, single precision result).  State persists across calls
// exactly like the Fortran SAVE variables.
void orc_par_rand(int32_t iseed, int64_t n, double* out) {
  const int32_t IM1 = 2147483563, IM2 = 2147483399, IMM1 = IM1 - 1;
  const int32_t IA1 = 40014, IA2 = 40692, IQ1 = 53668, IQ2 = 52774, IR1 = 12211, IR2 = 3791;
  const int NTAB = 32;
  const int32_t NDIV = 1 + IMM1 / NTAB;
  const float AM = 1.0f / (float)IM1;
  const float RNMX = 1.0f - 1.2e-7f;
  static int32_t idum = -1, idum2 = 123456789, iy = 0, iv[32];
  bool seeded = iseed >= 0;
  for (int64_t c = 0; c < n; ++c) {
    if (idum <= 0 || (seeded && c == 0)) {
      if (seeded && c == 0) idum = iseed;
      else idum = (-idum < 1) ? 1 : -idum;
      idum2 = idum;
      for (int j = NTAB + 7; j >= 0; --j) {
        int32_t k = idum / IQ1;
        idum = IA1 * (idum - k * IQ1) - k * IR1;
        if (idum < 0) idum += IM1;
        if (j < NTAB) iv[j] = idum;
      }
      iy = iv[0];
    }
    int32_t k = idum / IQ1;
    idum = IA1 * (idum - k * IQ1) - k * IR1;
    if (idum < 0) idum += IM1;
    k = idum2 / IQ2;
    idum2 = IA2 * (idum2 - k * IQ2) - k * IR2;
    if (idum2 < 0) idum2 += IM2;
    int j = iy / NDIV;
    iy = iv[j] - idum2;
    iv[j] = idum;
    if (iy < 1) iy += IMM1;
    float r = AM * (float)iy;
    if (r > RNMX) r = RNMX;
    out[c] = (double)r;
  }
}

orc_ctx* orc_create(const orc_params* p) {
  orc_ctx* c = new orc_ctx;
  c->p = *p;
  if (c->periodic_far()) c->fmm = orc_fmm_create(c->p);
  return c;
}

void orc_destroy(orc_ctx* c) {
  if (!c) return;
  if (c->fmm) orc_fmm_destroy(c->fmm);
  delete c;
}

int orc_grow_tree(orc_ctx* c, int64_t n, const double* x, const double* y, const double* z,
                  const double* q, int64_t* key_out, int64_t* perm_out, double* x_out,
                  double* y_out, double* z_out, double* q_out) {
  if (n < 2) return -1;  // module_domains.f90:187-189: a rank needs >= 2 particles
  c->n = n;
  // tree_grow, module_tree_grow.f90:69-72
  c->box = box_create(n, x, y, z, c->p.force_cubic_domain != 0);
  std::vector<int64_t> keys(n), idx(n);
  orc_compute_keys(n, x, y, z, c->box.min, c->box.size, c->p.curve, keys.data());
  for (int64_t i = 0; i < n; ++i) idx[i] = i;
  // domain_decompose at one rank, module_domains.f90:158-319: sort, permute
  rs_rec_ip(keys.data(), idx.data(), n, 63, 0, 10);
  c->keys = keys;
  c->perm = idx;
  c->x.resize(n); c->y.resize(n); c->z.resize(n); c->q.resize(n);
  for (int64_t i = 0; i < n; ++i) {
    c->x[i] = x[idx[i]]; c->y[i] = y[idx[i]]; c->z[i] = z[idx[i]]; c->q[i] = q[idx[i]];
  }
  // duplicate-key fix, module_domains.f90:268-307
  std::vector<int64_t> lk = c->keys;
  std::vector<int64_t> kd(n);
  for (int64_t i = 0; i + 1 < n; ++i) kd[i] = lk[i + 1] - lk[i];
  kd[n - 1] = 1;
  for (int64_t i = 0; i < n; ++i) {
    if (kd[i] < 1) {
      for (int64_t j = 1; j <= std::max(n - 1 - i, i + 1); ++j) {
        // Fortran 1-based: key_diffs(max(1, i-j)) with i 1-based -> 0-based max(0, i-j)
        if (kd[std::max<int64_t>(0, i - j)] > 1) {
          for (int64_t t = i - j + 1; t <= i; ++t) lk[t] -= 1;
          kd[i] += 1;
          kd[i - j] -= 1;
          break;
        } else if (kd[std::min<int64_t>(n - 2, i + j)] > 1) {
          for (int64_t t = i + 1; t <= i + j; ++t) lk[t] += 1;
          kd[i] += 1;
          kd[i + j] -= 1;
          break;
        }
      }
    }
  }
  for (int64_t i = 0; i < n; ++i) {
    if (lk[i] != c->keys[i]) {
      c->keys[i] = lk[i];
      double xx[3];
      key_to_coord(c->box, lk[i], c->p.curve, xx);
      c->x[i] = xx[0]; c->y[i] = xx[1]; c->z[i] = xx[2];
    }
  }
  // tree_create, module_tree.f90:196-201
  c->boxlength2[0] = std::max(c->box.size[0], std::max(c->box.size[1], c->box.size[2]));
  c->boxlength2[0] = c->boxlength2[0] * c->boxlength2[0];
  for (int i = 1; i <= kMaxLevel; ++i) c->boxlength2[i] = c->boxlength2[i - 1] / 4.0;
  // tree_build_from_particles, module_tree_grow.f90:552-697
  c->nodes.clear();
  c->nodes.reserve(2 * n + 8);
  int64_t cur = 0;
  int err = 0;
  c->root = insert_helper(c, 1, 0, cur, err);
  if (err) return err;
  // tree_build_upwards at one rank recomputes the root from its children
  // (module_tree_grow.f90:410-536 with the level-1 branch nodes); identical
  // inputs in identical order, so the root is unchanged.
  if (c->nodes[c->root].leaves != n) return -4;
  if (key_out) std::memcpy(key_out, c->keys.data(), n * sizeof(int64_t));
  if (perm_out) std::memcpy(perm_out, c->perm.data(), n * sizeof(int64_t));
  if (x_out) std::memcpy(x_out, c->x.data(), n * sizeof(double));
  if (y_out) std::memcpy(y_out, c->y.data(), n * sizeof(double));
  if (z_out) std::memcpy(z_out, c->z.data(), n * sizeof(double));
  if (q_out) std::memcpy(q_out, c->q.data(), n * sizeof(double));
  if (c->fmm) orc_fmm_timestep(c->fmm, n, c->x.data(), c->y.data(), c->z.data(), c->q.data());
  return 0;
}

int orc_traverse_tree(orc_ctx* c, int64_t nt, const double* tx, const double* ty,
                      const double* tz, const int64_t* tkeys, double* ex, double* ey,
                      double* ez, double* pot, double* work) {
  auto boxes = neighbour_boxes(c->p);
  int nth = std::max(1, c->p.num_threads);
  std::vector<Counters> cnt(nth);
  std::atomic<int> bad{0};
  // the Kelbg law needs each target's charge: the targets must be the grown
  // particles in key order
  const double* tq = nullptr;
  if (c->p.force_law == 5) {
    if (nt != c->n) return -6;
    tq = c->q.data();
  }
  // libpepc_traverse_tree, module_libpepc_main.f90:161-200: one walk per box,
  // central box last, then the per-particle lattice term.
  if (c->p.walk == 0) {
    parallel_for(nt, nth, [&](int64_t i, int t) {
      std::vector<int64_t> todo;
      todo.reserve(1024);
      double xt[3] = {tx[i], ty[i], tz[i]};
      double e[3] = {ex[i], ey[i], ez[i]}, ph = pot[i], w = work[i];
      for (auto& bx : boxes) {
        double vb[3];
        lattice_vect(c->p, bx, vb);
        int64_t partner = walk_pthreads(c, xt, vb, e, ph, w, cnt[t], todo, tq ? tq[i] : 0.0);
        if (partner != c->n) bad.store(1);
      }
      ex[i] = e[0]; ey[i] = e[1]; ez[i] = e[2]; pot[i] = ph; work[i] = w;
    });
  } else {
    std::vector<std::pair<int64_t, int64_t>> tiles;
    int err = 0;
    if (c->p.walk == 2) {
      // the GPU library's group walk: buckets of tile_size (<= 64)
      // key-consecutive targets with the simple walk's rule
      const int64_t g = std::min(64, std::max(1, c->p.tile_size));
      for (int64_t i = 0; i < nt; i += g) tiles.push_back({i, std::min(nt, i + g)});
    } else if (tkeys == nullptr) {
      for (int64_t i = 0; i < nt; ++i) tiles.push_back({i, i + 1});
    } else {
      make_tiles(tkeys, 0, nt, 1, 0, std::min(32, std::max(1, c->p.tile_size)), tiles, err);
      if (err) return err;
    }
    parallel_for((int64_t)tiles.size(), nth, [&](int64_t it, int t) {
      int64_t lo = tiles[it].first, np = tiles[it].second - tiles[it].first;
      double xs[64][3], e[64][3], ph[64], w[64], qs[64];
      for (int k = 0; k < np; ++k) {
        qs[k] = tq ? tq[lo + k] : 0.0;
        xs[k][0] = tx[lo + k]; xs[k][1] = ty[lo + k]; xs[k][2] = tz[lo + k];
        e[k][0] = ex[lo + k]; e[k][1] = ey[lo + k]; e[k][2] = ez[lo + k];
        ph[k] = pot[lo + k]; w[k] = work[lo + k];
      }
      for (auto& bx : boxes) {
        double vb[3];
        lattice_vect(c->p, bx, vb);
        int64_t partner = 0;
        walk_simple_aux(c, c->root, (int)np, xs, vb, e, ph, w, partner, cnt[t], qs);
        if (partner != c->n) bad.store(1);
      }
      for (int k = 0; k < np; ++k) {
        ex[lo + k] = e[k][0]; ey[lo + k] = e[k][1]; ez[lo + k] = e[k][2];
        pot[lo + k] = ph[k]; work[lo + k] = w[k];
      }
    });
  }
  c->n_interactions = 0;
  c->n_mac = 0;
  for (auto& k : cnt) { c->n_interactions += k.inter; c->n_mac += k.mac; }
  if (c->fmm) {  // calc_force_per_particle, coulomb/...specific.f90:393-427
    parallel_for(nt, nth, [&](int64_t i, int) {
      double pos[3] = {tx[i], ty[i], tz[i]}, e[3], ph;
      orc_fmm_sum_lattice_force(c->fmm, pos, e, &ph);
      ex[i] += e[0]; ey[i] += e[1]; ez[i] += e[2]; pot[i] += ph;
    });
  }
  return bad.load() ? -3 : 0;
}

int64_t orc_num_nodes(const orc_ctx* c) { return (int64_t)c->nodes.size(); }

void orc_tree_export(const orc_ctx* c, int64_t* key, int32_t* level, int64_t* leaves,
                     int64_t* descendants, int64_t* parent, int64_t* first_child,
                     int64_t* next_sibling, double* moments15) {
  for (size_t i = 0; i < c->nodes.size(); ++i) {
    const Node& nd = c->nodes[i];
    if (key) key[i] = nd.key;
    if (level) level[i] = nd.level;
    if (leaves) leaves[i] = nd.leaves;
    if (descendants) descendants[i] = nd.descendants;
    if (parent) parent[i] = nd.parent;
    if (first_child) first_child[i] = nd.first_child;
    if (next_sibling) next_sibling[i] = nd.next_sibling;
    if (moments15) std::memcpy(moments15 + 15 * i, nd.m, 15 * sizeof(double));
  }
}

void orc_box(const orc_ctx* c, double box9[9]) {
  for (int d = 0; d < 3; ++d) {
    box9[d] = c->box.min[d];
    box9[3 + d] = c->box.max[d];
    box9[6 + d] = c->box.size[d];
  }
}

void orc_counters(const orc_ctx* c, int64_t out[2]) {
  out[0] = c->n_interactions;
  out[1] = c->n_mac;
}

int orc_direct(orc_ctx* c, int64_t ntest, const int64_t* tidx, double* ex, double* ey,
               double* ez, double* pot) {
  auto boxes = neighbour_boxes(c->p);
  const int64_t n = c->n;
  int nth = std::max(1, c->p.num_threads);
  // directforce, utils/module_directsum.f90:86-159 (one rank: currank = 0)
  parallel_for(ntest, nth, [&](int64_t j, int) {
    int64_t tj = tidx[j];
    double xt[3] = {c->x[tj], c->y[tj], c->z[tj]};
    double e[3] = {0, 0, 0}, ph = 0;
    for (int64_t i = 0; i < n; ++i) {
      double m[M_N];
      double pos[3] = {c->x[i], c->y[i], c->z[i]};
      multipole_from_particle(pos, c->q[i], m);
      for (size_t ib = 0; ib < boxes.size(); ++ib) {
        double vb[3];
        lattice_vect(c->p, boxes[ib], vb);
        double d[3] = {(xt[0] - vb[0]) - m[M_COCX], (xt[1] - vb[1]) - m[M_COCY],
                       (xt[2] - vb[2]) - m[M_COCZ]};
        if (ib + 1 == boxes.size() && tj == i) continue;  // self, :119-124
        double dist2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
        double ee[3], pp;
        law_leaf(c->p.force_law, m, d, dist2, c->p.eps2, ee, pp, c->q[tj], c->p.kelbg_invsqrttemp);
        e[0] += ee[0]; e[1] += ee[1]; e[2] += ee[2];
        ph += pp;
      }
    }
    if (c->fmm) {  // :163-171
      double le[3], lp;
      orc_fmm_sum_lattice_force(c->fmm, xt, le, &lp);
      e[0] += le[0]; e[1] += le[1]; e[2] += le[2]; ph += lp;
    }
    ex[j] = e[0]; ey[j] = e[1]; ez[j] = e[2]; pot[j] = ph;
  });
  return 0;
}

// Install lattice coefficients (861 complex, interleaved re/im), e.g. the
// reference's pretabulated unit-cube table (load_lattice_coefficients,
// module_fmm_framework.f90:260-508).  Must be called before grow.
int orc_set_lattice_coefficients(orc_ctx* c, const double* re_im) {
  if (!c->fmm) return -1;
  orc_fmm_set_mlattice(c->fmm, re_im);
  return 0;
}

int orc_lattice(orc_ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                double* ex, double* ey, double* ez, double* pot) {
  if (!c->fmm) return -1;
  for (int64_t i = 0; i < nt; ++i) {
    double pos[3] = {tx[i], ty[i], tz[i]}, e[3], ph;
    orc_fmm_sum_lattice_force(c->fmm, pos, e, &ph);
    ex[i] = e[0]; ey[i] = e[1]; ez[i] = e[2]; pot[i] = ph;
  }
  return 0;
}


// Adjoint of the per-target walk (module_tree_walk_pthreads.f90 semantics), or
// with walk 2 of the bucket walk (the group walk's lists): dL/dq and dL/dx of
// the grown particles, in the caller's original order.  With a periodic far
// field the lattice term's adjoint (orc_fmm_adjoint) is added.
int orc_traverse_adjoint(orc_ctx* c, int64_t nt, const double* tx, const double* ty,
                         const double* tz, const double* gex, const double* gey,
                         const double* gez, const double* gphi, double* dLdq, double* dLdx,
                         double* dLdy, double* dLdz) {
  if (c->p.force_law == 5) return -7;  // Kelbg: needs each target's own charge
  auto boxes = neighbour_boxes(c->p);
  const int64_t M = (int64_t)c->nodes.size();
  std::vector<Adj> adj(M);
  std::vector<int64_t> todo;
  if (c->p.walk == 2) {
    // buckets of tile_size consecutive targets, the simple walk's rule
    // (module_tree_walk_simple.f90:343-382): a twig is accepted only if
    // every target of the bucket passes the MAC, else its children are
    // visited; leaves interact with every target but itself
    const int64_t ts = std::max(1, std::min(64, c->p.tile_size));
    for (int64_t b0 = 0; b0 < nt; b0 += ts) {
      const int64_t np = std::min(ts, nt - b0);
      for (auto& bx : boxes) {
        double vb[3];
        lattice_vect(c->p, bx, vb);
        todo.clear();
        todo.push_back(c->root);
        while (!todo.empty()) {
          const int64_t ni = todo.back();
          todo.pop_back();
          const Node& nd = c->nodes[ni];
          bool all = true;
          for (int64_t i = b0; i < b0 + np && nd.descendants != 0; ++i) {
            const double d[3] = {(tx[i] - vb[0]) - nd.m[M_COCX], (ty[i] - vb[1]) - nd.m[M_COCY],
                                 (tz[i] - vb[2]) - nd.m[M_COCZ]};
            const double dist2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
            if (!mac_pass(c, nd, dist2)) { all = false; break; }
          }
          if (!all) {
            // children last to first onto the stack, so they are visited first to last
            std::vector<int64_t> ch;
            for (int64_t k = nd.first_child; k != kNodeInvalid; k = c->nodes[k].next_sibling)
              ch.push_back(k);
            for (auto it = ch.rbegin(); it != ch.rend(); ++it) todo.push_back(*it);
            continue;
          }
          for (int64_t i = b0; i < b0 + np; ++i) {
            const double gE[3] = {gex[i], gey[i], gez[i]};
            const double d[3] = {(tx[i] - vb[0]) - nd.m[M_COCX], (ty[i] - vb[1]) - nd.m[M_COCY],
                                 (tz[i] - vb[2]) - nd.m[M_COCZ]};
            const double dist2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
            if (cut_off(c, d)) continue;  // the forward's skip (:330, :377)
            if (nd.descendants == 0) {
              if (dist2 > 0.0) any_leaf_adjoint(c->p.force_law, nd.m, d, c->p.eps2, gphi[i], gE, adj[ni]);
            } else {
              any_twig_adjoint(c->p.force_law, nd.m, d, c->p.eps2, gphi[i], gE, adj[ni]);
            }
          }
        }
      }
    }
  }
  for (int64_t i = 0; i < nt && c->p.walk != 2; ++i) {
    const double gE[3] = {gex[i], gey[i], gez[i]};
    for (auto& bx : boxes) {
      double vb[3];
      lattice_vect(c->p, bx, vb);
      const double sh[3] = {tx[i] - vb[0], ty[i] - vb[1], tz[i] - vb[2]};
      todo.clear();
      for (int64_t ch = c->nodes[c->root].first_child; ch != kNodeInvalid; ch = c->nodes[ch].next_sibling)
        todo.push_back(ch);
      while (!todo.empty()) {
        int64_t ni = todo.back();
        todo.pop_back();
        const Node& nd = c->nodes[ni];
        const double d[3] = {sh[0] - nd.m[M_COCX], sh[1] - nd.m[M_COCY], sh[2] - nd.m[M_COCZ]};
        const double dist2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
        if (nd.descendants == 0) {
          if (dist2 > 0.0 && !cut_off(c, d))  // :622
            any_leaf_adjoint(c->p.force_law, nd.m, d, c->p.eps2, gphi[i], gE, adj[ni]);
        } else if (mac_pass(c, nd, dist2)) {
          if (!cut_off(c, d))  // :639
            any_twig_adjoint(c->p.force_law, nd.m, d, c->p.eps2, gphi[i], gE, adj[ni]);
        } else {
          for (int64_t ch = nd.first_child; ch != kNodeInvalid; ch = c->nodes[ch].next_sibling)
            todo.push_back(ch);
        }
      }
    }
  }
  // preorder (insertion order) visits every parent before its children
  for (int64_t ni = 0; ni < M; ++ni) {
    const Node& nd = c->nodes[ni];
    if (nd.descendants == 0) continue;
    const double* chm[8];
    int64_t chi[8];
    int nc = 0;
    for (int64_t ch = nd.first_child; ch != kNodeInvalid; ch = c->nodes[ch].next_sibling) {
      chm[nc] = c->nodes[ch].m;
      chi[nc] = ch;
      ++nc;
    }
    Adj ca[8];
    shift_up_adjoint(nd.m, chm, nc, adj[ni], ca);
    for (int k = 0; k < nc; ++k) {
      Adj& a = adj[chi[k]];
      a.q += ca[k].q;
      for (int j = 0; j < 3; ++j) { a.p[j] += ca[k].p[j]; a.c[j] += ca[k].c[j]; }
      for (int j = 0; j < 6; ++j) a.Q[j] += ca[k].Q[j];
      a.A += ca[k].A;
    }
  }
  for (int64_t ni = 0; ni < M; ++ni) {
    const Node& nd = c->nodes[ni];
    if (nd.descendants != 0) continue;
    const int64_t ip = nd.particle;
    const int64_t io = c->perm[ip];
    const Adj& a = adj[ni];
    dLdq[io] = a.q + a.A * sgn(c->q[ip]);
    dLdx[io] = a.c[0];
    dLdy[io] = a.c[1];
    dLdz[io] = a.c[2];
  }
  if (c->fmm) {
    const int64_t n = c->n;
    std::vector<double> fq(n), fx(n), fy(n), fz(n);
    orc_fmm_adjoint(c->fmm, nt, tx, ty, tz, gex, gey, gez, gphi, n, c->x.data(), c->y.data(),
                    c->z.data(), c->q.data(), fq.data(), fx.data(), fy.data(), fz.data());
    for (int64_t ip = 0; ip < n; ++ip) {
      const int64_t io = c->perm[ip];
      dLdq[io] += fq[ip];
      dLdx[io] += fx[ip];
      dLdy[io] += fy[ip];
      dLdz[io] += fz[ip];
    }
  }
  return 0;
}

// FP64 direct-sum gradient of sum_t (gphi phi_t + gE . E_t) over the grown
// particles (no tree), in the caller's original order.
int orc_direct_adjoint(orc_ctx* c, int64_t nt, const double* tx, const double* ty,
                       const double* tz, const double* gex, const double* gey, const double* gez,
                       const double* gphi, double* dLdq, double* dLdx, double* dLdy, double* dLdz) {
  if (c->p.force_law == 5) return -7;  // Kelbg: needs each target's own charge
  auto boxes = neighbour_boxes(c->p);
  const int64_t n = c->n;
  int nth = std::max(1, c->p.num_threads);
  parallel_for(n, nth, [&](int64_t j, int) {
    Adj a;
    for (int64_t i = 0; i < nt; ++i) {
      const double gE[3] = {gex[i], gey[i], gez[i]};
      for (auto& bx : boxes) {
        double vb[3];
        lattice_vect(c->p, bx, vb);
        const double d[3] = {(tx[i] - vb[0]) - c->x[j], (ty[i] - vb[1]) - c->y[j],
                             (tz[i] - vb[2]) - c->z[j]};
        if (d[0] == 0.0 && d[1] == 0.0 && d[2] == 0.0) continue;
        double t[M_N] = {};
        t[M_Q] = c->q[j];
        any_leaf_adjoint(c->p.force_law, t, d, c->p.eps2, gphi[i], gE, a);
      }
    }
    const int64_t io = c->perm[j];
    dLdq[io] = a.q;
    dLdx[io] = a.c[0];
    dLdy[io] = a.c[1];
    dLdz[io] = a.c[2];
  });
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The frontend's time step around the path.  Test infrastructure: restates
// pepc-mini's push_particles / apply_external_field (module_helper.f90:205-222,
// :321-334) and constrain_periodic (module_mirror_boxes.f90:177-218) with
// inverse3 / det3 / det2f (module_math_tools.f90:55-150).
// ---------------------------------------------------------------------------
namespace {
// Fortran MODULO for reals, as fmod with the sign moved to the divisor's
double fortran_modulo(double a, double p) {
  double r = std::fmod(a, p);
  if (r != 0.0 && ((r < 0.0) != (p < 0.0))) r = r + p;
  return r;
}

void lattice_inverse(const orc_params* p, double L[3][3], double Li[3][3]) {
  for (int j = 0; j < 3; ++j) {
    L[0][j] = p->t_lattice_1[j];
    L[1][j] = p->t_lattice_2[j];
    L[2][j] = p->t_lattice_3[j];
  }
  // m(i, j) = L[i-1][j-1]
  auto m = [&](int i, int j) { return L[i - 1][j - 1]; };
  const double det = m(1, 1) * m(2, 2) * m(3, 3) + m(1, 2) * m(2, 3) * m(3, 1) +
                     m(1, 3) * m(2, 1) * m(3, 2) - m(1, 3) * m(2, 2) * m(3, 1) -
                     m(1, 2) * m(2, 1) * m(3, 3) - m(1, 1) * m(2, 3) * m(3, 2);
  auto d2 = [](double a, double b, double c, double d) { return a * d - b * c; };
  // column-major reshape of the nine 2x2 determinants
  Li[0][0] = d2(m(2, 2), m(3, 2), m(2, 3), m(3, 3)) / det;
  Li[1][0] = d2(m(2, 3), m(3, 3), m(2, 1), m(3, 1)) / det;
  Li[2][0] = d2(m(2, 1), m(3, 1), m(2, 2), m(3, 2)) / det;
  Li[0][1] = d2(m(1, 3), m(3, 3), m(1, 2), m(3, 2)) / det;
  Li[1][1] = d2(m(1, 1), m(3, 1), m(1, 3), m(3, 3)) / det;
  Li[2][1] = d2(m(1, 2), m(3, 2), m(1, 1), m(3, 1)) / det;
  Li[0][2] = d2(m(1, 2), m(2, 2), m(1, 3), m(2, 3)) / det;
  Li[1][2] = d2(m(1, 3), m(2, 3), m(1, 1), m(2, 1)) / det;
  Li[2][2] = d2(m(1, 1), m(2, 1), m(1, 2), m(2, 2)) / det;
}
}  // namespace

extern "C" {

void orc_push_particles(int64_t n, double dt, const double* q, const double* m, const double* ex,
                        const double* ey, const double* ez, double* vx, double* vy, double* vz,
                        double* x, double* y, double* z) {
  const double fact = dt;
  for (int64_t i = 0; i < n; ++i) {
    const double f = fact * q[i] / m[i];
    vx[i] = vx[i] + f * ex[i];
    vy[i] = vy[i] + f * ey[i];
    vz[i] = vz[i] + f * ez[i];
    x[i] = x[i] + dt * vx[i];
    y[i] = y[i] + dt * vy[i];
    z[i] = z[i] + dt * vz[i];
  }
}

void orc_apply_external_field(int64_t n, double ez_ext, const double* z, double* ez, double* pot) {
  for (int64_t i = 0; i < n; ++i) {
    ez[i] = ez[i] + ez_ext;
    pot[i] = pot[i] - z[i] * ez_ext;
  }
}

void orc_constrain_periodic(const orc_params* p, int64_t n, double* x, double* y, double* z) {
  const double* o = p->lattice_origin;
  const bool simple = p->t_lattice_1[0] > 0.0 && p->t_lattice_1[1] == 0.0 &&
                      p->t_lattice_1[2] == 0.0 && p->t_lattice_2[0] == 0.0 &&
                      p->t_lattice_2[1] > 0.0 && p->t_lattice_2[2] == 0.0 &&
                      p->t_lattice_3[0] == 0.0 && p->t_lattice_3[1] == 0.0 &&
                      p->t_lattice_3[2] > 0.0;
  double L[3][3], Li[3][3];
  lattice_inverse(p, L, Li);
  double* c[3] = {x, y, z};
  for (int64_t i = 0; i < n; ++i) {
    if (simple) {
      const double walls[3] = {p->t_lattice_1[0], p->t_lattice_2[1], p->t_lattice_3[2]};
      for (int d = 0; d < 3; ++d)
        if (p->periodicity[d]) c[d][i] = fortran_modulo(c[d][i] - o[d], walls[d]) + o[d];
    } else {
      const double v[3] = {x[i] - o[0], y[i] - o[1], z[i] - o[2]};
      double lc[3];
      bool out = false;
      for (int j = 0; j < 3; ++j) {
        lc[j] = (v[0] * Li[0][j] + v[1] * Li[1][j]) + v[2] * Li[2][j];
        if (lc[j] > 1.0 || lc[j] < 0.0) out = true;
      }
      if (out) {
        for (int j = 0; j < 3; ++j) lc[j] = fortran_modulo(lc[j], 1.0);
        for (int j = 0; j < 3; ++j) {
          const double r = ((lc[0] * L[0][j] + lc[1] * L[1][j]) + lc[2] * L[2][j]) + o[j];
          if (p->periodicity[j]) c[j][i] = r;
        }
      }
    }
  }
}

}  // extern "C"

