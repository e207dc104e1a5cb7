// scalar.cu -- the Coulomb backend's scalar entry points, evaluated by the
// same device functions that the walk and the upward pass use (one tiny
// launch per call; meant for shims and unit tests, not for throughput).
// References: coulomb/module_interaction_specific.f90:67-79 (multipole_from_particle),
// :84-140 (shift_multipoles_up), :256-275 (mac), :314-387 (with_leaf / with_twig).
// Compiled with --fmad=false.

#include <cstring>

#include "internal.cuh"

namespace pepcg {
namespace {

__global__ void k_scalar(int op, const double* in, int nin, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (op == 0) {  // multipole_from_particle: in = pos(3), q
    out[0] = in[0]; out[1] = in[1]; out[2] = in[2];
    out[3] = in[3];
    out[4] = fabs(in[3]);
    for (int k = 5; k < 15; ++k) out[k] = 0.0;
  } else if (op == 1) {  // shift_multipoles_up: in = nchild x 15
    Moments ch[8];
    int nc = nin;
    for (int j = 0; j < nc; ++j) {
      const double* c = in + 15 * j;
      for (int d = 0; d < 3; ++d) ch[j].coc[d] = c[d];
      ch[j].q = c[3];
      ch[j].absq = c[4];
      for (int k = 0; k < 9; ++k) ch[j].m[k] = c[5 + k];
      ch[j].bmax = c[14];
    }
    Moments p;
    shift_up64(ch, nc, p);
    for (int d = 0; d < 3; ++d) out[d] = p.coc[d];
    out[3] = p.q;
    out[4] = p.absq;
    for (int k = 0; k < 9; ++k) out[5 + k] = p.m[k];
    out[14] = p.bmax;
  } else if (op == 2 || op == 3) {  // with_leaf / with_twig: in = node15, delta3, dist2, eps2
    const double* nd = in;
    double dx = in[15], dy = in[16], dz = in[17], d2 = in[18] + in[19];
    if (op == 2) force_leaf64(nd[3], dx, dy, dz, d2, out[0], out[1], out[2], out[3]);
    else force_twig64(nd[3], nd + 5, dx, dy, dz, d2, out[0], out[1], out[2], out[3]);
  } else if (op == 4) {  // mac: theta2 * dist2 > boxlength2
    out[0] = (in[0] * in[1] > in[2]) ? 1.0 : 0.0;
  }
}

int run_scalar(int op, const double* in, int nin_doubles, int nchild, double* out, int nout) {
  double* d = nullptr;
  if (cudaMalloc((void**)&d, (nin_doubles + nout) * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return PEPCG_ERR_CUDA;
  }
  cudaMemcpy(d, in, nin_doubles * sizeof(double), cudaMemcpyHostToDevice);
  COUNT_LAUNCH();
  k_scalar<<<1, 32>>>(op, d, nchild, d + nin_doubles);
  cudaError_t e = cudaMemcpy(out, d + nin_doubles, nout * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? PEPCG_OK : PEPCG_ERR_CUDA;
}

}  // namespace
}  // namespace pepcg

using namespace pepcg;

extern "C" {

int pepcg_multipole_from_particle(const double pos[3], double q, double mp[15]) {
  if (!pos || !mp) return PEPCG_ERR_BAD_ARG;
  double in[4] = {pos[0], pos[1], pos[2], q};
  return run_scalar(0, in, 4, 0, mp, 15);
}

int pepcg_shift_multipoles_up(double parent[15], const double* children, int32_t nchild) {
  if (!parent || !children || nchild < 1 || nchild > 8) return PEPCG_ERR_BAD_ARG;
  return run_scalar(1, children, 15 * nchild, nchild, parent, 15);
}

int pepcg_force_with_leaf(const double node[15], const double delta[3], double dist2, double eps2,
                          double e[3], double* phi) {
  if (!node || !delta || !e || !phi) return PEPCG_ERR_BAD_ARG;
  double in[20];
  std::memcpy(in, node, 15 * sizeof(double));
  in[15] = delta[0]; in[16] = delta[1]; in[17] = delta[2]; in[18] = dist2; in[19] = eps2;
  double out[4];
  int rc = run_scalar(2, in, 20, 0, out, 4);
  e[0] = out[0]; e[1] = out[1]; e[2] = out[2]; *phi = out[3];
  return rc;
}

int pepcg_force_with_twig(const double node[15], const double delta[3], double dist2, double eps2,
                          double e[3], double* phi) {
  if (!node || !delta || !e || !phi) return PEPCG_ERR_BAD_ARG;
  double in[20];
  std::memcpy(in, node, 15 * sizeof(double));
  in[15] = delta[0]; in[16] = delta[1]; in[17] = delta[2]; in[18] = dist2; in[19] = eps2;
  double out[4];
  int rc = run_scalar(3, in, 20, 0, out, 4);
  e[0] = out[0]; e[1] = out[1]; e[2] = out[2]; *phi = out[3];
  return rc;
}

int pepcg_mac(double theta2, double dist2, double boxlength2, int32_t* accept) {
  if (!accept) return PEPCG_ERR_BAD_ARG;
  double in[3] = {theta2, dist2, boxlength2}, out[1];
  int rc = run_scalar(4, in, 3, 0, out, 1);
  *accept = out[0] != 0.0;
  return rc;
}

}  // extern "C"
