// api.cu -- the C ABI of libpepcg (include/pepcg.h): context lifetime,
// device buffers, host <-> device staging and status reporting.
//
// Host-side orchestration only: every computation on particles and nodes is a
// device kernel (grow.cu, walk_*.cu, lattice.cu, direct.cu).  There is no CPU
// fallback: without a usable CUDA device every entry point fails with
// PEPCG_ERR_CUDA.

#include <cfloat>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "internal.cuh"

namespace pepcg {

static thread_local std::string g_static_err;
std::atomic<long long> g_launches{0};

void set_static_error(const std::string& msg) { g_static_err = msg; }

bool cuda_ok(Ctx* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  std::string msg = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  if (c) c->err = msg;
  else g_static_err = msg;
  return false;
}

// allocations left before the injected failures start (< 0: no injection)
static std::atomic<int64_t> g_fail_after{-1};

// true when the injection makes this allocation fail
static bool injected_failure() {
  int64_t left = g_fail_after.load();
  while (left > 0 && !g_fail_after.compare_exchange_weak(left, left - 1)) {
  }
  return left == 0;
}

template <class T>
bool ensure(Ctx* c, DBuf<T>& b, size_t n, const char* what) {
  if (n <= b.cap) return true;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t want = n + n / 8 + 64;
  if (injected_failure()) {
    c->err = std::string("device allocation failed for ") + what + " (" +
             std::to_string(want * sizeof(T)) + " bytes): injected by pepcg_debug_fail_allocations";
    return false;
  }
  cudaError_t e = cudaMalloc((void**)&b.p, want * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    c->err = std::string("device allocation failed for ") + what + " (" +
             std::to_string(want * sizeof(T)) + " bytes): " + cudaGetErrorString(e);
    b.p = nullptr;
    return false;
  }
  b.cap = want;
  return true;
}

template bool ensure<double>(Ctx*, DBuf<double>&, size_t, const char*);
template bool ensure<float>(Ctx*, DBuf<float>&, size_t, const char*);
template bool ensure<int64_t>(Ctx*, DBuf<int64_t>&, size_t, const char*);
template bool ensure<int32_t>(Ctx*, DBuf<int32_t>&, size_t, const char*);
template bool ensure<int8_t>(Ctx*, DBuf<int8_t>&, size_t, const char*);
template bool ensure<uint64_t>(Ctx*, DBuf<uint64_t>&, size_t, const char*);
template bool ensure<uint32_t>(Ctx*, DBuf<uint32_t>&, size_t, const char*);
template bool ensure<unsigned long long>(Ctx*, DBuf<unsigned long long>&, size_t, const char*);
template bool ensure<double4>(Ctx*, DBuf<double4>&, size_t, const char*);
template bool ensure<double2>(Ctx*, DBuf<double2>&, size_t, const char*);
template bool ensure<int2>(Ctx*, DBuf<int2>&, size_t, const char*);
template bool ensure<int4>(Ctx*, DBuf<int4>&, size_t, const char*);
template bool ensure<LevelRecord>(Ctx*, DBuf<LevelRecord>&, size_t, const char*);

template <class T>
static void release(DBuf<T>& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

int status_to_code(Ctx* c, uint32_t st) {
  if (st & ST_NONFINITE) {
    c->err = "non-finite particle coordinate";
    return PEPCG_ERR_BAD_ARG;
  }
  if (st & ST_MAXLEVEL) {
    c->err = "no more levels: keys could not be separated (module_tree_grow.f90:671-675)";
    return PEPCG_ERR_MAXLEVEL;
  }
  if (st & ST_DUP_OVERFLOW) {
    c->err = "too many duplicate keys for the duplicate-key fix";
    return PEPCG_ERR_MAXLEVEL;
  }
  if (st & ST_SORT_REPLAY) {
    c->err = "internal error: the replay of the reference's key order for equal keys "
             "found an inconsistent class list";
    return PEPCG_ERR_CUDA;
  }
  if (st & ST_TIMEOUT) {
    c->err = "a bounded device wait gave up";
    return PEPCG_ERR_TIMEOUT;
  }
  if (st & ST_INCOMPLETE) {
    c->err = "walk incomplete: a target did not interact with all leaves "
             "(module_tree_walk_pthreads.f90:452-457)";
    return PEPCG_ERR_INCOMPLETE_WALK;
  }
  if (st & ST_NOT_NEUTRAL) {
    c->err = "central box not charge-neutral: monopole removed (module_fmm_framework.f90:570-573)";
    return PEPCG_WARN_NOT_NEUTRAL;
  }
  return PEPCG_OK;
}

// neighbour_boxes_prepare (module_mirror_boxes.f90:99-156) and lattice_vect (:73-79)
static void prepare_boxes(Ctx* c) {
  const pepcg_params& p = c->prm;
  int sw[3];
  for (int d = 0; d < 3; ++d) sw[d] = p.periodicity[d] ? p.mirror_box_layers : 0;
  std::vector<int> nb;
  auto push = [&](int i, int j, int k) {
    nb.push_back(i);
    nb.push_back(j);
    nb.push_back(k);
  };
  for (int i = -sw[0]; i <= -1; ++i)
    for (int j = -sw[1]; j <= sw[1]; ++j)
      for (int k = -sw[2]; k <= sw[2]; ++k) {
        push(i, j, k);
        push(-i, -j, -k);
      }
  for (int j = -sw[1]; j <= -1; ++j)
    for (int k = -sw[2]; k <= sw[2]; ++k) {
      push(0, j, k);
      push(0, -j, -k);
    }
  for (int k = -sw[2]; k <= -1; ++k) {
    push(0, 0, k);
    push(0, 0, -k);
  }
  push(0, 0, 0);
  c->nboxes = (int)nb.size() / 3;
  for (int b = 0; b < c->nboxes; ++b)
    for (int d = 0; d < 3; ++d)
      c->vbox[3 * b + d] = ((double)nb[3 * b] * p.t_lattice_1[d] + (double)nb[3 * b + 1] * p.t_lattice_2[d]) +
                           (double)nb[3 * b + 2] * p.t_lattice_3[d];
  c->periodic = p.periodicity[0] || p.periodicity[1] || p.periodicity[2];
  c->far_field = c->periodic && p.include_far_field_if_periodic;
}

static int check_params(Ctx* c, const pepcg_params* p) {
  if (p->force_law < 2 || p->force_law > 5) {
    c->err = "force_law must be 3 (3D Coulomb), 2 (2D Coulomb), 4 (Lennard-Jones) or 5 (Kelbg)";
    return PEPCG_ERR_UNSUPPORTED;
  }
  if (p->force_law != 3 && p->precision != PEPCG_PRECISION_PLAIN) {
    c->err = "the mixed-precision walks evaluate the 3D Coulomb law only (force_law = 3)";
    return PEPCG_ERR_UNSUPPORTED;
  }
  if (p->mac_select < 0) {
    c->err = "mac_select must be 0 (Barnes-Hut), 1 (Bmax) or another positive value (no acceptance, N^2)";
    return PEPCG_ERR_BAD_ARG;
  }
  if (p->curve != PEPCG_CURVE_HILBERT && p->curve != PEPCG_CURVE_MORTON) {
    c->err = "curve must be PEPCG_CURVE_HILBERT or PEPCG_CURVE_MORTON";
    return PEPCG_ERR_BAD_ARG;
  }
  if (p->precision != PEPCG_PRECISION_PLAIN && p->precision != PEPCG_PRECISION_MIXED &&
      p->precision != PEPCG_PRECISION_MIXED_STRICT) {
    c->err = "precision must be PLAIN, MIXED or MIXED_STRICT";
    return PEPCG_ERR_BAD_ARG;
  }
  if (p->precision == PEPCG_PRECISION_MIXED_STRICT &&
      (p->walk != PEPCG_WALK_GROUP || (p->group_size != 0 && p->group_size != 64))) {
    c->err = "MIXED_STRICT is built for the GROUP walk with 64-target buckets";
    return PEPCG_ERR_UNSUPPORTED;
  }
  if (p->walk < 0 || p->walk > 2) {
    c->err = "walk must be PER_TARGET, PER_TILE or GROUP";
    return PEPCG_ERR_BAD_ARG;
  }
  if (p->tile_size < 1 || p->tile_size > 32) {
    c->err = "tile_size must be in 1..32";
    return PEPCG_ERR_BAD_ARG;
  }
  if (!(p->theta2 >= 0.0) || !(p->eps2 >= 0.0)) {
    c->err = "theta2 and eps2 must be >= 0";
    return PEPCG_ERR_BAD_ARG;
  }
  if (p->group_size != 0 && p->group_size != 32 && p->group_size != 64) {
    c->err = "group_size must be 0 (automatic), 32 or 64";
    return PEPCG_ERR_BAD_ARG;
  }
  if (p->mirror_box_layers < 0 || p->mirror_box_layers > 2) {
    c->err = "mirror_box_layers must be in 0..2";
    return PEPCG_ERR_BAD_ARG;
  }
  for (int k = 0; k < 3; ++k)
    if (!(p->spatial_interaction_cutoff[k] >= 0.0)) {
      c->err = "spatial_interaction_cutoff must be >= 0 (DBL_MAX: no cutoff)";
      return PEPCG_ERR_BAD_ARG;
    }
  if (has_spatial_cutoff(*p) && p->precision != PEPCG_PRECISION_PLAIN) {
    c->err = "spatial_interaction_cutoff is applied by the plain (FP64) walks only";
    return PEPCG_ERR_UNSUPPORTED;
  }
  return PEPCG_OK;
}

// tree_walk_init_aux (module_tree_walk_simple.f90:168-211) for keyed targets
// that are not the grown particles: recursive split of the key-ordered
// target keys into groups of at most T.
static void tiles_rec(const int64_t* keys, int64_t lo, int64_t hi, int64_t k, int l, int T,
                      std::vector<int32_t>& out, bool& err) {
  int64_t np = hi - lo;
  if (np == 0) return;
  if (np <= T) {
    out.push_back((int32_t)lo);
    out.push_back((int32_t)np);
    return;
  }
  if (l >= kMaxLevel) {
    err = true;
    return;
  }
  int64_t ps = lo;
  for (int ic = 0; ic < 8; ++ic) {
    int64_t ck = (k << 3) + ic;
    int64_t pe = ps;
    while (pe < hi && (keys[pe] >> (3 * (kMaxLevel - (l + 1)))) == ck) ++pe;
    tiles_rec(keys, ps, pe, ck, l + 1, T, out, err);
    if (err) return;
    ps = pe;
  }
}

int host_tiles(Ctx* c, int64_t nt, const int64_t* d_tkeys, int T, int2* d_tiles,
               int64_t* ntiles) {
  std::vector<int32_t> out;
  if (d_tkeys == nullptr) {  // unkeyed targets: one tile each (:156-160)
    out.resize(2 * nt);
    for (int64_t i = 0; i < nt; ++i) {
      out[2 * i] = (int32_t)i;
      out[2 * i + 1] = 1;
    }
  } else {
    std::vector<int64_t> keys(nt);
    if (!cuda_ok(c, cudaMemcpyAsync(keys.data(), d_tkeys, nt * 8, cudaMemcpyDeviceToHost, c->stream),
                 "tile keys") ||
        !cuda_ok(c, cudaStreamSynchronize(c->stream), "tile keys"))
      return PEPCG_ERR_CUDA;
    if (keys[0] == 0) {  // KEY_INVALID: unkeyed (module_tree_walk_simple.f90:156)
      out.resize(2 * nt);
      for (int64_t i = 0; i < nt; ++i) {
        out[2 * i] = (int32_t)i;
        out[2 * i + 1] = 1;
      }
    } else {
      bool err = false;
      tiles_rec(keys.data(), 0, nt, 1, 0, T, out, err);
      if (err) {
        c->err = "walk_simple: insufficient key resolution in tile formation";
        return PEPCG_ERR_MAXLEVEL;
      }
    }
  }
  *ntiles = (int64_t)out.size() / 2;
  if (!cuda_ok(c, cudaMemcpyAsync(d_tiles, out.data(), out.size() * 4, cudaMemcpyHostToDevice,
                                  c->stream), "tiles upload") ||
      !cuda_ok(c, cudaStreamSynchronize(c->stream), "tiles upload"))
    return PEPCG_ERR_CUDA;
  return PEPCG_OK;
}

}  // namespace pepcg

using namespace pepcg;

static Ctx* as_ctx(void* p) { return static_cast<Ctx*>(p); }

extern "C" {

void pepcg_params_default(pepcg_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->theta2 = 0.36;  // coulomb/module_interaction_specific.f90:38
  p->eps2 = 0.0;     // :39
  p->force_law = 3;  // :35
  p->mac_select = 0; // :36
  p->curve = PEPCG_CURVE_HILBERT;
  p->precision = PEPCG_PRECISION_PLAIN;
  p->walk = PEPCG_WALK_PER_TARGET;
  p->tile_size = 16;  // module_tree_walk_simple.f90:40
  p->mirror_box_layers = 1;
  p->include_far_field_if_periodic = 1;
  p->fmm_extrinsic_correction = 2;
  p->t_lattice_1[0] = 1.0;
  p->t_lattice_2[1] = 1.0;
  p->t_lattice_3[2] = 1.0;
  p->device = 0;
  for (int k = 0; k < 3; ++k)  // huge(0._kind_physics), module_mirror_boxes.f90:52
    p->spatial_interaction_cutoff[k] = DBL_MAX;
}

const char* pepcg_last_error(const void* ctx) {
  if (!ctx) return g_static_err.c_str();
  return static_cast<const Ctx*>(ctx)->err.c_str();
}

int pepcg_create(void** out, const pepcg_params* p) {
  if (!out || !p) {
    g_static_err = "pepcg_create: null argument";
    return PEPCG_ERR_BAD_ARG;
  }
  *out = nullptr;
  Ctx* c = new (std::nothrow) Ctx;
  if (!c) return PEPCG_ERR_OOM;
  int rc = check_params(c, p);
  if (rc) {
    g_static_err = c->err;
    delete c;
    return rc;
  }
  c->prm = *p;
  c->device = p->device;
  int ndev = 0;
  if (!cuda_ok(nullptr, cudaGetDeviceCount(&ndev), "cudaGetDeviceCount") || ndev == 0 ||
      p->device < 0 || p->device >= ndev) {
    if (ndev == 0 && g_static_err.empty()) g_static_err = "no CUDA device";
    delete c;
    return PEPCG_ERR_CUDA;
  }
  if (!cuda_ok(nullptr, cudaSetDevice(c->device), "cudaSetDevice") ||
      !cuda_ok(nullptr, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream")) {
    delete c;
    return PEPCG_ERR_CUDA;
  }
  c->own_stream = true;
  for (int i = 0; i < Ctx::kEvents; ++i) cudaEventCreate(&c->ev[i]);
  bool ok = cuda_ok(nullptr, cudaMalloc((void**)&c->d_box, 64 * sizeof(double)), "box") &&
            cuda_ok(nullptr, cudaMalloc((void**)&c->d_status, 16), "status") &&
            cuda_ok(nullptr, cudaMalloc((void**)&c->d_small, 16 * sizeof(unsigned long long)), "small") &&
            cuda_ok(nullptr, cudaMalloc((void**)&c->d_vbox, 3 * 125 * sizeof(double)), "vbox") &&
            cuda_ok(nullptr, cudaMalloc((void**)&c->d_part, 6 * 512 * sizeof(double)), "part") &&
            cuda_ok(nullptr, cudaHostAlloc((void**)&c->h_sum, sizeof(Ctx::GrowSummary),
                                           cudaHostAllocMapped), "grow summary") &&
            cuda_ok(nullptr, cudaHostGetDevicePointer((void**)&c->d_sum, c->h_sum, 0), "grow summary") &&
            cuda_ok(nullptr, cudaEventCreateWithFlags(&c->sum_ev, cudaEventDisableTiming), "grow summary") &&
            cuda_ok(nullptr, cudaEventCreateWithFlags(&c->keys_ev, cudaEventDisableTiming), "grow keys");
  if (!ok) {
    pepcg_destroy(c);
    return PEPCG_ERR_CUDA;
  }
  prepare_boxes(c);
  cudaMemcpy(c->d_vbox, c->vbox, 3 * c->nboxes * sizeof(double), cudaMemcpyHostToDevice);
  if (!ensure(c, c->counters, 8, "counters")) {
    g_static_err = c->err;
    pepcg_destroy(c);
    return PEPCG_ERR_OOM;
  }
  if (c->far_field) {
    rc = lattice_prepare(c);
    if (rc) {
      g_static_err = c->err;
      pepcg_destroy(c);
      return rc;
    }
  }
  *out = c;
  return PEPCG_OK;
}

int pepcg_destroy(void* ctx) {
  Ctx* c = as_ctx(ctx);
  if (!c) return PEPCG_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  release(c->x); release(c->y); release(c->z); release(c->q);
  release(c->key); release(c->perm);
  release(c->in_x); release(c->in_y); release(c->in_z); release(c->in_q);
  release(c->packed); release(c->skey); release(c->skey_alt); release(c->sval); release(c->sval_alt);
  release(c->hist); release(c->orig_key); release(c->dup_list); release(c->tiepre); release(c->sortio);
  release(c->lev); release(c->lcpn);
  release(c->cstart); release(c->cend); release(c->sstart); release(c->send);
  release(c->scan_tmp);
  release(c->nc4); release(c->meta); release(c->fwd); release(c->fwdf); release(c->tflag); release(c->tpack); release(c->mom);
  release(c->mom32);
  release(c->parent); release(c->nchild); release(c->twiglist); release(c->lvlcnt); release(c->lvlblk);
  release(c->drec); release(c->lvlpos); release(c->dmom);
  release(c->tinfo); release(c->tcounts); release(c->macb); release(c->first_part);
  release(c->nleaves); release(c->child8); release(c->wstack); release(c->leafnode);
  release(c->adj); release(c->fpo2rpo); release(c->rpo2fpo); release(c->nkey);
  release(c->tiles); release(c->counters); release(c->tgt); release(c->tkeys);
  for (void* p : {(void*)c->d_box, (void*)c->d_status, (void*)c->d_small, (void*)c->d_vbox,
                  (void*)c->d_part, (void*)c->d_mlattice, (void*)c->d_omega, (void*)c->d_mu,
                  (void*)c->d_fmm_aux, (void*)c->d_factorial})
    if (p) cudaFree(p);
  for (int i = 0; i < Ctx::kEvents; ++i)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  if (c->h_sum) cudaFreeHost(c->h_sum);
  if (c->sum_ev) cudaEventDestroy(c->sum_ev);
  if (c->keys_ev) cudaEventDestroy(c->keys_ev);
  for (int i = 0; i < Ctx::kMaxChunks; ++i) {
    if (c->ready[i]) cudaEventDestroy(c->ready[i]);
    if (c->done[i]) cudaEventDestroy(c->done[i]);
  }
  for (cudaEvent_t e : {c->fork, c->join})
    if (e) cudaEventDestroy(e);
  for (cudaStream_t t : {c->h2d, c->d2h, c->walk2})
    if (t) {
      cudaStreamSynchronize(t);
      cudaStreamDestroy(t);
    }
  if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
  return PEPCG_OK;
}

int pepcg_set_params(void* ctx, const pepcg_params* p) {
  Ctx* c = as_ctx(ctx);
  if (!c || !p) return PEPCG_ERR_BAD_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  bool geom_changed = std::memcmp(p->periodicity, c->prm.periodicity, sizeof(p->periodicity)) ||
                      p->mirror_box_layers != c->prm.mirror_box_layers ||
                      std::memcmp(p->t_lattice_1, c->prm.t_lattice_1, 12 * sizeof(double)) ||
                      p->include_far_field_if_periodic != c->prm.include_far_field_if_periodic ||
                      p->fmm_extrinsic_correction != c->prm.fmm_extrinsic_correction ||
                      p->curve != c->prm.curve || p->force_cubic_domain != c->prm.force_cubic_domain ||
                      p->device != c->prm.device;
  if (geom_changed) {
    c->err = "pepcg_set_params: geometry, curve and device are fixed at creation";
    return PEPCG_ERR_BAD_ARG;
  }
  c->prm = *p;
  return PEPCG_OK;
}

// The copy streams and chunk events of the host-array entry points, created on
// first use.
static bool copy_streams(Ctx* c) {
  if (c->h2d) return true;
  bool ok = cuda_ok(c, cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking), "copy stream") &&
            cuda_ok(c, cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking), "copy stream") &&
            cuda_ok(c, cudaStreamCreateWithFlags(&c->walk2, cudaStreamNonBlocking), "walk stream") &&
            cuda_ok(c, cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming), "event") &&
            cuda_ok(c, cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming), "event");
  for (int i = 0; ok && i < Ctx::kMaxChunks; ++i)
    ok = cuda_ok(c, cudaEventCreateWithFlags(&c->ready[i], cudaEventDisableTiming), "event") &&
         cuda_ok(c, cudaEventCreateWithFlags(&c->done[i], cudaEventDisableTiming), "event");
  return ok;
}

// Waits for both copy streams (they may hold transfers of caller arrays) and
// folds their status into ok.
static bool drain_copies(Ctx* c, bool ok) {
  for (cudaStream_t t : {c->h2d, c->d2h})
    if (t) ok = cuda_ok(c, cudaStreamSynchronize(t), "copy stream") && ok;
  return ok;
}

int pepcg_grow_tree_device(void* ctx, int64_t n, const double* d_x, const double* d_y,
                           const double* d_z, const double* d_q) {
  Ctx* c = as_ctx(ctx);
  if (!c || !d_x || !d_y || !d_z || !d_q) return PEPCG_ERR_BAD_ARG;
  cudaSetDevice(c->device);
  int rc = grow_device(c, n, d_x, d_y, d_z, d_q);
  if (rc) return rc;
  if (c->far_field) {
    rc = lattice_timestep(c);
    if (rc && rc != PEPCG_WARN_NOT_NEUTRAL) return rc;
  }
  c->grow_times_pending = true;  // read the phase events later, without a sync here
  return rc;
}

int pepcg_grow_tree(void* ctx, int64_t n, const double* x, const double* y, const double* z,
                    const double* q, int64_t* key_out, int64_t* perm_out, double* x_out,
                    double* y_out, double* z_out) {
  Ctx* c = as_ctx(ctx);
  if (!c || !x || !y || !z || !q || n < 0) return PEPCG_ERR_BAD_ARG;
  cudaSetDevice(c->device);
  if (n < 2) {
    c->err = "pepcg_grow_tree: need at least 2 particles (module_domains.f90:187)";
    return PEPCG_ERR_BAD_ARG;
  }
  if (!ensure(c, c->in_x, n, "in_x") || !ensure(c, c->in_y, n, "in_y") ||
      !ensure(c, c->in_z, n, "in_z") || !ensure(c, c->in_q, n, "in_q"))
    return PEPCG_ERR_OOM;
  cudaStream_t s = c->stream;
  if (!copy_streams(c)) return PEPCG_ERR_CUDA;
  // x y z on the context stream; the charges follow on the upload stream and
  // cross PCIe while the keys are formed and sorted (the gather into key order
  // is the first step that reads them)
  if (!cuda_ok(c, cudaMemcpyAsync(c->in_x.p, x, n * 8, cudaMemcpyHostToDevice, s), "H2D x") ||
      !cuda_ok(c, cudaMemcpyAsync(c->in_y.p, y, n * 8, cudaMemcpyHostToDevice, s), "H2D y") ||
      !cuda_ok(c, cudaMemcpyAsync(c->in_z.p, z, n * 8, cudaMemcpyHostToDevice, s), "H2D z") ||
      !cuda_ok(c, cudaEventRecord(c->fork, s), "H2D q") ||
      !cuda_ok(c, cudaStreamWaitEvent(c->h2d, c->fork, 0), "H2D q") ||
      !cuda_ok(c, cudaMemcpyAsync(c->in_q.p, q, n * 8, cudaMemcpyHostToDevice, c->h2d), "H2D q") ||
      !cuda_ok(c, cudaEventRecord(c->join, c->h2d), "H2D q"))
    return drain_copies(c, false), PEPCG_ERR_CUDA;
  int rc = grow_device(c, n, c->in_x.p, c->in_y.p, c->in_z.p, c->in_q.p, c->join);
  if (rc) return drain_copies(c, false), rc;
  if (c->far_field) {
    rc = lattice_timestep(c);
    if (rc && rc != PEPCG_WARN_NOT_NEUTRAL) return drain_copies(c, false), rc;
  }
  c->grow_times_pending = true;
  // Copy the outputs back on the device-to-host stream while the rest of the
  // grow runs on the context stream: the keys and the permutation (the sorted
  // indices) once the duplicate fix has shifted the keys (keys_ev), the
  // coordinates once the particles stand in key order (event 2, before the
  // tree build).  The call returns when the copies are done; the rest of the
  // grow stays stream-ordered before the next call's work.
  cudaStream_t t = c->d2h;
  bool ok = cuda_ok(c, cudaStreamWaitEvent(t, c->keys_ev, 0), "grow outputs");
  if (key_out)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(key_out, c->key.p, n * 8, cudaMemcpyDeviceToHost, t), "D2H key");
  if (perm_out) {
    // widened to 64 bits on the device (scratch: the target-key buffer)
    if (!ensure(c, c->tkeys, n, "perm")) return drain_copies(c, false), PEPCG_ERR_OOM;
    ok = ok && widen_perm_device(c, c->tkeys.p, t, c->sval.p) == PEPCG_OK &&
         cuda_ok(c, cudaMemcpyAsync(perm_out, c->tkeys.p, n * 8, cudaMemcpyDeviceToHost, t),
                 "D2H perm");
  }
  ok = ok && cuda_ok(c, cudaStreamWaitEvent(t, c->ev[2], 0), "grow outputs");
  if (x_out) ok = ok && cuda_ok(c, cudaMemcpyAsync(x_out, c->x.p, n * 8, cudaMemcpyDeviceToHost, t), "D2H x");
  if (y_out) ok = ok && cuda_ok(c, cudaMemcpyAsync(y_out, c->y.p, n * 8, cudaMemcpyDeviceToHost, t), "D2H y");
  if (z_out) ok = ok && cuda_ok(c, cudaMemcpyAsync(z_out, c->z.p, n * 8, cudaMemcpyDeviceToHost, t), "D2H z");
  if (!drain_copies(c, ok)) return PEPCG_ERR_CUDA;
  return rc;
}

int pepcg_get_particles_device(void* ctx, int64_t* d_key, int64_t* d_perm, double* d_x,
                               double* d_y, double* d_z, double* d_q) {
  Ctx* c = as_ctx(ctx);
  if (!c) return PEPCG_ERR_BAD_ARG;
  if (!c->has_tree) {
    c->err = "no grown tree";
    return PEPCG_ERR_NO_TREE;
  }
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  const int64_t n = c->n;
  bool ok = true;
  if (d_key) ok = ok && cuda_ok(c, cudaMemcpyAsync(d_key, c->key.p, n * 8, cudaMemcpyDeviceToDevice, s), "key");
  if (d_x) ok = ok && cuda_ok(c, cudaMemcpyAsync(d_x, c->x.p, n * 8, cudaMemcpyDeviceToDevice, s), "x");
  if (d_y) ok = ok && cuda_ok(c, cudaMemcpyAsync(d_y, c->y.p, n * 8, cudaMemcpyDeviceToDevice, s), "y");
  if (d_z) ok = ok && cuda_ok(c, cudaMemcpyAsync(d_z, c->z.p, n * 8, cudaMemcpyDeviceToDevice, s), "z");
  if (d_q) ok = ok && cuda_ok(c, cudaMemcpyAsync(d_q, c->q.p, n * 8, cudaMemcpyDeviceToDevice, s), "q");
  if (d_perm && ok) ok = widen_perm_device(c, d_perm) == PEPCG_OK;
  ok = ok && cuda_ok(c, cudaStreamSynchronize(s), "get particles");
  return ok ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int pepcg_traverse_tree_device(void* ctx, int64_t nt, const double* d_tx, const double* d_ty,
                               const double* d_tz, const int64_t* d_tkeys, double* d_ex,
                               double* d_ey, double* d_ez, double* d_pot, double* d_work) {
  Ctx* c = as_ctx(ctx);
  if (!c || nt < 0 || !d_tx || !d_ty || !d_tz || !d_ex || !d_ey || !d_ez || !d_pot || !d_work)
    return PEPCG_ERR_BAD_ARG;
  cudaSetDevice(c->device);
  const double* tq = c->prm.force_law == 5 ? grown_charges_if_same(c, nt, d_tkeys) : nullptr;
  return traverse_device(c, nt, d_tx, d_ty, d_tz, d_tkeys, false, d_ex, d_ey, d_ez, d_pot, d_work,
                         tq);
}

int pepcg_traverse_self_device(void* ctx, double* d_ex, double* d_ey, double* d_ez,
                               double* d_pot, double* d_work) {
  Ctx* c = as_ctx(ctx);
  if (!c || !d_ex || !d_ey || !d_ez || !d_pot || !d_work) return PEPCG_ERR_BAD_ARG;
  if (!c->has_tree) {
    c->err = "no grown tree";
    return PEPCG_ERR_NO_TREE;
  }
  cudaSetDevice(c->device);
  return traverse_device(c, c->n, c->x.p, c->y.p, c->z.p, c->key.p, true, d_ex, d_ey, d_ez, d_pot,
                         d_work, c->q.p);
}

int pepcg_traverse_range_device(void* ctx, int64_t t0, int64_t t1, double* d_ex, double* d_ey,
                                double* d_ez, double* d_pot, double* d_work) {
  Ctx* c = as_ctx(ctx);
  if (!c || !d_ex || !d_ey || !d_ez || !d_pot || !d_work) return PEPCG_ERR_BAD_ARG;
  if (!c->has_tree) {
    c->err = "no grown tree";
    return PEPCG_ERR_NO_TREE;
  }
  if (t0 < 0 || t1 < t0 || t1 > c->n) {
    c->err = "pepcg_traverse_range_device: need 0 <= t0 <= t1 <= n";
    return PEPCG_ERR_BAD_ARG;
  }
  if (t0 == t1) return PEPCG_OK;
  cudaSetDevice(c->device);
  if (t0 == 0 && t1 == c->n)
    return traverse_device(c, c->n, c->x.p, c->y.p, c->z.p, c->key.p, true, d_ex, d_ey, d_ez,
                           d_pot, d_work, c->q.p);
  // the range's own keys give the per-tile walk its tiles, as a rank's local keys would
  return traverse_device(c, t1 - t0, c->x.p + t0, c->y.p + t0, c->z.p + t0, c->key.p + t0, false,
                         d_ex, d_ey, d_ez, d_pot, d_work, c->q.p + t0);
}

int pepcg_restore_device(void* ctx, const double* d_in, double* d_out) {
  Ctx* c = as_ctx(ctx);
  if (!c || !d_in || !d_out || d_in == d_out) {
    if (c) c->err = "pepcg_restore_device: distinct input and output arrays are required";
    return PEPCG_ERR_BAD_ARG;
  }
  if (!c->has_tree) {
    c->err = "pepcg_restore_device: no grown tree (the permutation comes from the last grow)";
    return PEPCG_ERR_NO_TREE;
  }
  cudaSetDevice(c->device);
  return restore_device(c, d_in, d_out);
}

// Host targets at least this many are walked in chunks, overlapping the
// uploads and downloads with the walk.
constexpr int64_t kChunkedTargets = 1 << 18;

int pepcg_traverse_tree(void* ctx, int64_t nt, const double* tx, const double* ty,
                        const double* tz, const int64_t* tkeys, double* ex, double* ey,
                        double* ez, double* pot, double* work) {
  Ctx* c = as_ctx(ctx);
  if (!c || nt < 0 || !tx || !ty || !tz || !ex || !ey || !ez || !pot || !work)
    return PEPCG_ERR_BAD_ARG;
  if (nt == 0) return PEPCG_OK;
  cudaSetDevice(c->device);
  // the keys steer only the per-tile walk's tiles and the Kelbg law's charges
  const bool keys_used = tkeys && (c->prm.walk == PEPCG_WALK_PER_TILE || c->prm.force_law == 5);
  if (!ensure(c, c->tgt, 8 * nt, "targets") || (keys_used && !ensure(c, c->tkeys, nt, "tkeys")))
    return PEPCG_ERR_OOM;
  cudaStream_t s = c->stream;
  double* b = c->tgt.p;
  const double* hin[8] = {tx, ty, tz, ex, ey, ez, pot, work};
  double* hout[5] = {ex, ey, ez, pot, work};
  // with overwrite_results the old values are not uploaded: the walk adds to zeros
  const int nin = c->prm.overwrite_results ? 3 : 8;
  const bool chunked = nt >= kChunkedTargets && !keys_used && c->prm.walk != PEPCG_WALK_PER_TILE &&
                       !c->far_field && c->has_tree;
  if (chunked) {
    // five chunks of 1/32, 2/32, 25/32, 3/32 and 1/32 of the targets: the walk
    // starts after 1/32 of the upload, each later chunk's upload finishes
    // while the earlier chunks walk (an upload moves 24 bytes per target, the
    // walk takes ~8 ns per target, PCIe ~50 GB/s), each chunk's download (40
    // bytes per target) runs while the later chunks walk, and only the last
    // 1/32 of the download trails the walk
    if (!copy_streams(c)) return PEPCG_ERR_CUDA;
    const int nch = 5;
    auto al = [](int64_t v) { return v & ~(int64_t)63; };  // whole group-walk buckets
    const int64_t bounds[nch + 1] = {0, al(nt / 32), al(3 * (nt / 32)), al(nt - 4 * (nt / 32)),
                                     al(nt - nt / 32), nt};
    bool ok = true;
    for (int k = 0; k < nch; ++k) {
      const int64_t t0 = bounds[k], len = bounds[k + 1] - bounds[k];
      for (int a = 0; a < nin && len > 0; ++a)
        ok = ok && cuda_ok(c, cudaMemcpyAsync(b + a * nt + t0, hin[a] + t0, len * 8,
                                              cudaMemcpyHostToDevice, c->h2d), "H2D");
      ok = ok && cuda_ok(c, cudaEventRecord(c->ready[k], c->h2d), "event");
    }
    if (nin == 3)
      ok = ok && cuda_ok(c, cudaMemsetAsync(b + 3 * nt, 0, 5 * nt * 8, s), "clear results");
    if (!ok) return drain_copies(c, false), PEPCG_ERR_CUDA;
    ChunkPlan plan;
    plan.nchunks = nch;
    plan.bounds = bounds;
    plan.ready = c->ready;
    plan.done = c->done;
    plan.before_sync = [&]() {
      bool okd = true;
      for (int k = 0; k < nch; ++k) {
        const int64_t t0 = bounds[k], len = bounds[k + 1] - bounds[k];
        okd = okd && cuda_ok(c, cudaStreamWaitEvent(c->d2h, c->done[k], 0), "chunk wait");
        for (int r = 0; r < 5 && len > 0; ++r)
          okd = okd && cuda_ok(c, cudaMemcpyAsync(hout[r] + t0, b + (3 + r) * nt + t0, len * 8,
                                                  cudaMemcpyDeviceToHost, c->d2h), "D2H");
      }
      return okd;
    };
    int rc = traverse_device(c, nt, b, b + nt, b + 2 * nt, nullptr, false, b + 3 * nt,
                             b + 4 * nt, b + 5 * nt, b + 6 * nt, b + 7 * nt, nullptr, &plan);
    const bool drained = drain_copies(c, true);
    if (rc && rc != PEPCG_WARN_NOT_NEUTRAL) return rc;
    return drained ? rc : PEPCG_ERR_CUDA;
  }
  bool ok = true;
  for (int k = 0; k < nin; ++k)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(b + k * nt, hin[k], nt * 8, cudaMemcpyHostToDevice, s), "H2D");
  if (nin == 3)
    ok = ok && cuda_ok(c, cudaMemsetAsync(b + 3 * nt, 0, 5 * nt * 8, s), "clear results");
  if (keys_used)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(c->tkeys.p, tkeys, nt * 8, cudaMemcpyHostToDevice, s), "H2D");
  if (!ok) return PEPCG_ERR_CUDA;
  const double* tq =
      c->prm.force_law == 5 ? grown_charges_if_same(c, nt, keys_used ? c->tkeys.p : nullptr) : nullptr;
  int rc = traverse_device(c, nt, b, b + nt, b + 2 * nt, keys_used ? c->tkeys.p : nullptr, false,
                           b + 3 * nt, b + 4 * nt, b + 5 * nt, b + 6 * nt, b + 7 * nt, tq);
  if (rc && rc != PEPCG_WARN_NOT_NEUTRAL) return rc;
  for (int k = 0; k < 5; ++k)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(hout[k], b + (3 + k) * nt, nt * 8, cudaMemcpyDeviceToHost, s), "D2H");
  ok = ok && cuda_ok(c, cudaStreamSynchronize(s), "traverse");
  return ok ? rc : PEPCG_ERR_CUDA;
}

int pepcg_set_stream(void* ctx, void* stream) {
  Ctx* c = as_ctx(ctx);
  if (!c) return PEPCG_ERR_BAD_ARG;
  cudaSetDevice(c->device);
  if (!cuda_ok(c, cudaStreamSynchronize(c->stream), "set stream")) return PEPCG_ERR_CUDA;
  if (c->own_stream) {
    cudaStreamDestroy(c->stream);
    c->own_stream = false;
  }
  if (stream == nullptr) {
    if (!cuda_ok(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream"))
      return PEPCG_ERR_CUDA;
    c->own_stream = true;
  } else {
    c->stream = static_cast<cudaStream_t>(stream);
  }
  return PEPCG_OK;
}

long long pepcg_kernel_launches(void) { return g_launches.load(); }

int pepcg_traverse_adjoint_device(void* ctx, int64_t nt, const double* d_tx, const double* d_ty,
                                  const double* d_tz, const double* d_gex, const double* d_gey,
                                  const double* d_gez, const double* d_gphi, double* d_dq,
                                  double* d_dx, double* d_dy, double* d_dz) {
  Ctx* c = as_ctx(ctx);
  if (!c || nt < 0 || !d_tx || !d_ty || !d_tz || !d_gex || !d_gey || !d_gez || !d_gphi || !d_dq ||
      !d_dx || !d_dy || !d_dz)
    return PEPCG_ERR_BAD_ARG;
  cudaSetDevice(c->device);
  return adjoint_device(c, nt, d_tx, d_ty, d_tz, d_gex, d_gey, d_gez, d_gphi, d_dq, d_dx, d_dy, d_dz);
}

int pepcg_traverse_adjoint(void* ctx, int64_t nt, const double* tx, const double* ty,
                           const double* tz, const double* dLdEx, const double* dLdEy,
                           const double* dLdEz, const double* dLdphi, double* dLdq, double* dLdx,
                           double* dLdy, double* dLdz) {
  Ctx* c = as_ctx(ctx);
  if (!c || nt < 0 || !tx || !ty || !tz || !dLdEx || !dLdEy || !dLdEz || !dLdphi || !dLdq ||
      !dLdx || !dLdy || !dLdz)
    return PEPCG_ERR_BAD_ARG;
  if (!c->has_tree) {
    c->err = "no grown tree";
    return PEPCG_ERR_NO_TREE;
  }
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  const int64_t n = c->n;
  if (!ensure(c, c->tgt, 7 * nt + 4 * n, "adjoint staging")) return PEPCG_ERR_OOM;
  double* b = c->tgt.p;
  const double* hin[7] = {tx, ty, tz, dLdEx, dLdEy, dLdEz, dLdphi};
  bool ok = true;
  for (int k = 0; k < 7; ++k)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(b + k * nt, hin[k], nt * 8, cudaMemcpyHostToDevice, s), "H2D");
  if (!ok) return PEPCG_ERR_CUDA;
  double* o = b + 7 * nt;
  int rc = adjoint_device(c, nt, b, b + nt, b + 2 * nt, b + 3 * nt, b + 4 * nt, b + 5 * nt,
                          b + 6 * nt, o, o + n, o + 2 * n, o + 3 * n);
  if (rc) return rc;
  double* hout[4] = {dLdq, dLdx, dLdy, dLdz};
  for (int k = 0; k < 4; ++k)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(hout[k], o + k * n, n * 8, cudaMemcpyDeviceToHost, s), "D2H");
  ok = ok && cuda_ok(c, cudaStreamSynchronize(s), "adjoint");
  return ok ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int pepcg_timber_tree(void* ctx) {
  Ctx* c = as_ctx(ctx);
  if (!c) return PEPCG_ERR_BAD_ARG;
  c->has_tree = false;  // buffers are kept for the next grow (reused, grow-only)
  return PEPCG_OK;
}

int pepcg_stats_get(void* ctx, pepcg_stats* s) {
  Ctx* c = as_ctx(ctx);
  if (!c || !s) return PEPCG_ERR_BAD_ARG;
  if (c->grow_times_pending && cudaEventSynchronize(c->ev[4]) == cudaSuccess) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]) == cudaSuccess) c->st.t_keys_ms = ms;
    // the particle gather (a sort-phase step) runs after the node counts (a
    // tree-phase step), while the host reads the grow summary
    float a = 0, b = 0;
    if (cudaEventElapsedTime(&a, c->ev[1], c->ev[8]) == cudaSuccess &&
        cudaEventElapsedTime(&b, c->ev[9], c->ev[2]) == cudaSuccess)
      c->st.t_sort_ms = a + b;
    if (cudaEventElapsedTime(&a, c->ev[8], c->ev[9]) == cudaSuccess &&
        cudaEventElapsedTime(&b, c->ev[2], c->ev[3]) == cudaSuccess)
      c->st.t_tree_ms = a + b;
    if (cudaEventElapsedTime(&ms, c->ev[3], c->ev[4]) == cudaSuccess) c->st.t_upward_ms = ms;
    c->grow_times_pending = false;
  }
  c->st.npart = c->n;
  c->st.nleaf = c->n;
  c->st.ntwig = c->ntwig;
  c->st.max_level = c->max_level;
  c->st.dup_count = c->dup_count;
  for (int i = 0; i < 9; ++i) c->st.box[i] = c->box[i];
  *s = c->st;
  return PEPCG_OK;
}

int64_t pepcg_num_nodes(void* ctx) {
  Ctx* c = as_ctx(ctx);
  if (!c || !c->has_tree) return 0;
  return c->nnodes;
}

int pepcg_tree_export(void* ctx, int64_t* key, int32_t* level, int64_t* leaves,
                      int64_t* descendants, int64_t* parent, int64_t* first_child,
                      int64_t* next_sibling, double* moments15) {
  Ctx* c = as_ctx(ctx);
  if (!c) return PEPCG_ERR_BAD_ARG;
  if (!c->has_tree) {
    c->err = "no grown tree";
    return PEPCG_ERR_NO_TREE;
  }
  cudaSetDevice(c->device);
  return export_tree(c, key, level, leaves, descendants, parent, first_child, next_sibling,
                     moments15);
}

int pepcg_direct(void* ctx, int64_t ntest, const int64_t* tidx, double* ex, double* ey,
                 double* ez, double* pot) {
  Ctx* c = as_ctx(ctx);
  if (!c || ntest < 0 || !tidx || !ex || !ey || !ez || !pot) return PEPCG_ERR_BAD_ARG;
  if (!c->has_tree) {
    c->err = "no grown tree";
    return PEPCG_ERR_NO_TREE;
  }
  if (ntest == 0) return PEPCG_OK;
  for (int64_t i = 0; i < ntest; ++i)
    if (tidx[i] < 0 || tidx[i] >= c->n) {
      c->err = "pepcg_direct: target index out of range";
      return PEPCG_ERR_BAD_ARG;
    }
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  if (!ensure(c, c->tgt, 4 * ntest, "direct") || !ensure(c, c->tkeys, ntest, "direct idx"))
    return PEPCG_ERR_OOM;
  if (!cuda_ok(c, cudaMemcpyAsync(c->tkeys.p, tidx, ntest * 8, cudaMemcpyHostToDevice, s), "H2D"))
    return PEPCG_ERR_CUDA;
  double* b = c->tgt.p;
  int rc = direct_device(c, ntest, c->tkeys.p, b, b + ntest, b + 2 * ntest, b + 3 * ntest);
  if (rc) return rc;
  double* hout[4] = {ex, ey, ez, pot};
  bool ok = true;
  for (int k = 0; k < 4; ++k)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(hout[k], b + k * ntest, ntest * 8, cudaMemcpyDeviceToHost, s), "D2H");
  ok = ok && cuda_ok(c, cudaStreamSynchronize(s), "direct");
  return ok ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int pepcg_lattice(void* ctx, int64_t nt, const double* tx, const double* ty, const double* tz,
                  double* ex, double* ey, double* ez, double* pot) {
  Ctx* c = as_ctx(ctx);
  if (!c || nt < 0 || !tx || !ty || !tz || !ex || !ey || !ez || !pot) return PEPCG_ERR_BAD_ARG;
  if (!c->far_field) {
    c->err = "pepcg_lattice: context is not periodic with far field";
    return PEPCG_ERR_BAD_ARG;
  }
  if (!c->has_tree) {
    c->err = "no grown tree (the lattice expansion is formed at grow)";
    return PEPCG_ERR_NO_TREE;
  }
  if (nt == 0) return PEPCG_OK;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  if (!ensure(c, c->tgt, 7 * nt, "lattice")) return PEPCG_ERR_OOM;
  double* b = c->tgt.p;
  const double* hin[3] = {tx, ty, tz};
  bool ok = true;
  for (int k = 0; k < 3; ++k)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(b + k * nt, hin[k], nt * 8, cudaMemcpyHostToDevice, s), "H2D");
  if (!ok) return PEPCG_ERR_CUDA;
  int rc = lattice_add(c, nt, b, b + nt, b + 2 * nt, b + 3 * nt, b + 4 * nt, b + 5 * nt, b + 6 * nt, true);
  if (rc) return rc;
  double* hout[4] = {ex, ey, ez, pot};
  for (int k = 0; k < 4; ++k)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(hout[k], b + (3 + k) * nt, nt * 8, cudaMemcpyDeviceToHost, s), "D2H");
  ok = ok && cuda_ok(c, cudaStreamSynchronize(s), "lattice");
  return ok ? PEPCG_OK : PEPCG_ERR_CUDA;
}

int pepcg_lattice_force(void* ctx, const double pos[3], double e[3], double* phi) {
  if (!pos || !e || !phi) {
    if (ctx) as_ctx(ctx)->err = "pepcg_lattice_force: null argument";
    return PEPCG_ERR_BAD_ARG;
  }
  return pepcg_lattice(ctx, 1, pos, pos + 1, pos + 2, e, e + 1, e + 2, phi);
}

int pepcg_push_particles_device(void* ctx, int64_t n, double dt, const double* d_q,
                                const double* d_m, const double* d_ex, const double* d_ey,
                                const double* d_ez, double* d_vx, double* d_vy, double* d_vz,
                                double* d_x, double* d_y, double* d_z) {
  Ctx* c = as_ctx(ctx);
  if (!c || n < 0 || (n > 0 && (!d_q || !d_m || !d_ex || !d_ey || !d_ez || !d_vx || !d_vy ||
                                !d_vz || !d_x || !d_y || !d_z)))
    return PEPCG_ERR_BAD_ARG;
  if (n == 0) return PEPCG_OK;
  cudaSetDevice(c->device);
  return push_device(c, n, dt, d_q, d_m, d_ex, d_ey, d_ez, d_vx, d_vy, d_vz, d_x, d_y, d_z);
}

int pepcg_apply_external_field_device(void* ctx, int64_t n, double ez_ext, const double* d_z,
                                      double* d_ez, double* d_pot) {
  Ctx* c = as_ctx(ctx);
  if (!c || n < 0 || (n > 0 && (!d_z || !d_ez || !d_pot))) return PEPCG_ERR_BAD_ARG;
  if (n == 0) return PEPCG_OK;
  cudaSetDevice(c->device);
  return external_field_device(c, n, ez_ext, d_z, d_ez, d_pot);
}

int pepcg_potential_energy_device(void* ctx, int64_t n, const double* d_q, const double* d_pot,
                                  double* epot) {
  Ctx* c = as_ctx(ctx);
  if (!c || n < 0 || !epot || (n > 0 && (!d_q || !d_pot))) return PEPCG_ERR_BAD_ARG;
  *epot = 0.0;
  if (n == 0) return PEPCG_OK;
  cudaSetDevice(c->device);
  return potential_energy_device(c, n, d_q, d_pot, epot);
}

int pepcg_constrain_periodic_device(void* ctx, int64_t n, double* d_x, double* d_y, double* d_z) {
  Ctx* c = as_ctx(ctx);
  if (!c || n < 0 || (n > 0 && (!d_x || !d_y || !d_z))) return PEPCG_ERR_BAD_ARG;
  if (n == 0) return PEPCG_OK;
  cudaSetDevice(c->device);
  return wrap_device(c, n, d_x, d_y, d_z);
}

int pepcg_gather_device(void* ctx, const double* d_in, double* d_out) {
  Ctx* c = as_ctx(ctx);
  if (!c || !d_in || !d_out || d_in == d_out) {
    if (c) c->err = "pepcg_gather_device: distinct input and output arrays are required";
    return PEPCG_ERR_BAD_ARG;
  }
  if (!c->has_tree) {
    c->err = "pepcg_gather_device: no grown tree (the permutation comes from the last grow)";
    return PEPCG_ERR_NO_TREE;
  }
  cudaSetDevice(c->device);
  return gather_device(c, d_in, d_out);
}

void pepcg_debug_fail_allocations(int64_t after) { g_fail_after.store(after < 0 ? -1 : after); }

int pepcg_sort_keys_device(void* ctx, int64_t n, const int64_t* d_keys, int64_t* d_keys_out,
                           int64_t* d_perm_out) {
  Ctx* c = as_ctx(ctx);
  if (!c || n < 0 || (n > 0 && !d_keys)) return PEPCG_ERR_BAD_ARG;
  cudaSetDevice(c->device);
  return sort_keys_device(c, n, d_keys, d_keys_out, d_perm_out);
}

int pepcg_sort_keys(void* ctx, int64_t n, const int64_t* keys, int64_t* keys_out,
                    int64_t* perm_out) {
  Ctx* c = as_ctx(ctx);
  if (!c || n < 0 || (n > 0 && !keys)) return PEPCG_ERR_BAD_ARG;
  if (n == 0) return PEPCG_OK;
  cudaSetDevice(c->device);
  if (!ensure(c, c->sortio, 3 * (size_t)n, "sort staging")) return PEPCG_ERR_OOM;
  cudaStream_t s = c->stream;
  int64_t* d_in = c->sortio.p;
  int64_t* d_k = d_in + n;
  int64_t* d_p = d_k + n;
  if (!cuda_ok(c, cudaMemcpyAsync(d_in, keys, n * 8, cudaMemcpyHostToDevice, s), "H2D keys"))
    return PEPCG_ERR_CUDA;
  int rc = sort_keys_device(c, n, d_in, keys_out ? d_k : nullptr, perm_out ? d_p : nullptr);
  if (rc) return rc;
  bool ok = true;
  if (keys_out)
    ok = cuda_ok(c, cudaMemcpyAsync(keys_out, d_k, n * 8, cudaMemcpyDeviceToHost, s), "D2H keys");
  if (perm_out)
    ok = ok && cuda_ok(c, cudaMemcpyAsync(perm_out, d_p, n * 8, cudaMemcpyDeviceToHost, s), "D2H perm");
  ok = ok && cuda_ok(c, cudaStreamSynchronize(s), "sort");
  return ok ? PEPCG_OK : PEPCG_ERR_CUDA;
}

}  // extern "C"
