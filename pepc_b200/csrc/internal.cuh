// internal.cuh -- shared declarations of libpepcg (sm_100a).
//
// Data layout in HBM (all device arrays owned by Ctx):
//   particles, key order, SoA FP64: x y z q, keys (int64), perm (int32: key
//     order -> caller order)
//   nodes, "reverse preorder" (RPO) order: the depth-first preorder of the
//     octree whose children are visited from the LAST key-ordered child to
//     the first.  In that order the per-target LIFO walk of the reference
//     (module_tree_walk_pthreads.f90:604-687: pop last pushed child first) is
//     a forward scan: open a node -> u + 1, accept/leaf -> skip[u].
//       nc4[u]   = (coc x, coc y, coc z, charge)           FP64, every node
//       meta[u]  = (skip, level | leaf flag << 8)          int32 x 2
//       fwd[u]   = (first child in key order, next node after the subtree in
//                   key-order preorder)                     int32 x 2
//       mom[u]   = twig moments (dip x3, quad xx yy zz, xy yz zx), then
//                  abs_charge and bmax                      FP64 x 12 (96 B)
//       mom32[u] = the moments in FP32 (mixed walk)         float4 x 4 (64 B)
//     rpo2fpo / fpo2rpo map RPO to the reference's node order (forward
//     preorder = insertion order of module_tree_grow.f90:623-696).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <functional>
#include <string>

#include "../../include/pepcg.h"

namespace pepcg {

constexpr int kMaxLevel = 20;    // treevars.f90:55 for idim = 3, 64-bit keys

// number of kernels this library has launched (process-wide, for the record
// of GPU work per call)
extern std::atomic<long long> g_launches;
#define COUNT_LAUNCH() (::pepcg::g_launches.fetch_add(1, std::memory_order_relaxed))
constexpr int kLeafFlag = 1 << 8;

// device status word bits (set by kernels, read by the host after a launch)
enum : uint32_t {
  ST_OK = 0,
  ST_MAXLEVEL = 1u << 0,
  ST_INCOMPLETE = 1u << 1,
  ST_TIMEOUT = 1u << 2,
  ST_NONFINITE = 1u << 3,
  ST_DUP_OVERFLOW = 1u << 4,
  ST_NOT_NEUTRAL = 1u << 5,
  ST_SORT_REPLAY = 1u << 6,  // the replay of the reference's sort lost its way (internal)
};

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;  // elements
};

struct Walk;

// Per-node records are whole 32-byte sectors, so that the upward pass writes
// no partial sector (a partial sector costs HBM a read-modify-write):
//   mom  : kMomStride doubles per node, moments [0, 9), abs_charge, bmax, pad
//   mom32: kMom32Stride float4 per node, the FP32 moments of the mixed walk
constexpr int kMomStride = 12;
constexpr int kMomAbs = 9;
constexpr int kMomBmax = 10;
constexpr int kMom32Stride = 4;
// The upward pass's level-ordered twig moments (dmom): the nine moments padded
// to ten doubles, so that each entry is five aligned 16-byte pairs
constexpr int kDmomStride = 10;

// 256-bit global loads and stores (sm_100): one instruction for 32 bytes at a
// 32-byte aligned address.  ld256 is free to be scheduled like a plain load:
// only for data that the running kernel does not write.
__device__ __forceinline__ double4 ld256(const void* p) {
  double4 v;
  asm("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ void st256(void* p, double4 v) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(v.x), "d"(v.y), "d"(v.z),
               "d"(v.w) : "memory");
}
__device__ __forceinline__ void st256f(void* p, float4 a, float4 b) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(a.x),
               "f"(a.y), "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w) : "memory");
}

// The upward pass's level-ordered copy of a node: centre and charge,
// (abs_charge, bmax), and the links by which the 64-target group walk
// traverses the tree in this order (a twig's children are consecutive here):
//   link.x  level-order position of child slot 0 (twigs; 0 for leaves)
//   link.y  level | leaf flag << 8 | number of children << 16
//   link.z  leaves below the node (1 for a leaf)
//   link.w  the node's RPO index (moments, MAC thresholds)
// 64 bytes, two whole sectors.
struct __align__(16) LevelRecord {
  double4 pos;
  double2 ab;
  int4 link;
};

struct Ctx {
  pepcg_params prm;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;

  int64_t n = 0;       // particles in the tree
  int64_t nnodes = 0;  // M
  int64_t ntwig = 0;
  bool has_tree = false;

  // particles (key order)
  DBuf<double> x, y, z, q;
  DBuf<int64_t> key;
  DBuf<int32_t> perm;
  // grow scratch
  DBuf<double> in_x, in_y, in_z, in_q;  // staging for host inputs
  DBuf<double4> packed;                 // (x, y, z, q) in input order, for the permutation
  DBuf<uint64_t> skey, skey_alt;
  DBuf<int32_t> sval, sval_alt;
  DBuf<uint32_t> hist;
  DBuf<int64_t> orig_key;               // sorted keys before the duplicate fix
  DBuf<int32_t> dup_list;
  DBuf<int32_t> tiepre;                 // equal-key pairs before each sorted position (tieorder.cu)
  DBuf<int64_t> sortio;                 // host-array staging of pepcg_sort_keys
  DBuf<int8_t> lev, lcpn;
  DBuf<int32_t> cstart, cend, sstart, send;
  DBuf<int32_t> scan_tmp;
  // nodes (RPO)
  DBuf<double4> nc4;
  DBuf<int2> meta;
  DBuf<int2> fwd;
  DBuf<int2> fwdf;    // fwd's two nodes as forward-preorder indices
  DBuf<int32_t> tflag;  // per target: the length of the tile that starts there, else 0
  DBuf<int32_t> tpack;  // greedy packing of tiles into warps (walk_plain.cu)
  // kMomStride doubles per node (96 B, three whole sectors): the 9 moments,
  // then abs_charge and bmax
  DBuf<double> mom;
  DBuf<float> mom32;  // 16 floats per node (64 B): the FP32 moments, padded
  DBuf<int32_t> parent, nchild, first_part, nleaves;
  DBuf<int32_t> twiglist;  // twig RPO indices grouped by level (upward and adjoint passes)
  DBuf<int32_t> lvlcnt;    // [0, 32) twigs per level
  DBuf<int32_t> lvlblk;    // twigs, then nodes, per (level, block of 256 nodes), scanned
  // level-ordered copy of the node records for the upward pass: centre /
  // charge and (abs_charge, bmax); the twigs' moments by twig-list position
  DBuf<LevelRecord> drec;
  DBuf<int32_t> lvlpos;    // RPO index -> position in drec (the adjoint records' order)
  DBuf<double> dmom;
  DBuf<int2> tinfo;        // per twig-list position: child count | leaf mask << 8, own position
  DBuf<int32_t> tcounts;   // per twig-list position: children, then twig children (scanned)
  DBuf<double> macb;       // per-twig MAC threshold for mac_select != 0
  int32_t lvl_host[kMaxLevel + 1] = {0};  // twigs per level of the grown tree
  DBuf<int4> child8;  // up to 8 children (RPO indices) per twig, as 2 x int4
  DBuf<int32_t> wstack;  // per-warp traversal stacks of the wide group walk
  DBuf<int32_t> leafnode;  // key-ordered particle -> RPO index of its leaf
  DBuf<double> adj;        // adjoint records, 16 doubles per node
  DBuf<int32_t> fpo2rpo, rpo2fpo;
  DBuf<int64_t> nkey;
  // walk scratch
  DBuf<int32_t> tiles;        // PER_TILE tile boundaries
  DBuf<unsigned long long> counters;  // interaction counters
  DBuf<double> tgt;           // staging for host targets / results
  DBuf<int64_t> tkeys;
  // small device state: box (9), boxlength2 (21), status word, dup count ...
  double* d_box = nullptr;    // [0..8] box, [9..29] boxlength2
  uint32_t* d_status = nullptr;
  unsigned long long* d_small = nullptr;  // [0] dup count, [1] nnodes, [2] tile count, ...
                                          // [8], [9] walk bucket queues (one per walk
                                          // stream), [10] adjoint item queue
  double box[9];
  double boxlength2[kMaxLevel + 1];
  int max_level = 0;
  int64_t dup_count = 0;
  // What the host needs from the first half of a grow (node count, box,
  // levels, status), written by one kernel into mapped pinned host memory:
  // the host waits on sum_ev while the particle gather runs on the device.
  struct GrowSummary {
    double box[9 + kMaxLevel + 1];  // box, then boxlength2
    unsigned long long dup_count;
    int32_t starts_before_last;     // nodes started by particles 0 .. n-2
    int32_t starts_last;            // nodes started by particle n-1
    uint32_t status;
    int32_t max_level;
    int32_t lvl[kMaxLevel + 1];
  };
  GrowSummary* h_sum = nullptr;  // host address
  GrowSummary* d_sum = nullptr;  // its device address
  cudaEvent_t sum_ev = nullptr;
  cudaEvent_t keys_ev = nullptr;  // the keys and the sorted indices are final (before the gather)

  // periodic lattice state
  bool periodic = false, far_field = false;
  int nboxes = 1;
  double vbox[3 * 125];      // lattice vectors of the near-field boxes, central last
  double* d_vbox = nullptr;   // the same on the device
  double* d_part = nullptr;   // bbox partials (6 * 296)
  double2* d_mlattice = nullptr;  // 861 complex
  double2* d_omega = nullptr;     // 231 complex
  double2* d_mu = nullptr;        // 861 complex
  double* d_fmm_aux = nullptr;    // box dipole (3), quad trace, fict (4 x 4), nfict, ...
  double* d_factorial = nullptr;  // 0..80

  // statistics
  pepcg_stats st{};
  // phase events: [0] grow start, [1] keys done, [8] sort done, [9] node
  // counts done, [2] particles in key order, [3] tree, [4] upward; [5..7] walk
  static constexpr int kEvents = 10;
  cudaEvent_t ev[kEvents];
  bool grow_times_pending = false;

  // host-transfer overlap (the host-array entry points): one stream per copy
  // direction, untimed events that order chunks across the streams, and a
  // second walk stream, so that a chunk's walk starts on the SMs that the
  // previous chunk's last buckets leave idle; created on first use
  cudaStream_t h2d = nullptr, d2h = nullptr, walk2 = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  static constexpr int kMaxChunks = 8;
  cudaEvent_t ready[kMaxChunks] = {}, done[kMaxChunks] = {};

  int32_t* nleaves_ptr() { return nleaves.p; }
  // The persistent walks take buckets from a counter in the context's own
  // memory, so walks of different contexts may run concurrently on one device.
  // targets per bucket of the group walk (pepcg_params.group_size, 0 resolved)
  int group_size() const {
    return prm.group_size ? prm.group_size : (prm.precision != PEPCG_PRECISION_PLAIN ? 64 : 32);
  }
  // Slot 0 serves walks on the context stream, slot 1 walks on walk2.
  unsigned int* walk_queue(int slot = 0) { return reinterpret_cast<unsigned int*>(d_small + 8 + slot); }
  unsigned long long* item_queue() { return d_small + 10; }
};

// The lanes of one pack of the packed per-tile walks: pack b holds the whole
// tiles in targets [pstart[b], pstart[b + 1]), at most 32, and tflag gives
// each tile's length at its first target.  Returns whether this lane holds a
// target; tl0 is the lane of its tile's first target and len the tile's length.
__device__ __forceinline__ bool pack_lane(const int32_t* __restrict__ pstart,
                                          const int32_t* __restrict__ tflag, int64_t b, int lane,
                                          int& tl0, int& len) {
  const int64_t t0 = pstart[b];
  const int64_t cnt = pstart[b + 1] - t0;
  const int fl = lane < cnt ? tflag[t0 + lane] : 0;
  const unsigned starts = __ballot_sync(0xffffffffu, fl > 0);
  const unsigned upto = lane == 31 ? starts : (starts & ((2u << lane) - 1u));
  tl0 = upto ? 31 - __clz(upto) : 0;
  len = __shfl_sync(0xffffffffu, fl, tl0);
  return (starts & 1u) && lane < cnt && cnt <= 32;
}

// a finite spatial_interaction_cutoff in any direction (the default, huge,
// cuts nothing)
inline bool has_spatial_cutoff(const pepcg_params& p) {
  return p.spatial_interaction_cutoff[0] < 1.0e308 || p.spatial_interaction_cutoff[1] < 1.0e308 ||
         p.spatial_interaction_cutoff[2] < 1.0e308;
}

// ---- helpers implemented in api.cu ----
bool cuda_ok(Ctx* c, cudaError_t e, const char* what);
// error text for entry points without a context (pepcg_last_error(NULL))
void set_static_error(const std::string& msg);
template <class T>
bool ensure(Ctx* c, DBuf<T>& b, size_t n, const char* what);
int status_to_code(Ctx* c, uint32_t st);

// ---- grow.cu ----
// q_ready: the charges dq arrive after the keys are formed; the gather into
// key order waits for this event and reads them from dq (null: dq is ready)
int grow_device(Ctx* c, int64_t n, const double* dx, const double* dy, const double* dz,
                const double* dq, cudaEvent_t q_ready = nullptr);
// the local key sort in the reference's order (keys as unsigned 64-bit values)
int sort_keys_device(Ctx* c, int64_t n, const int64_t* d_in, int64_t* d_kout, int64_t* d_pout);
int export_tree(Ctx* c, int64_t* key, int32_t* level, int64_t* leaves, int64_t* desc,
                int64_t* parent, int64_t* first_child, int64_t* next_sibling, double* mom15);
// device scan helper (exclusive, int32), returns the total through *total (device)
void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, int32_t* tmp,
                        cudaStream_t s);

// ---- tieorder.cu ----
// The replay of the reference's sort on runs of equal keys (k_tie_order).
// Device arrays; scratch of n elements each unless stated.
struct TieArgs {
  int64_t n;
  const uint64_t* skey;            // keys sorted by the LSD sort
  int32_t* sval;                   // input index of each sorted key; rewritten on equal runs
  const unsigned long long* ndup;  // equal neighbours in skey; 0 -> nothing to do
  uint64_t* kb;                    // scratch: keys by input index
  int32_t* A;                      // scratch: the arrangement being replayed
  int32_t* B;                      // scratch
  int32_t* fp;                     // scratch: foreign slot positions
  int32_t* src;                    // scratch: the slot each foreign slot receives from
  int32_t* dpre;                   // scratch, n + 1: equal pairs before each position
  uint16_t* cl;                    // scratch: class per position
  uint16_t* fc;                    // scratch: class per foreign slot
  int2* seg;                       // scratch: 2 * segcap ranges
  int64_t segcap;                  // tie_segcap(n)
  uint32_t* status;
};
int64_t tie_segcap(int64_t n);
bool tie_order_launch(Ctx* c, const TieArgs& a, cudaStream_t s);
// adds the number of i with skey[i] == skey[i + 1] to *npair
void count_pairs_launch(int64_t n, const uint64_t* skey, unsigned long long* npair,
                        cudaStream_t s);

// ---- walk_plain.cu / walk_mixed.cu ----
// tiles of keyed targets that are not the grown particles (host recursion,
// module_tree_walk_simple.f90:168-211); writes (first, count) pairs
int host_tiles(Ctx* c, int64_t nt, const int64_t* d_tkeys, int T, int2* d_tiles, int64_t* ntiles);
// tq: the targets' charges when they are grown particles (the Kelbg law needs
// them), else nullptr
//
// plan (optional) splits the walk into consecutive target ranges so that host
// transfers overlap it: chunk k is launched after the context stream waits on
// ready[k] (when set), done[k] is recorded on the context stream after it, and
// before_sync runs once every chunk is enqueued, before the call waits for
// the walk.  Only the per-target and group walks without the periodic far
// field are split (their per-target results do not depend on the split when
// the interior bounds are multiples of 32).
struct ChunkPlan {
  int nchunks = 1;
  const int64_t* bounds = nullptr;  // nchunks + 1 target offsets
  const cudaEvent_t* ready = nullptr;
  const cudaEvent_t* done = nullptr;
  std::function<bool()> before_sync;
};
int traverse_device(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                    const int64_t* tkeys, bool self, double* ex, double* ey, double* ez,
                    double* pot, double* work, const double* tq = nullptr,
                    const ChunkPlan* plan = nullptr);

// walk_mixed.cu: the transposed adjoint walk of the mixed 64-target group walk
int launch_adjoint_group64(Ctx* c, int64_t nt, const double* tx, const double* ty,
                           const double* tz, const double* gex, const double* gey,
                           const double* gez, const double* gphi, bool with_e, cudaStream_t s);

// ---- adjoint.cu ----
int adjoint_device(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                   const double* gex, const double* gey, const double* gez, const double* gphi,
                   double* dq, double* dx, double* dy, double* dz);

// ---- lattice.cu ----
int lattice_prepare(Ctx* c);
int lattice_timestep(Ctx* c);
// walk_plain.cu: per-twig MAC thresholds for mac_select != 0 (nullptr for Barnes-Hut)
int prepare_mac(Ctx* c, const double** macb);
// the grown particles' charges when the targets are exactly the grown
// particles in key order (same keys), else nullptr
const double* grown_charges_if_same(Ctx* c, int64_t nt, const int64_t* d_tkeys);
// timeloop.cu
int push_device(Ctx* c, int64_t n, double dt, const double* q, const double* m, const double* ex,
                const double* ey, const double* ez, double* vx, double* vy, double* vz, double* x,
                double* y, double* z);
int external_field_device(Ctx* c, int64_t n, double ez_ext, const double* z, double* ez,
                          double* pot);
int wrap_device(Ctx* c, int64_t n, double* x, double* y, double* z);
int gather_device(Ctx* c, const double* in, double* out);
int potential_energy_device(Ctx* c, int64_t n, const double* q, const double* pot,
                            double* epot);
int restore_device(Ctx* c, const double* in, double* out);
// out = the last grow's permutation as int64 (from src, default c->perm);
// st null: c->stream
int widen_perm_device(Ctx* c, int64_t* out, cudaStream_t st = nullptr, const int32_t* src = nullptr);
int lattice_add(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                double* ex, double* ey, double* ez, double* pot, bool overwrite);
// adds the lattice term's dL/dq, dL/dx of the grown particles to dq..dz (the
// caller's original order) for dL/dE, dL/dphi at nt targets
int lattice_adjoint(Ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                    const double* gex, const double* gey, const double* gez, const double* gphi,
                    double* dq, double* dx, double* dy, double* dz);

// ---- direct.cu ----
int direct_device(Ctx* c, int64_t ntest, const int64_t* d_tidx, double* ex, double* ey,
                  double* ez, double* pot);

// ---- scalar.cu ----
// (C entry points only)

}  // namespace pepcg

// ---------------------------------------------------------------------------
// Device arithmetic shared by the kernels (restatements of the reference
// backend, operation order as written in the Fortran source).  The FP64
// translation units are compiled with --fmad=false so that these are
// bit-identical to a non-contracted IEEE evaluation.
// ---------------------------------------------------------------------------
namespace pepcg {

// calc_force_coulomb_3D_direct, coulomb/module_coulomb_kernels.f90:242-257
__host__ __device__ __forceinline__ void force_leaf64(double q, double dx, double dy, double dz,
                                                      double dist2, double& ex, double& ey,
                                                      double& ez, double& phi) {
  double r = sqrt(dist2);
  double rd = 1.0 / r;
  double rd3charge = ((q * rd) * rd) * rd;
  phi = q * rd;
  ex = rd3charge * dx;
  ey = rd3charge * dy;
  ez = rd3charge * dz;
}

// calc_force_coulomb_3D, coulomb/module_coulomb_kernels.f90:60-145.
// m = (dip x, dip y, dip z, quad xx, yy, zz, xy, yz, zx)
__host__ __device__ __forceinline__ void force_twig64(double q, const double* m, double dx,
                                                      double dy, double dz, double dist2,
                                                      double& ex, double& ey, double& ez,
                                                      double& phi) {
  const double r = sqrt(dist2);
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
  const double d1 = m[0], d2 = m[1], d3 = m[2];
  const double q1 = m[3], q2 = m[4], q3 = m[5], qxy = m[6], qyz = m[7], qzx = m[8];
  const double preQx = pre2x * q1;
  const double preQy = pre2y * q2;
  const double preQz = pre2z * q3;
  phi = (((((((q * rd) - (((dx * d1) + (dy * d2)) + (dz * d3)) * rd3) + fdx * q1) + fdy * q2) +
           fdz * q3) + fdxy * qxy) + fdyz * qyz) + fdxz * qzx;
  ex = (((q * dx) * rd3) - (((fdx * d1) + (fdxy * d2)) + (fdxz * d3))) +
       3.0 * ((((dx * ((((pre2x - m2rd5) * q1) + preQy) + preQz)) + ((dy * pre2x) * qxy)) +
               ((dz * pre2x) * qzx)) + (pre1 * qyz));
  ey = (((q * dy) * rd3) - (((fdy * d2) + (fdxy * d1)) + (fdyz * d3))) +
       3.0 * ((((dy * ((((pre2y - m2rd5) * q2) + preQx) + preQz)) + ((dx * pre2y) * qxy)) +
               ((dz * pre2y) * qyz)) + (pre1 * qzx));
  ez = (((q * dz) * rd3) - (((fdz * d3) + (fdyz * d2)) + (fdxz * d1))) +
       3.0 * ((((dz * ((((pre2z - m2rd5) * q3) + preQy) + preQx)) + ((dx * pre2z) * qzx)) +
               ((dy * pre2z) * qyz)) + (pre1 * qxy));
}

// shift_multipoles_up, coulomb/module_interaction_specific.f90:84-140.
// Children in key order; each child c gives coc (3), charge, abs_charge,
// moments m (9) and bmax.  Output: coc, charge, abs_charge, m, bmax.
struct Moments {
  double coc[3];
  double q, absq;
  double m[9];
  double bmax;
};

__host__ __device__ __forceinline__ void shift_up64(const Moments* ch, int nc, Moments& p) {
  double charge = 0.0, absq = 0.0;
  for (int j = 0; j < nc; ++j) charge = charge + ch[j].q;
  for (int j = 0; j < nc; ++j) absq = absq + ch[j].absq;
  double coc[3] = {0.0, 0.0, 0.0};
  if (absq != 0.0) {
    for (int j = 0; j < nc; ++j)
      for (int d = 0; d < 3; ++d) coc[d] = coc[d] + ch[j].coc[d] * ch[j].absq;
    for (int d = 0; d < 3; ++d) coc[d] = coc[d] / absq;
  } else {
    for (int j = 0; j < nc; ++j)
      for (int d = 0; d < 3; ++d) coc[d] = coc[d] + ch[j].coc[d];
    for (int d = 0; d < 3; ++d) coc[d] = coc[d] / (double)nc;
  }
  double dip[3] = {0, 0, 0}, quad[3] = {0, 0, 0}, xy = 0, yz = 0, zx = 0;
  for (int j = 0; j < nc; ++j) {
    const Moments& c = ch[j];
    double s[3];
    for (int d = 0; d < 3; ++d) s[d] = coc[d] - c.coc[d];
    for (int d = 0; d < 3; ++d) dip[d] = (dip[d] + c.m[d]) + c.q * s[d];
    for (int d = 0; d < 3; ++d)
      quad[d] = ((quad[d] + c.m[3 + d]) + c.m[d] * s[d]) + (0.5 * c.q) * (s[d] * s[d]);
    xy = (((xy + c.m[6]) + c.m[0] * s[1]) + c.m[1] * s[0]) + (c.q * s[0]) * s[1];
    yz = (((yz + c.m[7]) + c.m[1] * s[2]) + c.m[2] * s[1]) + (c.q * s[1]) * s[2];
    zx = (((zx + c.m[8]) + c.m[2] * s[0]) + c.m[0] * s[2]) + (c.q * s[2]) * s[0];
  }
  double bmax = 0.0;
  for (int j = 0; j < nc; ++j) {
    double a = coc[0] - ch[j].coc[0], b = coc[1] - ch[j].coc[1], d = coc[2] - ch[j].coc[2];
    double v = sqrt((a * a + b * b) + d * d) + ch[j].bmax;
    if (j == 0 || v > bmax) bmax = v;
  }
  for (int d = 0; d < 3; ++d) p.coc[d] = coc[d];
  p.q = charge;
  p.absq = absq;
  p.m[0] = dip[0]; p.m[1] = dip[1]; p.m[2] = dip[2];
  p.m[3] = quad[0]; p.m[4] = quad[1]; p.m[5] = quad[2];
  p.m[6] = xy; p.m[7] = yz; p.m[8] = zx;
  p.bmax = bmax;
}

// A number with its derivatives along three directions (forward-mode
// differentiation): the adjoint walk evaluates the 2D Coulomb and
// Lennard-Jones kernels below on D3 offsets to get the fields' derivatives
// with respect to the offset.  Those kernels are templates on the scalar
// type; their double instantiation is the walk's arithmetic, unchanged.
// (the namespace's sqrt / log overloads for D3 must not hide the global ones)
using ::log;
using ::sqrt;
struct D3 {
  double v, g[3];
  __host__ __device__ D3() : v(0.0), g{0.0, 0.0, 0.0} {}
  __host__ __device__ D3(double a) : v(a), g{0.0, 0.0, 0.0} {}
  __host__ __device__ D3(double a, double g0, double g1, double g2) : v(a), g{g0, g1, g2} {}
};
__host__ __device__ __forceinline__ D3 operator+(const D3& a, const D3& b) {
  return D3(a.v + b.v, a.g[0] + b.g[0], a.g[1] + b.g[1], a.g[2] + b.g[2]);
}
__host__ __device__ __forceinline__ D3 operator-(const D3& a, const D3& b) {
  return D3(a.v - b.v, a.g[0] - b.g[0], a.g[1] - b.g[1], a.g[2] - b.g[2]);
}
__host__ __device__ __forceinline__ D3 operator-(const D3& a) {
  return D3(-a.v, -a.g[0], -a.g[1], -a.g[2]);
}
__host__ __device__ __forceinline__ D3 operator*(const D3& a, const D3& b) {
  return D3(a.v * b.v, a.g[0] * b.v + a.v * b.g[0], a.g[1] * b.v + a.v * b.g[1],
            a.g[2] * b.v + a.v * b.g[2]);
}
__host__ __device__ __forceinline__ D3 operator/(const D3& a, const D3& b) {
  const double r = 1.0 / b.v, v = a.v * r;
  return D3(v, (a.g[0] - v * b.g[0]) * r, (a.g[1] - v * b.g[1]) * r, (a.g[2] - v * b.g[2]) * r);
}
__host__ __device__ __forceinline__ D3 operator+(const D3& a, double b) { return a + D3(b); }
__host__ __device__ __forceinline__ D3 operator+(double a, const D3& b) { return D3(a) + b; }
__host__ __device__ __forceinline__ D3 operator-(const D3& a, double b) { return a - D3(b); }
__host__ __device__ __forceinline__ D3 operator-(double a, const D3& b) { return D3(a) - b; }
__host__ __device__ __forceinline__ D3 operator*(const D3& a, double b) {
  return D3(a.v * b, a.g[0] * b, a.g[1] * b, a.g[2] * b);
}
__host__ __device__ __forceinline__ D3 operator*(double a, const D3& b) { return b * a; }
__host__ __device__ __forceinline__ D3 operator/(const D3& a, double b) { return a / D3(b); }
__host__ __device__ __forceinline__ D3 operator/(double a, const D3& b) { return D3(a) / b; }
__host__ __device__ __forceinline__ bool operator>(const D3& a, double b) { return a.v > b; }
__host__ __device__ __forceinline__ D3 sqrt(const D3& a) {
  const double r = ::sqrt(a.v), h = 0.5 / r;
  return D3(r, a.g[0] * h, a.g[1] * h, a.g[2] * h);
}
__host__ __device__ __forceinline__ D3 log(const D3& a) {
  const double r = 1.0 / a.v;
  return D3(::log(a.v), a.g[0] * r, a.g[1] * r, a.g[2] * r);
}

// calc_force_coulomb_2D_direct, coulomb/module_coulomb_kernels.f90:267-279
// (d2 = dx^2 + dy^2 + eps2; E_z = 0)
template <class T>
__host__ __device__ __forceinline__ void force_leaf_2d64(double q, T dx, T dy, T d2, T& ex, T& ey,
                                                         T& ez, T& phi) {
  phi = -((0.5 * q) * log(d2));
  const T rd2charge = q / d2;
  ex = rd2charge * dx;
  ey = rd2charge * dy;
  ez = 0.0;
}

// calc_force_coulomb_2D, coulomb/module_coulomb_kernels.f90:155-195
template <class T>
__host__ __device__ __forceinline__ void force_twig_2d64(double q, const double* m, T dx, T dy,
                                                         T d2, T& ex, T& ey, T& ez, T& phi) {
  const T rd2 = 1.0 / d2, rd4 = rd2 * rd2, rd6 = rd4 * rd2;
  const T dx2 = dx * dx, dy2 = dy * dy, dx3 = dx2 * dx, dy3 = dy2 * dy;
  const double p1 = m[0], p2 = m[1], q1 = m[3], q2 = m[4], qxy = m[6];
  phi = ((((-((0.5 * q) * log(d2))) - ((dx * p1) + (dy * p2)) * rd2) +
          q1 * (((2.0 * dx2) * rd4) - rd2)) +
         q2 * (((2.0 * dy2) * rd4) - rd2)) +
        (((2.0 * qxy) * dx) * dy) * rd4;
  ex = (((((q * dx) * rd2 - p1 * (((2.0 * dx2) * rd4) - rd2)) - (((p2 * 2.0) * dx) * dy) * rd4) +
         q1 * (((8.0 * dx3) * rd6) - ((6.0 * dx) * rd4))) +
        q2 * ((((8.0 * dx) * dy2) * rd6) - ((2.0 * dx) * rd4))) +
       qxy * ((((8.0 * dx2) * dy) * rd6) - ((2.0 * dy) * rd4));
  ey = (((((q * dy) * rd2 - p2 * (((2.0 * dy2) * rd4) - rd2)) - (((p1 * 2.0) * dx) * dy) * rd4) +
         q2 * (((8.0 * dy3) * rd6) - ((6.0 * dy) * rd4))) +
        q1 * ((((8.0 * dy) * dx2) * rd6) - ((2.0 * dy) * rd4))) +
       qxy * ((((8.0 * dy2) * dx) * rd6) - ((2.0 * dx) * rd4));
  ez = 0.0;
}

// calc_force_LJ, coulomb/module_coulomb_kernels.f90:204-235 (r2 unsoftened,
// aii2 = eps2; leaves and twigs alike, phi = 0)
template <class T>
__host__ __device__ __forceinline__ void force_lj64(T dx, T dy, T dz, T r2, double aii2, T& ex,
                                                    T& ey, T& ez, T& phi) {
  const double epsc2 = 0.8 * aii2;
  const T aii2_r2 = (r2 > epsc2) ? T(aii2 / r2) : T(aii2 / epsc2);
  const T aii4_r4 = aii2_r2 * aii2_r2;
  const T flj = 2.0 * (aii4_r4 * aii4_r4) - aii4_r4;
  phi = 0.0;
  const T fljrd = flj / sqrt(r2);
  ex = dx * fljrd;
  ey = dy * fljrd;
  ez = dz * fljrd;
}

// calc_force_kelbg_3D_direct, coulomb/module_coulomb_kernels.f90:286-325:
// tq the target's charge, kinv = kelbg_invsqrttemp, sqrtpi = sqrt(acos(-1));
// dist2 unsoftened
struct KelbgArgs {
  double tq, kinv, sqrtpi;
};
__host__ __device__ __forceinline__ void force_kelbg64(double q, double dx, double dy, double dz,
                                                       double dist2, const KelbgArgs& k,
                                                       double& ex, double& ey, double& ez,
                                                       double& phi) {
  double lambda;
  if (k.tq * q < 0.0) lambda = 1.00027227 * k.kinv;  // e-i
  else if (q > 0.0) lambda = 0.03300355 * k.kinv;    // i-i
  else lambda = 1.41421356 * k.kinv;                 // e-e
  const double r = sqrt(dist2);
  const double rd = 1.0 / r;
  const double rd3 = (rd * rd) * rd;
  const double rol = r / lambda;
  const double ome = 1.0 - exp(-(rol * rol));
  phi = (q * rd) * (ome + (k.sqrtpi * rol) * (1.0 - erf(rol)));
  const double fprefac = (q * rd3) * ome;
  ex = fprefac * dx;
  ey = fprefac * dy;
  ez = fprefac * dz;
}

// calc_force_per_interaction_with_leaf / _with_twig
// (coulomb/module_interaction_specific.f90:314-387) for force_law kLaw
// (3: 3D Coulomb, 2: 2D Coulomb, 4: Lennard-Jones, 5: Kelbg leaves with
// unsoftened Coulomb twigs); dist2 is unsoftened
template <int kLaw>
__host__ __device__ __forceinline__ void law_leaf64(double q, double dx, double dy, double dz,
                                                    double dist2, double eps2, double& ex,
                                                    double& ey, double& ez, double& phi,
                                                    const KelbgArgs& kel = KelbgArgs{0, 0, 0}) {
  if (kLaw == 2) force_leaf_2d64(q, dx, dy, (dx * dx + dy * dy) + eps2, ex, ey, ez, phi);
  else if (kLaw == 4) force_lj64(dx, dy, dz, dist2, eps2, ex, ey, ez, phi);
  else if (kLaw == 5) force_kelbg64(q, dx, dy, dz, dist2, kel, ex, ey, ez, phi);
  else force_leaf64(q, dx, dy, dz, dist2 + eps2, ex, ey, ez, phi);
}
template <int kLaw>
__host__ __device__ __forceinline__ void law_twig64(double q, const double* m, double dx,
                                                    double dy, double dz, double dist2,
                                                    double eps2, double& ex, double& ey,
                                                    double& ez, double& phi) {
  if (kLaw == 2) force_twig_2d64(q, m, dx, dy, (dx * dx + dy * dy) + eps2, ex, ey, ez, phi);
  else if (kLaw == 4) force_lj64(dx, dy, dz, dist2, eps2, ex, ey, ez, phi);
  else if (kLaw == 5) force_twig64(q, m, dx, dy, dz, dist2, ex, ey, ez, phi);
  else force_twig64(q, m, dx, dy, dz, dist2 + eps2, ex, ey, ez, phi);
}

}  // namespace pepcg
