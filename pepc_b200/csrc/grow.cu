// grow.cu -- pepc_grow_tree on the device (sm_100a):
//   bounding box -> space-filling-curve keys -> LSD radix sort of (key, index)
//   -> permutation of the particle payload -> duplicate-key fix -> octree from
//   the sorted keys -> upward multipole pass.
// Reference: tree_grow (src/treecode/lpepcsrc/module_tree_grow.f90:37-138).
// Compiled with --fmad=false: the FP64 arithmetic below must equal a plain
// IEEE evaluation of the reference's expressions.

#include <algorithm>
#include <mutex>
#include <utility>
#include <string>

#include "internal.cuh"

namespace pepcg {

namespace {

constexpr int kThreads = 256;

// ---------------------------------------------------------------------------
// Bounding box: box_create (module_box.f90:48-93)
// ---------------------------------------------------------------------------
__global__ void k_bbox_partial(int64_t n, const double* __restrict__ x,
                               const double* __restrict__ y, const double* __restrict__ z,
                               double* __restrict__ part, uint32_t* status) {
  double lo[3] = {INFINITY, INFINITY, INFINITY};
  double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  bool bad = false;
  auto take = [&](double vx, double vy, double vz) {
    const double v[3] = {vx, vy, vz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      bad |= !isfinite(v[d]);
      lo[d] = fmin(lo[d], v[d]);
      hi[d] = fmax(hi[d], v[d]);
    }
  };
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {  // four particles' loads in flight
    double vx[4], vy[4], vz[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      vx[j] = x[i + j * stride];
      vy[j] = y[i + j * stride];
      vz[j] = z[i + j * stride];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) take(vx[j], vy[j], vz[j]);
  }
  for (; i < n; i += stride) take(x[i], y[i], z[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, ST_NONFINITE);
  __shared__ double s[6][kThreads / 32];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  }
  int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    for (int d = 0; d < 3; ++d) {
      s[d][w] = lo[d];
      s[3 + d][w] = hi[d];
    }
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double r = s[threadIdx.x][0];
    for (int k = 1; k < kThreads / 32; ++k)
      r = threadIdx.x < 3 ? fmin(r, s[threadIdx.x][k]) : fmax(r, s[threadIdx.x][k]);
    part[blockIdx.x * 6 + threadIdx.x] = r;
  }
}

// final reduction + margin (module_box.f90:71-84) + boxlength2 (module_tree.f90:196-201)
__global__ void k_bbox_final(int nparts, const double* __restrict__ part, int cubic,
                             double* __restrict__ box) {
  const int lane = threadIdx.x;  // one warp
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int b = lane; b < nparts; b += 32)
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], part[b * 6 + d]);
      hi[d] = fmax(hi[d], part[b * 6 + 3 + d]);
    }
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  if (lane != 0) return;
  if (cubic) {
    double l = fmin(lo[0], fmin(lo[1], lo[2])), h = fmax(hi[0], fmax(hi[1], hi[2]));
    for (int d = 0; d < 3; ++d) {
      lo[d] = l;
      hi[d] = h;
    }
  }
  for (int d = 0; d < 3; ++d) {
    double s = hi[d] - lo[d];
    double mn = lo[d] - s / 10000.0;
    double mx = hi[d] + s / 10000.0;
    box[d] = mn;
    box[3 + d] = mx;
    box[6 + d] = mx - mn;
  }
  double b0 = fmax(box[6], fmax(box[7], box[8]));
  double bl = b0 * b0;
  box[9] = bl;
  for (int l = 1; l <= kMaxLevel; ++l) {
    bl = bl / 4.0;
    box[9 + l] = bl;
  }
}

// ---------------------------------------------------------------------------
// Keys: compute_particle_keys (module_spacefilling.f90:224-257) with
// intcoord_to_key_hilbert3D (:380-440) or the 3D Morton interleave.
// ---------------------------------------------------------------------------
__constant__ int8_t c_G3x[8] = {5, 6, 0, 5, 5, 0, 6, 5};  // :390 exchange
__constant__ int8_t c_G3r[8] = {0, 0, 0, 5, 0, 0, 6, 5};  // :390 reverse

__device__ __forceinline__ uint64_t morton3d(int64_t i0, int64_t i1, int64_t i2) {
  uint64_t key = 1;
#pragma unroll 4
  for (int i = kMaxLevel - 1; i >= 0; --i)
    key = (key << 3) | (uint64_t)((((i2 >> i) & 1) << 2) | (((i1 >> i) & 1) << 1) | ((i0 >> i) & 1));
  return key;
}

// The reference's Hilbert recursion (module_spacefilling.f90:380-440) keeps
// three transformed coordinates; every exchange / reverse step permutes and
// complements their remaining bits, so the transform applied so far is a
// signed permutation of the axes (at most 48 states).  HilbertTable holds, for
// every (state, raw octant of the original coordinates), the key digit and the
// next state, built on the host by running the reference's own exchange and
// reverse rules (hilbert_table() below); one lookup per level then reproduces
// the reference's key bit for bit.
struct HilbertTable {
  uint16_t e[48 * 8];  // digit | next_state << 3
};

// int((v - lo) / s), coord_to_intcoord_with_refinement_length
// (module_spacefilling.f90:218).  The quotient is formed by multiplying with
// the rounded reciprocal rs wherever that cannot change the integer part: the
// product p is within 1.5 * 2^-52 * p of the correctly rounded quotient, so
// their floors agree unless an integer lies within that distance of p; the
// test below leaves a margin (2^-50 * p) and otherwise divides.  The
// difference v - lo is positive (the box has a margin), so the floor is the
// truncation.
__device__ __forceinline__ int64_t quantise(double v, double lo, double s, double rs) {
  const double d = v - lo;
  const double p = d * rs;
  const double f = floor(p);
  const double tol = p * 0x1p-50;
  if (p >= 0.0 && p - f > tol && (f + 1.0) - p > tol) return (int64_t)f;
  return __double2ll_rz(d / s);
}

__global__ void k_keys(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                       const double* __restrict__ z, const double* __restrict__ q,
                       const double* __restrict__ box, int curve, HilbertTable tab,
                       uint64_t* __restrict__ keys, int32_t* __restrict__ idx,
                       double4* __restrict__ packed) {
  __shared__ double sb[9];
  __shared__ uint16_t st[48 * 8];
  __shared__ uint16_t st2[48 * 64];  // two levels per lookup: 6 key bits | next state << 6
  if (threadIdx.x < 3) {
    sb[threadIdx.x] = box[threadIdx.x];
    // s = boxsize / 2**maxlevel (module_spacefilling.f90:238), exact
    sb[3 + threadIdx.x] = box[6 + threadIdx.x] / 1048576.0;
    sb[6 + threadIdx.x] = 1.0 / sb[3 + threadIdx.x];
  }
  for (int i = threadIdx.x; i < 48 * 8; i += blockDim.x) st[i] = tab.e[i];
  __syncthreads();
  for (int t = threadIdx.x; t < 48 * 64; t += blockDim.x) {
    const unsigned e1 = st[(t >> 6) * 8 + ((t >> 3) & 7)];
    const unsigned e2 = st[(e1 >> 3) * 8 + (t & 7)];
    st2[t] = (uint16_t)((((e1 & 7u) << 3) | (e2 & 7u)) | ((e2 >> 3) << 6));
  }
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double xi = x[i], yi = y[i], zi = z[i];
    // the particle, packed in input order for the permutation's gather
    st256(packed + i, make_double4(xi, yi, zi, q ? q[i] : 0.0));
    const int64_t i0 = quantise(xi, sb[0], sb[3], sb[6]);
    const int64_t i1 = quantise(yi, sb[1], sb[4], sb[7]);
    const int64_t i2 = quantise(zi, sb[2], sb[5], sb[8]);
    uint64_t key;
    if (curve == PEPCG_CURVE_MORTON) {
      key = morton3d(i0, i1, i2);
    } else {
      // levels 2p+1 and 2p per lookup, octants (z << 2 | y << 1 | x) of the
      // upper level in bits 3..5 of the index
      const unsigned a = (unsigned)i0, b = (unsigned)i1, c = (unsigned)i2;
      unsigned state = 0;
      uint64_t k = 1;  // the placeholder bit
#pragma unroll
      for (int p = kMaxLevel / 2 - 1; p >= 0; --p) {
        const unsigned ax = (a >> (2 * p)) & 3u, by = (b >> (2 * p)) & 3u, cz = (c >> (2 * p)) & 3u;
        const unsigned o = ((cz & 2u) << 4) | ((by & 2u) << 3) | ((ax & 2u) << 2) |
                           ((cz & 1u) << 2) | ((by & 1u) << 1) | (ax & 1u);
        const unsigned ent = st2[state * 64 + o];
        k = (k << 6) | (ent & 63u);
        state = ent >> 6;
      }
      key = k;
    }
    keys[i] = key;
    idx[i] = (int32_t)i;
  }
}

// ---------------------------------------------------------------------------
// LSD radix sort of (uint64 key, int32 index), stable, digits of 8 or 9 bits.
// Pass = per-block digit histogram -> exclusive scan over (digit, block) ->
// stable scatter (per-bit ballots + block prefix per 256-key row).
// ---------------------------------------------------------------------------
constexpr int kSortRows = 16;                       // rows of 256 keys per block
constexpr int kSortChunk = kSortRows * kThreads;    // 4096 keys per block
constexpr int kMaxDigits = 512;                     // 9-bit digits at most

template <int kBits>
__global__ void k_sort_hist(int64_t n, const uint64_t* __restrict__ keys, int shift,
                            uint32_t* __restrict__ hist, int nblocks) {
  constexpr int D = 1 << kBits;
  __shared__ uint32_t h[D];
  for (int d = threadIdx.x; d < D; d += kThreads) h[d] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kSortChunk;
  uint64_t kr[kSortRows];  // every row's key requested before the first count
#pragma unroll
  for (int r = 0; r < kSortRows; ++r) {
    const int64_t i = base + r * kThreads + threadIdx.x;
    kr[r] = i < n ? keys[i] : 0;
  }
#pragma unroll
  for (int r = 0; r < kSortRows; ++r)
    if (base + r * kThreads + threadIdx.x < n) atomicAdd(&h[(kr[r] >> shift) & (D - 1)], 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < D; d += kThreads) hist[(int64_t)d * nblocks + blockIdx.x] = h[d];
}

// barrier for the first 256 threads of the block only (the digit lanes)
__device__ __forceinline__ void named_barrier_256() {
  asm volatile("bar.sync 1, 256;\n" ::: "memory");
}

// Stable scatter of one 4096-key tile.  Warp w owns the tile's keys
// [256 w, 256 w + 256) and reads their digits in one round (8 per lane,
// coalesced); it ranks them among themselves by digit, in order -- the lanes
// sharing a digit from one ballot per digit bit, the digit's running count in
// shared memory, updated by the peers' leader -- with no block barrier.  The
// per-digit counts are then prefixed over the warps, which keeps the ranks
// stable, and over the digits, which gives each digit's run in the tile.
// The tile is sorted by digit in shared memory (the keys and indices re-read
// from global memory, which keeps the kernel small enough for three blocks
// per SM) and written out in that order, so that consecutive threads store
// consecutive addresses of a digit's run in the output (the run of digit d of
// tile b starts at offs[d * nblocks + b]).  A warp's count of one digit is at
// most 256, so the per-warp counts are 16-bit.
constexpr int kScatterThreads = 512;
constexpr int kWarpsSort = kScatterThreads / 32;
constexpr int kPerWarp = kSortChunk / kWarpsSort;  // 256 keys
template <int kBits>
constexpr int scatter_smem() {
  return kSortChunk * 8 + kSortChunk * 4 + 2 * (1 << kBits) * 4 + kWarpsSort * (1 << kBits) * 2;
}

template <int kBits>
__global__ void __launch_bounds__(kScatterThreads, 3) k_sort_scatter(int64_t n, const uint64_t* __restrict__ kin,
                                                           const int32_t* __restrict__ vin,
                                                           uint64_t* __restrict__ kout,
                                                           int32_t* __restrict__ vout, int shift,
                                                           const uint32_t* __restrict__ offs,
                                                           int nblocks) {
  constexpr int D = 1 << kBits;
  static_assert(D == 256 || D == kScatterThreads, "one digit per prefix thread");
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t wtot[D / 32];
  uint64_t* sk = reinterpret_cast<uint64_t*>(smem);
  int32_t* sv = reinterpret_cast<int32_t*>(sk + kSortChunk);
  uint32_t* lstart = reinterpret_cast<uint32_t*>(sv + kSortChunk);  // tile-local run starts
  uint32_t* gbase = lstart + D;                                     // output run starts
  uint16_t(*wcnt)[D] = reinterpret_cast<uint16_t(*)[D]>(gbase + D);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t base = (int64_t)blockIdx.x * kSortChunk;
  const int cnt = (int)min((int64_t)kSortChunk, n - base);
  if (threadIdx.x < D) gbase[threadIdx.x] = offs[(int64_t)threadIdx.x * nblocks + blockIdx.x];
  for (int i = threadIdx.x; i < kWarpsSort * D; i += kScatterThreads) (&wcnt[0][0])[i] = 0;
  uint16_t dg[kPerWarp / 32];
#pragma unroll
  for (int j = 0; j < kPerWarp / 32; ++j) {
    const int i = warp * kPerWarp + j * 32 + lane;
    dg[j] = i < cnt ? (uint16_t)((kin[base + i] >> shift) & (D - 1)) : 0;
  }
  __syncthreads();
  int rk[kPerWarp / 32];
  uint16_t* my = wcnt[warp];
#pragma unroll
  for (int j = 0; j < kPerWarp / 32; ++j) {
    const bool valid = warp * kPerWarp + j * 32 + lane < cnt;
    const int d = dg[j];
    // the lanes with this lane's digit, from one ballot per digit bit
    unsigned peers = __ballot_sync(0xffffffffu, valid);
    if (!valid) peers = ~peers;
#pragma unroll
    for (int bit = 0; bit < kBits; ++bit) {
      const bool on = (d >> bit) & 1;
      const unsigned m = __ballot_sync(0xffffffffu, on);
      peers &= on ? m : ~m;
    }
    const int leader = __ffs(peers) - 1;
    uint32_t c0 = 0;
    if (valid && lane == leader) c0 = my[d];
    c0 = __shfl_sync(0xffffffffu, c0, leader);
    rk[j] = (int)c0 + __popc(peers & lt);
    if (valid && lane == leader) my[d] = (uint16_t)(c0 + __popc(peers));
    __syncwarp();
  }
  __syncthreads();
  if (threadIdx.x < D) {  // digit threadIdx.x: prefix over the warps, then the tile's run starts
    const int b = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarpsSort; ++w) {
      const uint32_t t = wcnt[w][b];
      wcnt[w][b] = (uint16_t)run;  // at most 4096 - 256: fits
      run += t;
    }
    uint32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wtot[warp] = x;
    if constexpr (D == kScatterThreads) __syncthreads();
    else named_barrier_256();
    uint32_t pre = 0;
    for (int w = 0; w < warp; ++w) pre += wtot[w];
    lstart[b] = pre + x - run;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kPerWarp / 32; ++j) {
    const int i = warp * kPerWarp + j * 32 + lane;
    if (i < cnt) {
      const int d = dg[j];
      const int pos = (int)(lstart[d] + wcnt[warp][d]) + rk[j];
      sk[pos] = kin[base + i];
      sv[pos] = vin[base + i];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < cnt; i += kScatterThreads) {
    const uint64_t k = sk[i];
    const int d = (int)((k >> shift) & (D - 1));
    const uint32_t dst = gbase[d] + (uint32_t)(i - (int)lstart[d]);
    kout[dst] = k;
    vout[dst] = sv[i];
  }
}

// ---------------------------------------------------------------------------
// Exclusive scans (uint32 / int32): reduce per block, then apply (each block
// adding the sums of the blocks before it).
// ---------------------------------------------------------------------------
constexpr int kScanItems = 8;
constexpr int kScanTile = kThreads * kScanItems;  // 2048

template <class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* smem, T& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T s = lane < kThreads / 32 ? smem[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kThreads / 32) smem[lane] = s;
  }
  __syncthreads();
  T wpre = warp > 0 ? smem[warp - 1] : T(0);
  total = smem[kThreads / 32 - 1];
  __syncthreads();
  return wpre + x - v;
}

// One or two arrays of the same length per launch (blockIdx.y picks the
// array); block sums at bsum[blockIdx.y * gridDim.x + blockIdx.x].
template <class T>
struct ScanPair {
  const T* in[2];
  T* out[2];
};

// a thread's kScanItems consecutive values: two 16-byte loads for a full tile
// of an aligned array, else element by element
template <class T>
__device__ __forceinline__ void scan_load(const T* __restrict__ in, int64_t base, int64_t n,
                                          T (&v)[kScanItems]) {
  static_assert(sizeof(T) == 4 && kScanItems == 8, "two 16-byte loads per thread");
  const int64_t i0 = base + (int64_t)threadIdx.x * kScanItems;
  if (base + kScanTile <= n && ((reinterpret_cast<uintptr_t>(in) & 15) == 0)) {
    const int4 a = reinterpret_cast<const int4*>(in + i0)[0];
    const int4 b = reinterpret_cast<const int4*>(in + i0)[1];
    v[0] = (T)a.x; v[1] = (T)a.y; v[2] = (T)a.z; v[3] = (T)a.w;
    v[4] = (T)b.x; v[5] = (T)b.y; v[6] = (T)b.z; v[7] = (T)b.w;
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) v[k] = i0 + k < n ? in[i0 + k] : T(0);
  }
}

template <class T>
__global__ void k_scan_reduce(ScanPair<T> a, int64_t n, T* __restrict__ bsum) {
  __shared__ T sm[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  T v[kScanItems];
  scan_load<T>(blockIdx.y ? a.in[1] : a.in[0], base, n, v);
  T s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) s += v[k];
  T tot;
  block_exclusive_scan<T>(s, sm, tot);
  if (threadIdx.x == 0) bsum[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = tot;
}

// Each block adds the sums of the blocks before it itself (at most a few
// thousand integers, read from L2) instead of a separate single-block scan of
// the block sums: one launch fewer per scan.
template <class T>
__global__ void k_scan_apply(ScanPair<T> a, int64_t n, const T* __restrict__ bsum) {
  __shared__ T sm[32];
  const T* bs = bsum + (int64_t)blockIdx.y * gridDim.x;
  T pre = 0;
  for (int64_t b = threadIdx.x; b < (int64_t)blockIdx.x; b += blockDim.x) pre += bs[b];
  {
    T t;
    block_exclusive_scan<T>(pre, sm, t);
    pre = t;
  }
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  T v[kScanItems];
  scan_load<T>(blockIdx.y ? a.in[1] : a.in[0], base, n, v);
  T s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) s += v[k];
  T tot;
  T ex = block_exclusive_scan<T>(s, sm, tot) + pre;
  T* out = blockIdx.y ? a.out[1] : a.out[0];
  const int64_t i0 = base + (int64_t)threadIdx.x * kScanItems;
  T o[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    o[k] = ex;
    ex += v[k];
  }
  if (base + kScanTile <= n && ((reinterpret_cast<uintptr_t>(out) & 15) == 0)) {
    reinterpret_cast<int4*>(out + i0)[0] = make_int4((int)o[0], (int)o[1], (int)o[2], (int)o[3]);
    reinterpret_cast<int4*>(out + i0)[1] = make_int4((int)o[4], (int)o[5], (int)o[6], (int)o[7]);
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
      if (i0 + k < n) out[i0 + k] = o[k];
  }
}

// exclusive scans of one array, or of two arrays of the same length in the
// same launches (tmp: one block sum per 2048 elements and array)
template <class T>
void exclusive_scan2(const T* in0, T* out0, const T* in1, T* out1, int64_t n, T* tmp,
                     cudaStream_t s) {
  const int64_t nb = (n + kScanTile - 1) / kScanTile;
  ScanPair<T> a{{in0, in1}, {out0, out1}};
  const dim3 grid((unsigned)nb, in1 ? 2u : 1u);
  COUNT_LAUNCH();
  k_scan_reduce<T><<<grid, kThreads, 0, s>>>(a, n, tmp);
  COUNT_LAUNCH();
  k_scan_apply<T><<<grid, kThreads, 0, s>>>(a, n, tmp);
}

template <class T>
void exclusive_scan(const T* in, T* out, int64_t n, T* tmp, cudaStream_t s) {
  exclusive_scan2<T>(in, out, nullptr, nullptr, n, tmp, s);
}

// One LSD pass over digit bits [shift, shift + kBits): histogram, scan of the
// (digit, block) counts, scatter.  hist holds (1 << kBits) * nblocks + 1
// counts; k_sort_scatter needs more than the default 48 KB of dynamic shared
// memory.
template <int kBits>
void sort_pass(int64_t n, const uint64_t* kin, const int32_t* vin, uint64_t* kout, int32_t* vout,
               int shift, uint32_t* hist, uint32_t* scan_tmp, cudaStream_t s) {
  static thread_local int configured_device = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (configured_device != dev) {
    cudaFuncSetAttribute(k_sort_scatter<kBits>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         scatter_smem<kBits>());
    configured_device = dev;
  }
  const int nb = (int)((n + kSortChunk - 1) / kSortChunk);
  COUNT_LAUNCH();
  k_sort_hist<kBits><<<nb, kThreads, 0, s>>>(n, kin, shift, hist, nb);
  exclusive_scan<uint32_t>(hist, hist, (int64_t)(1 << kBits) * nb, scan_tmp, s);
  COUNT_LAUNCH();
  k_sort_scatter<kBits><<<nb, kScatterThreads, scatter_smem<kBits>(), s>>>(n, kin, vin, kout, vout,
                                                                          shift, hist, nb);
}

// ---------------------------------------------------------------------------
// Permute the payload into key order, flag duplicates (module_domains.f90:199-234)
// ---------------------------------------------------------------------------
// The sorted keys (also kept as the keys before the duplicate fix), and the
// positions i with key(i + 1) == key(i).
__global__ void k_sorted_keys(int64_t n, const uint64_t* __restrict__ skey,
                              int64_t* __restrict__ ko, int64_t* __restrict__ korig,
                              unsigned long long* dupcount, int32_t* duplist, int dupcap) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = skey[i];
    ko[i] = (int64_t)k;
    korig[i] = (int64_t)k;
    if (i + 1 < n && skey[i + 1] == k) {
      unsigned long long slot = atomicAdd(dupcount, 1ull);
      if (slot < (unsigned long long)dupcap) duplist[slot] = (int32_t)i;
    }
  }
}

// Particles into key order: one 32-byte gather per particle from the packed
// copy that k_keys wrote, with the charge from qsrc instead when the charges
// arrived after the keys were formed (the host-array grow uploads them while
// the keys are sorted).
__global__ void k_gather(int64_t n, const int32_t* __restrict__ sval,
                         const double4* __restrict__ packed, const double* __restrict__ qsrc,
                         double* __restrict__ xo, double* __restrict__ yo,
                         double* __restrict__ zo, double* __restrict__ qo,
                         int32_t* __restrict__ perm) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t j = sval[i];
    const double4 p = ld256(packed + j);
    xo[i] = p.x;
    yo[i] = p.y;
    zo[i] = p.z;
    qo[i] = qsrc ? qsrc[j] : p.w;
    perm[i] = j;
  }
}

// key_to_intcoord_hilbert, module_spacefilling.f90:501-565
__device__ void key_to_intcoord_hilbert(int64_t key, int64_t ic[3]) {
  const int C3[8] = {0, 1, 3, 2, 6, 7, 5, 4};
  int lev = (63 - __clzll((unsigned long long)key)) / 3;
  ic[0] = ic[1] = ic[2] = 0;
  for (int i = 0; i < lev; ++i) {
    int h = (int)((key >> (3 * i)) & 7);
    int cval = C3[h], rev = c_G3r[h], exch = c_G3x[h];
    if (i > 0) {
      for (int j = 0; j < 3; ++j)
        if ((rev >> j) & 1) ic[j] = (~ic[j]) & ((int64_t(1) << i) - 1);
      for (int j = 0; j < 2; ++j) {
        if (!((exch >> j) & 1)) continue;
        for (int k = j + 1; k < 3; ++k)
          if ((exch >> k) & 1) {
            int64_t t = ic[j]; ic[j] = ic[k]; ic[k] = t;
          }
      }
    }
    for (int j = 0; j < 3; ++j) ic[j] |= (int64_t)((cval >> j) & 1) << i;
  }
  for (int j = 0; j < 3; ++j) ic[j] <<= (kMaxLevel - lev);
}

__device__ void key_to_intcoord_morton(int64_t key, int64_t ic[3]) {
  int lev = (63 - __clzll((unsigned long long)key)) / 3;
  ic[0] = ic[1] = ic[2] = 0;
  for (int i = 0; i < lev; ++i)
    for (int j = 0; j < 3; ++j) ic[j] |= ((key >> (3 * i + j)) & 1) << i;
  for (int j = 0; j < 3; ++j) ic[j] <<= (kMaxLevel - lev);
}

// Duplicate-key fix, module_domains.f90:268-307, executed in the reference's
// sequential order by one thread over the (rare) duplicate positions.  The
// range of positions whose key may have changed goes to range[0..1] for
// k_dupfix_coords.
__global__ void k_dupfix_keys(int64_t n, int64_t* __restrict__ key,
                              const unsigned long long* __restrict__ dupcount,
                              int32_t* __restrict__ duplist, int dupcap,
                              int64_t* __restrict__ range, uint32_t* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long nd = *dupcount;
  if (nd == 0) return;
  if (nd > (unsigned long long)dupcap) {
    atomicOr(status, ST_DUP_OVERFLOW);
    return;
  }
  int m = (int)nd;
  for (int a = 1; a < m; ++a) {  // the atomic append is unordered: insertion sort
    int32_t v = duplist[a];
    int b = a - 1;
    while (b >= 0 && duplist[b] > v) {
      duplist[b + 1] = duplist[b];
      --b;
    }
    duplist[b + 1] = v;
  }
  // key_diffs(i) = key(i+1) - key(i), and key_diffs(npnew) = 1 (last rank)
  auto kd = [&](int64_t i) -> int64_t { return (i >= n - 1) ? 1 : key[i + 1] - key[i]; };
  int64_t lo_changed = n, hi_changed = -1;
  for (int a = 0; a < m; ++a) {
    int64_t i = duplist[a];
    if (kd(i) >= 1) continue;
    int64_t jmax = (n - 1 - i) > (i + 1) ? (n - 1 - i) : (i + 1);
    for (int64_t j = 1; j <= jmax; ++j) {
      int64_t dn = i - j < 0 ? 0 : i - j;
      int64_t up = (i + j < n - 2) ? i + j : n - 2;
      if (kd(dn) > 1) {
        for (int64_t t = (i - j + 1 < 0 ? 0 : i - j + 1); t <= i; ++t) key[t] -= 1;
        lo_changed = min(lo_changed, i - j + 1 < 0 ? (int64_t)0 : i - j + 1);
        hi_changed = max(hi_changed, i);
        break;
      } else if (up >= 0 && kd(up) > 1) {
        int64_t top = (i + j < n - 1) ? i + j : n - 1;
        for (int64_t t = i + 1; t <= top; ++t) key[t] += 1;
        lo_changed = min(lo_changed, i + 1);
        hi_changed = max(hi_changed, top);
        break;
      }
    }
  }
  range[0] = lo_changed;
  range[1] = hi_changed;
}

// The particles whose key the fix changed get the coordinates of their new
// key (key_to_coord, module_spacefilling.f90:445-471); runs after the gather.
__global__ void k_dupfix_coords(int64_t n, const int64_t* __restrict__ key,
                                const int64_t* __restrict__ korig, double* __restrict__ x,
                                double* __restrict__ y, double* __restrict__ z,
                                const unsigned long long* __restrict__ dupcount, int dupcap,
                                const int64_t* __restrict__ range, const double* __restrict__ box,
                                int curve) {
  const unsigned long long nd = *dupcount;
  if (nd == 0 || nd > (unsigned long long)dupcap) return;
  const int64_t lo = range[0], hi = range[1];
  for (int64_t i = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= hi;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (key[i] == korig[i]) continue;
    int64_t ic[3];
    if (curve == PEPCG_CURVE_MORTON) key_to_intcoord_morton(key[i], ic);
    else key_to_intcoord_hilbert(key[i], ic);
    double c[3];
    for (int d = 0; d < 3; ++d) {
      double s = box[6 + d] / 1048576.0;
      c[d] = ((double)ic[d] + 0.5) * s + box[d];
    }
    x[i] = c[0];
    y[i] = c[1];
    z[i] = c[2];
  }
}

// ---------------------------------------------------------------------------
// Octree from sorted, distinct keys.
// LCP(i, i+1) = number of leading octal digits shared (excluding the
// placeholder).  Particle i has its leaf at level
//   lev_i = max(LCP(i-1, i), LCP(i, i+1)) + 1
// (a twig exists for every prefix shared by >= 2 particles and a leaf holds
// one particle, module_tree_grow.f90:646-691), starts the nodes of levels
// LCP(i-1,i)+1 .. lev_i and ends the nodes of levels LCP(i,i+1)+1 .. lev_i.
// Forward-preorder index (the reference's insertion order) of the node that
// particle s starts at level l: S_s + (l - LCP(s-1,s) - 1).  Postorder index
// of the node that particle e ends at level l: E_e + (lev_e - l); the walk
// order RPO is the reverse of the postorder.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lcp_keys(uint64_t a, uint64_t b) {
  uint64_t d = a ^ b;
  if (d == 0) return kMaxLevel;  // identical: unsplittable
  int h = 63 - __clzll((unsigned long long)d);
  return (kMaxLevel - 1) - h / 3;
}

// Particle i starts the nodes of levels lp+1 .. l (l its leaf level); the
// ones below l are twigs (they also hold particle i+1), so the twigs of each
// level are counted here too (lvl[0..20]).
__global__ void k_node_counts(int64_t n, const int64_t* __restrict__ key,
                              int8_t* __restrict__ lev, int8_t* __restrict__ lcpn,
                              int32_t* __restrict__ cstart, int32_t* __restrict__ cend,
                              uint32_t* status, int* maxlev, int32_t* __restrict__ lvl) {
  __shared__ int h[kMaxLevel + 1];
  __shared__ int bmax;
  if (threadIdx.x <= kMaxLevel) h[threadIdx.x] = 0;
  if (threadIdx.x == 0) bmax = 0;
  __syncthreads();
  int mymax = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = (uint64_t)key[i];
    int lp = i > 0 ? lcp_keys((uint64_t)key[i - 1], k) : -1;
    int ln = i + 1 < n ? lcp_keys(k, (uint64_t)key[i + 1]) : -1;
    int l = (lp > ln ? lp : ln) + 1;
    if (l > kMaxLevel) {  // "no more levels", module_tree_grow.f90:671-675
      atomicOr(status, ST_MAXLEVEL);
      l = kMaxLevel;
    }
    lev[i] = (int8_t)l;
    lcpn[i] = (int8_t)ln;
    mymax = max(mymax, l);
    cstart[i] = l - (lp + 1) + 1;
    cend[i] = l - ln;
    for (int L = lp + 1; L < l; ++L) atomicAdd(&h[L], 1);
  }
  // the deepest leaf level: one global atomic per block
  for (int o = 16; o > 0; o >>= 1) mymax = max(mymax, __shfl_xor_sync(0xffffffffu, mymax, o));
  if ((threadIdx.x & 31) == 0 && mymax > 0) atomicMax(&bmax, mymax);
  __syncthreads();
  if (threadIdx.x == 0 && bmax > 0) atomicMax(maxlev, bmax);
  if (threadIdx.x <= kMaxLevel && h[threadIdx.x]) atomicAdd(&lvl[threadIdx.x], h[threadIdx.x]);
}

// The values the host needs before the rest of the tree can be launched,
// into mapped host memory: the node starts of the last particle (scanned and
// its own, their sum is the node count), box and boxlength2, the duplicate
// count, the deepest leaf level, twigs per level and the status word.
__global__ void k_grow_summary(int64_t n, const int32_t* __restrict__ sstart,
                               const int32_t* __restrict__ cstart, const double* __restrict__ box,
                               const unsigned long long* __restrict__ small,
                               const uint32_t* __restrict__ status,
                               const int32_t* __restrict__ lvl, Ctx::GrowSummary* out) {
  const int t = threadIdx.x;
  if (t < 9 + kMaxLevel + 1) out->box[t] = box[t];
  if (t <= kMaxLevel) out->lvl[t] = lvl[t];
  if (t == 0) {
    out->dup_count = small[0];
    out->starts_before_last = sstart[n - 1];
    out->starts_last = cstart[n - 1];
    out->status = *status;
    out->max_level = *reinterpret_cast<const int*>(small + 2);
  }
}

__device__ __forceinline__ int64_t group_end(const int64_t* __restrict__ key, int64_t n,
                                             int64_t from, uint64_t prefix, int sh) {
  // largest j >= from with key[j] >> sh == prefix (key[from] is known to match)
  int64_t step = 1, lo = from;
  while (lo + step < n && ((uint64_t)key[lo + step] >> sh) == prefix) {
    lo += step;
    step <<= 1;
  }
  int64_t hi = lo + step < n ? lo + step : n;  // exclusive bound, key[hi] mismatches or hi == n
  while (hi - lo > 1) {
    int64_t mid = lo + (hi - lo) / 2;
    if (((uint64_t)key[mid] >> sh) == prefix) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_build_nodes(int64_t n, int64_t M, const int64_t* __restrict__ key,
                              const int8_t* __restrict__ lev, const int8_t* __restrict__ lcpn,
                              const int32_t* __restrict__ S, const int32_t* __restrict__ E,
                              const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, const double* __restrict__ q,
                              double4* __restrict__ nc4, int2* __restrict__ meta,
                              int32_t* __restrict__ fpo2rpo, int32_t* __restrict__ rpo2fpo,
                              int32_t* __restrict__ first_part, int32_t* __restrict__ nleaves,
                              int64_t* __restrict__ nkey, int32_t* __restrict__ leafnode) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t ks = (uint64_t)key[s];
    const int ls = lev[s];
    const int Ls = s > 0 ? lcpn[s - 1] + 1 : 0;
    const int64_t Ss = S[s];
    int64_t e = s;
    for (int l = ls; l >= Ls; --l) {
      const int sh = 3 * (kMaxLevel - l);
      const uint64_t prefix = ks >> sh;
      if (l < ls) e = group_end(key, n, e, prefix, sh);
      const int64_t fpo = Ss + (l - Ls);
      const int le = lev[e];
      const int64_t rpo = M - 1 - ((int64_t)E[e] + (le - l));
      const int64_t next_fpo = (e + 1 < n) ? (int64_t)S[e + 1] : M;
      const int64_t size = next_fpo - fpo;
      const bool leaf = (l == ls);
      meta[rpo] = make_int2((int32_t)(rpo + size), l | (leaf ? kLeafFlag : 0));
      fpo2rpo[fpo] = (int32_t)rpo;
      rpo2fpo[rpo] = (int32_t)fpo;
      first_part[rpo] = (int32_t)s;
      nleaves[rpo] = (int32_t)(e - s + 1);
      nkey[rpo] = (int64_t)prefix;
      if (leaf) {
        st256(nc4 + rpo, make_double4(x[s], y[s], z[s], q[s]));
        leafnode[s] = (int32_t)rpo;
      }
    }
  }
}

// links: parent / number of children (twigs) and key-order traversal pointers;
// one node per thread, blocks of 256 nodes, each block also counting its
// twigs and nodes per level for the level lists (bcnt_*[level * nblk + block])
__global__ void __launch_bounds__(256) k_link(int64_t M, const int2* __restrict__ meta,
                       const int32_t* __restrict__ rpo2fpo, const int32_t* __restrict__ fpo2rpo,
                       int2* __restrict__ fwd, int2* __restrict__ fwdf,
                       int32_t* __restrict__ parent,
                       int32_t* __restrict__ nchild, int4* __restrict__ child8,
                       int32_t* __restrict__ bcnt_twig, int32_t* __restrict__ bcnt_all, int nblk) {
  __shared__ int ht[kMaxLevel + 1], ha[kMaxLevel + 1];
  if (threadIdx.x <= kMaxLevel) ht[threadIdx.x] = ha[threadIdx.x] = 0;
  __syncthreads();
  const int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (u < M) {
    int2 mu = meta[u];
    atomicAdd(&ha[mu.y & 0xff], 1);
    if (!(mu.y & kLeafFlag)) atomicAdd(&ht[mu.y & 0xff], 1);
    const bool leaf = (mu.y & kLeafFlag) != 0;
    const int64_t size = (int64_t)mu.x - u;
    const int64_t f = rpo2fpo[u];
    int first = leaf ? (int)M : fpo2rpo[f + 1];
    int after = (f + size >= M) ? (int)M : fpo2rpo[f + size];
    fwd[u] = make_int2(first, after);
    // the same two nodes as forward-preorder indices, the per-tile walk's visiting order
    fwdf[u] = make_int2(leaf ? (int)M : (int)(f + 1), (f + size >= M) ? (int)M : (int)(f + size));
    if (u == 0) parent[0] = -1;
    if (!leaf) {
      int cnt = 0;
      int ch[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
      for (int64_t c = u + 1; c < mu.x; c = meta[c].x) {
        parent[c] = (int32_t)u;
        if (cnt < 8) ch[cnt] = (int)c;
        ++cnt;
      }
      nchild[u] = cnt;
      child8[2 * u] = make_int4(ch[0], ch[1], ch[2], ch[3]);
      child8[2 * u + 1] = make_int4(ch[4], ch[5], ch[6], ch[7]);
    } else {
      nchild[u] = 0;
    }
  }
  __syncthreads();
  if (threadIdx.x <= kMaxLevel) {
    bcnt_twig[(int64_t)threadIdx.x * nblk + blockIdx.x] = ht[threadIdx.x];
    bcnt_all[(int64_t)threadIdx.x * nblk + blockIdx.x] = ha[threadIdx.x];
  }
}

// Twigs grouped by level for the upward pass and the adjoint's downward pass.
// lvl[0..20] counts the twigs of each level (k_node_counts); twiglist holds,
// level after level, the RPO indices of that level's twigs in increasing
// order.  The same ordering of all nodes gives every node a position in the
// level-ordered records drec (level after level, RPO order within a level).
// A twig's children are consecutive nodes of the next level in that order (a
// node of level L+1 between two children would lie inside the first child's
// subtree), so the upward pass reads a twig's children as one run of the
// level-ordered records: child slot k (child8 order) sits at the position of
// slot 0 plus k.
//
// Built from per-block counts of each level's twigs and nodes, exclusive
// scans over (level, block) in level-major order -- level L then starts
// after everything above it -- and a stable scatter.
__device__ __forceinline__ int level_base(const int32_t* lvl, int level) {
  int b = 0;
  for (int l = 0; l < level; ++l) b += lvl[l];
  return b;
}

// rank of this lane among the block's lanes with the same key (-1: none),
// in block order, plus the warp-level prefix held in wc[warp][key]
__device__ __forceinline__ int block_rank(int key, int warp, int lane, int (*wc)[kMaxLevel + 1]) {
  // the lanes with this lane's key (-1 .. 20), from one ballot per bit of key + 1
  const int kk = key + 1;
  unsigned peers = 0xffffffffu;
#pragma unroll
  for (int bit = 0; bit < 5; ++bit) {
    const bool on = (kk >> bit) & 1;
    const unsigned m = __ballot_sync(0xffffffffu, on);
    peers &= on ? m : ~m;
  }
  const int lrank = __popc(peers & ((1u << lane) - 1u));
  if (key >= 0 && lane == __ffs(peers) - 1) wc[warp][key] = __popc(peers);
  return lrank;
}

__device__ __forceinline__ void warp_prefix(int (*wc)[kMaxLevel + 1]) {
  if (threadIdx.x <= kMaxLevel) {  // exclusive prefix over the warps, level threadIdx.x
    int run = 0;
    for (int w = 0; w < 256 / 32; ++w) {
      const int t = wc[w][threadIdx.x];
      wc[w][threadIdx.x] = run;
      run += t;
    }
  }
}

// Also writes every leaf's level-ordered record (centre and charge from nc4,
// (abs_charge, bmax) = (|q|, 0)), and for the twig at list position P its
// child count and leaf mask with its own position (tinfo[P]), and its child
// and twig-child counts (ccnt[P], tcnt[P]).  Scanned over the twig list, the
// counts give the position of the twig's first child in the level order and
// of its first twig child in the twig list: every node but the root has one
// parent, so the scan at P counts the nodes (twigs) of levels 1 .. L and the
// children of the level-L twigs before P, one short of the position.
__global__ void __launch_bounds__(256) k_level_scatter(int64_t M, const int2* __restrict__ meta,
                                                       const int32_t* __restrict__ bofs_twig,
                                                       const int32_t* __restrict__ bofs_all,
                                                       int nblk, int32_t* __restrict__ twiglist,
                                                       const double4* __restrict__ nc4,
                                                       LevelRecord* __restrict__ drec,
                                                       int32_t* __restrict__ lvlpos,
                                                       const int4* __restrict__ child8,
                                                       const int32_t* __restrict__ nchild,
                                                       int2* __restrict__ tinfo,
                                                       int32_t* __restrict__ ccnt,
                                                       int32_t* __restrict__ tcnt) {
  __shared__ int wt[256 / 32][kMaxLevel + 1], wa[256 / 32][kMaxLevel + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x < (256 / 32) * (kMaxLevel + 1)) {
    (&wt[0][0])[threadIdx.x] = 0;
    (&wa[0][0])[threadIdx.x] = 0;
  }
  const int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int L = -1, end = 0;
  bool leaf = false;
  if (u < M) {
    const int2 mu = meta[u];
    L = mu.y & 0xff;
    leaf = (mu.y & kLeafFlag) != 0;
    end = mu.x;
  }
  __syncthreads();
  const int rt = block_rank(leaf ? -1 : L, warp, lane, wt);
  const int ra = block_rank(L, warp, lane, wa);
  __syncthreads();
  warp_prefix(wt);
  warp_prefix(wa);
  __syncthreads();
  if (L < 0) return;
  const int p = bofs_all[(int64_t)L * nblk + blockIdx.x] + wa[warp][L] + ra;
  lvlpos[u] = p;
  if (!leaf) {
    const int P = bofs_twig[(int64_t)L * nblk + blockIdx.x] + wt[warp][L] + rt;
    twiglist[P] = (int32_t)u;
    // child slot k is a leaf when the next child (or the subtree's end)
    // starts right after it
    const int4 c0 = child8[2 * u], c1 = child8[2 * u + 1];
    const int ch[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    const int nc = min(8, nchild[u]);
    unsigned lm = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k < nc && (k + 1 < nc ? ch[k + 1] : end) == ch[k] + 1) lm |= 1u << k;
    tinfo[P] = make_int2(nc | (int)(lm << 8), p);
    ccnt[P] = nc;
    tcnt[P] = nc - __popc(lm);
  } else {
    // the record as two 256-bit stores: (centre, charge), then (|charge|,
    // bmax = 0) and the links (first child 0, level | leaf flag, 1 leaf, u)
    const double4 a = ld256(nc4 + u);
    st256(drec + p, a);
    st256(reinterpret_cast<double*>(drec + p) + 4,
          make_double4(fabs(a.w), 0.0, __hiloint2double(L | kLeafFlag, 0),
                       __hiloint2double((int)u, 1)));
  }
}

// Upward pass: tree_node_update_from_children / shift_multipoles_up
// (module_tree_grow.f90:762-821, coulomb/module_interaction_specific.f90:84-140),
// level-synchronous: one launch per level, deepest first; every child of a
// level-L twig was finished by an earlier launch, so there are no fences and
// no atomics.  One thread per twig, in the level's RPO order; every sum runs
// over the children in key order (child slot k = nc-1 .. 0, slot 0 being the
// last child) with the reference's operations in its order (no contraction:
// this file is compiled with --fmad=false).
//
// Memory: a twig's own data (twig list, tinfo, scanned counts) is read at
// its list position; its children's records from the level-ordered copy
// (drec: consecutive threads read consecutive runs), and its twig children's
// nine moments from dmom at their twig-list positions (kDmomStride doubles
// each), likewise consecutive for consecutive parents.  The kernel is bound by
// its count of scattered memory instructions (each warp load touches ~10
// sectors), so the children are read in two passes (the sums that give the
// centre, then the shifted moments; the second pass re-reads from L1 rather
// than holding eight records in registers), centres as single 256-bit loads.
// The twig writes its record both to the RPO arrays the walks read (nc4, mom,
// mom32: whole sectors, 256-bit stores) and to the level-ordered copy its
// parent will read.
constexpr int kUpThreads = 128;

__global__ void __launch_bounds__(kUpThreads) k_upward_level(
    int level, const int32_t* __restrict__ lvl, const int32_t* __restrict__ twiglist,
    const int2* __restrict__ tinfo, const int32_t* __restrict__ cfirst,
    const int32_t* __restrict__ tfirst, const int32_t* __restrict__ nleaves,
    LevelRecord* __restrict__ drec, double* __restrict__ dmom, double4* __restrict__ nc4,
    double* __restrict__ mom, float4* __restrict__ mom32) {
  const int cnt = lvl[level];
  const int base = level_base(lvl, level);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int P = base + i;
    const int64_t u = twiglist[P];
    const int2 ti = tinfo[P];
    const int nc = ti.x & 0xff;
    const unsigned lm = (unsigned)ti.x >> 8;  // leaf children, by slot
    const int pu = ti.y;
    const int cs = cfirst[P] + 1;  // level-order position of child slot 0
    const int ts = tfirst[P] + 1;  // twig-list position of the first twig child
    // the twig children's moments are one run of dmom: into L1 now, so the
    // second pass does not wait for them after the first
    {
      const int ntc = nc - __popc(lm);
      const uintptr_t b0 = reinterpret_cast<uintptr_t>(dmom + kDmomStride * (int64_t)ts);
      const uintptr_t b1 = reinterpret_cast<uintptr_t>(dmom + kDmomStride * (int64_t)(ts + ntc));
      for (uintptr_t a = b0 & ~(uintptr_t)127; ntc > 0 && a < b1; a += 128)
        asm volatile("prefetch.global.L1 [%0];" ::"l"(a));
    }
    const int32_t nlv = nleaves[u];
    const LevelRecord* rc = drec + cs;
    // one pass over the children for the charge, the |charge| and both
    // centre-of-charge candidates (abs_charge-weighted, and the plain mean
    // used when the |charge| sum is 0): each sum keeps its own order
    double charge = 0.0, absq = 0.0;
    double wx = 0.0, wy = 0.0, wz = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
    for (int k = 7; k >= 0; --k) {
      if (k < nc) {
        const double4 a = ld256(&rc[k].pos);
        const double b = rc[k].ab.x;
        charge = charge + a.w;
        absq = absq + b;
        wx = wx + a.x * b;
        wy = wy + a.y * b;
        wz = wz + a.z * b;
        gx = gx + a.x;
        gy = gy + a.y;
        gz = gz + a.z;
      }
    }
    double cx, cy, cz;
    if (absq != 0.0) {
      cx = wx / absq;
      cy = wy / absq;
      cz = wz / absq;
    } else {
      cx = gx / (double)nc;
      cy = gy / (double)nc;
      cz = gz / (double)nc;
    }
    double d0 = 0, d1 = 0, d2 = 0, q0 = 0, q1 = 0, q2 = 0, xy = 0, yz = 0, zx = 0;
    double bmax = 0.0;
#pragma unroll
    for (int k = 7; k >= 0; --k) {
      if (k < nc) {
        const bool lf = (lm >> k) & 1u;
        const double2* src = reinterpret_cast<const double2*>(
            dmom + kDmomStride * (int64_t)(ts + __popc(~lm & ((1u << k) - 1u))));
        double m[10];
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          const double2 v = lf ? make_double2(0.0, 0.0) : src[j];
          m[2 * j] = v.x;
          m[2 * j + 1] = v.y;
        }
        const double4 a = ld256(&rc[k].pos);
        const double s0 = cx - a.x, s1 = cy - a.y, s2 = cz - a.z;
        const double q = a.w;
        d0 = (d0 + m[0]) + q * s0;
        d1 = (d1 + m[1]) + q * s1;
        d2 = (d2 + m[2]) + q * s2;
        q0 = ((q0 + m[3]) + m[0] * s0) + (0.5 * q) * (s0 * s0);
        q1 = ((q1 + m[4]) + m[1] * s1) + (0.5 * q) * (s1 * s1);
        q2 = ((q2 + m[5]) + m[2] * s2) + (0.5 * q) * (s2 * s2);
        xy = (((xy + m[6]) + m[0] * s1) + m[1] * s0) + (q * s0) * s1;
        yz = (((yz + m[7]) + m[1] * s2) + m[2] * s1) + (q * s1) * s2;
        zx = (((zx + m[8]) + m[2] * s0) + m[0] * s2) + (q * s2) * s0;
        const double v = sqrt((s0 * s0 + s1 * s1) + s2 * s2) + rc[k].ab.y;
        if (k == nc - 1 || v > bmax) bmax = v;
      }
    }
    const double4 c4 = make_double4(cx, cy, cz, charge);
    st256(nc4 + u, c4);
    LevelRecord* rp = drec + pu;
    st256(&rp->pos, c4);
    rp->ab = make_double2(absq, bmax);
    rp->link = make_int4(cs, level | (nc << 16), nlv, (int)u);
    double* o = mom + kMomStride * u;
    st256(o, make_double4(d0, d1, d2, q0));
    st256(o + 4, make_double4(q1, q2, xy, yz));
    st256(o + 8, make_double4(zx, absq, bmax, 0.0));
    double2* od = reinterpret_cast<double2*>(dmom + kDmomStride * (int64_t)P);
    od[0] = make_double2(d0, d1);
    od[1] = make_double2(d2, q0);
    od[2] = make_double2(q1, q2);
    od[3] = make_double2(xy, yz);
    od[4] = make_double2(zx, 0.0);
    // FP32 copy for the mixed walk, the quadrupole matrix M (off-diagonals
    // halved) scaled by 3: (px, py, pz, 3qxx), (3qyy, 3qzz, 1.5qxy, 1.5qyz),
    // (1.5qzx, qxx+qyy+qzz, charge, 0), padded to a whole 64-byte record
    float4* m4 = mom32 + kMom32Stride * u;
    st256f(m4, make_float4((float)d0, (float)d1, (float)d2, (float)(3.0 * q0)),
           make_float4((float)(3.0 * q1), (float)(3.0 * q2), (float)(1.5 * xy), (float)(1.5 * yz)));
    st256f(m4 + 2, make_float4((float)(1.5 * zx), (float)((q0 + q1) + q2), (float)charge, 0.f),
           make_float4(0.f, 0.f, 0.f, 0.f));
  }
}

// The reference's exchange / reverse rules (module_spacefilling.f90:389-438)
// applied to a (permutation, flip) state: slot j of the transformed
// coordinates holds original axis perm[j], complemented when flip bit j is set.
HilbertTable hilbert_table() {
  static const int CI3[8] = {0, 1, 3, 2, 7, 6, 4, 5};
  static const int G3x[8] = {5, 6, 0, 5, 5, 0, 6, 5};
  static const int G3r[8] = {0, 0, 0, 5, 0, 0, 6, 5};
  static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  auto pidx = [&](const int* p) {
    for (int k = 0; k < 6; ++k)
      if (perms[k][0] == p[0] && perms[k][1] == p[1] && perms[k][2] == p[2]) return k;
    return 0;
  };
  HilbertTable t{};
  for (int pi = 0; pi < 6; ++pi)
    for (int f = 0; f < 8; ++f)
      for (int o = 0; o < 8; ++o) {
        const int r[3] = {o & 1, (o >> 1) & 1, (o >> 2) & 1};
        int b[3];
        for (int j = 0; j < 3; ++j) b[j] = r[perms[pi][j]] ^ ((f >> j) & 1);
        const int cval = (b[2] << 2) | (b[1] << 1) | b[0];
        const int h = CI3[cval];
        int p2[3] = {perms[pi][0], perms[pi][1], perms[pi][2]};
        int fl[3] = {f & 1, (f >> 1) & 1, (f >> 2) & 1};
        if (G3x[h] == 5) {
          std::swap(p2[0], p2[2]);
          std::swap(fl[0], fl[2]);
        } else if (G3x[h] == 6) {
          std::swap(p2[1], p2[2]);
          std::swap(fl[1], fl[2]);
        }
        for (int j = 0; j < 3; ++j) fl[j] ^= (G3r[h] >> j) & 1;
        const int nf = fl[0] | (fl[1] << 1) | (fl[2] << 2);
        const int ns = pidx(p2) * 8 + nf;
        t.e[(pi * 8 + f) * 8 + o] = (uint16_t)(h | (ns << 3));
      }
  return t;
}

inline unsigned grid_for(int64_t n, int threads = kThreads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 64) b = 148 * 64;
  if (b < 1) b = 1;
  return (unsigned)b;
}

}  // namespace

void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, int32_t* tmp,
                        cudaStream_t s) {
  exclusive_scan<int32_t>(in, out, n, tmp, s);
}

// The LSD radix sort of the n (key, index) pairs in skey / sval, ping-ponging
// through skey_alt / sval_alt.  Grow keys (placeholder bit 60, key bits 0..59)
// take 7 passes over bits 0..59, any other 64-bit keys 8 passes of 8 bits; the
// result is in skey / sval (after an odd pass count the buffers are swapped).
static void lsd_sort(Ctx* c, int64_t n, bool grow_keys, cudaStream_t s) {
  uint64_t* kin = c->skey.p;
  uint64_t* kout = c->skey_alt.p;
  int32_t* vin = c->sval.p;
  int32_t* vout = c->sval_alt.p;
  uint32_t* tmp = reinterpret_cast<uint32_t*>(c->scan_tmp.p);
  auto swap = [&]() {
    std::swap(kin, kout);
    std::swap(vin, vout);
  };
  if (grow_keys) {
    // bits 0 .. 59 in four passes of 9 bits and three of 8
    for (int shift = 0; shift < 36; shift += 9, swap())
      sort_pass<9>(n, kin, vin, kout, vout, shift, c->hist.p, tmp, s);
    for (int shift = 36; shift < 60; shift += 8, swap())
      sort_pass<8>(n, kin, vin, kout, vout, shift, c->hist.p, tmp, s);
  } else {
    for (int shift = 0; shift < 64; shift += 8, swap())
      sort_pass<8>(n, kin, vin, kout, vout, shift, c->hist.p, tmp, s);
  }
  // an odd pass count leaves the result in the other buffers
  if (kin != c->skey.p) {
    std::swap(c->skey, c->skey_alt);
    std::swap(c->sval, c->sval_alt);
  }
}

// Scratch of the equal-key replay, borrowed from buffers that are idle between
// the sort and the tree build: the other LSD buffers, the tree-count arrays and
// the sort histogram.
static TieArgs tie_args(Ctx* c, int64_t n, const unsigned long long* ndup) {
  TieArgs a{};
  a.n = n;
  a.skey = c->skey.p;
  a.sval = c->sval.p;
  a.ndup = ndup;
  a.kb = c->skey_alt.p;
  a.A = c->cstart.p;
  a.B = c->cend.p;
  a.fp = c->sstart.p;
  a.src = c->send.p;
  a.dpre = c->tiepre.p;
  a.cl = reinterpret_cast<uint16_t*>(c->sval_alt.p);
  a.fc = a.cl + n;
  a.seg = reinterpret_cast<int2*>(c->hist.p);
  a.segcap = tie_segcap(n);
  a.status = c->d_status;
  return a;
}

int grow_device(Ctx* c, int64_t n, const double* dx, const double* dy, const double* dz,
                const double* dq, cudaEvent_t q_ready) {
  cudaStream_t s = c->stream;
  c->has_tree = false;
  if (n < 2) {
    c->err = "pepcg_grow_tree: need at least 2 particles (module_domains.f90:187)";
    return PEPCG_ERR_BAD_ARG;
  }
  if (n > (int64_t)INT32_MAX / 4) {
    c->err = "pepcg_grow_tree: too many particles for 32-bit node indices";
    return PEPCG_ERR_BAD_ARG;
  }
  const int64_t nblk_sort = (n + kSortChunk - 1) / kSortChunk;
  const int dupcap = 1 << 20;
  if (!ensure(c, c->tiepre, n + 1, "tiepre") ||
      !ensure(c, c->x, n, "x") || !ensure(c, c->y, n, "y") || !ensure(c, c->z, n, "z") ||
      !ensure(c, c->q, n, "q") || !ensure(c, c->key, n, "key") || !ensure(c, c->perm, n, "perm") ||
      !ensure(c, c->skey, n, "skey") || !ensure(c, c->skey_alt, n, "skey_alt") ||
      !ensure(c, c->sval, n, "sval") || !ensure(c, c->sval_alt, n, "sval_alt") ||
      !ensure(c, c->hist, kMaxDigits * nblk_sort + 1, "hist") ||
      !ensure(c, c->scan_tmp, 2 * ((kMaxDigits * nblk_sort + n) / 2048 + 64), "scan_tmp") ||
      !ensure(c, c->orig_key, n, "orig_key") || !ensure(c, c->dup_list, dupcap, "dup_list") ||
      !ensure(c, c->lev, n, "lev") || !ensure(c, c->lcpn, n, "lcpn") ||
      !ensure(c, c->cstart, n, "cstart") || !ensure(c, c->cend, n, "cend") ||
      !ensure(c, c->sstart, n, "sstart") || !ensure(c, c->send, n, "send") ||
      !ensure(c, c->leafnode, n, "leafnode") || !ensure(c, c->lvlcnt, 64, "lvlcnt") ||
      !ensure(c, c->packed, n, "packed"))
    return PEPCG_ERR_OOM;

  if (!cuda_ok(c, cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), s), "memset status") ||
      !cuda_ok(c, cudaMemsetAsync(c->d_small, 0, 8 * sizeof(unsigned long long), s), "memset") ||
      !cuda_ok(c, cudaMemsetAsync(c->lvlcnt.p, 0, 64 * sizeof(int32_t), s), "memset lvl"))
    return PEPCG_ERR_CUDA;

  cudaEventRecord(c->ev[0], s);
  // box
  const int nbb = 512;  // the partials buffer holds 6 x 512
  double* part = c->d_part;  // 6 * nbb doubles
  COUNT_LAUNCH();
  k_bbox_partial<<<nbb, kThreads, 0, s>>>(n, dx, dy, dz, part, c->d_status);
  COUNT_LAUNCH();
  k_bbox_final<<<1, 32, 0, s>>>(nbb, part, c->prm.force_cubic_domain, c->d_box);
  // keys
  COUNT_LAUNCH();
  static const HilbertTable htab = hilbert_table();
  k_keys<<<std::min(grid_for(n), 148u * 8u), kThreads, 0, s>>>(n, dx, dy, dz, q_ready ? nullptr : dq,
                                                              c->d_box, c->prm.curve, htab,
                                                              c->skey.p, c->sval.p, c->packed.p);
  cudaEventRecord(c->ev[1], s);
  // sort: 7 LSD passes over the 60 key bits below the placeholder; the result
  // is in skey / sval
  lsd_sort(c, n, true, s);
  uint64_t* kin = c->skey.p;
  int32_t* vin = c->sval.p;
  COUNT_LAUNCH();
  k_sorted_keys<<<grid_for(n), kThreads, 0, s>>>(n, kin, c->key.p, c->orig_key.p, c->d_small,
                                                 c->dup_list.p, dupcap);
  // equal keys in the reference's order (an empty launch when there are none),
  // before the duplicate fix shifts them: the replay rewrites the sorted
  // indices, which the gather below then follows
  {
    TieArgs ta = tie_args(c, n, c->d_small);
    if (!tie_order_launch(c, ta, s)) return PEPCG_ERR_CUDA;
  }
  int64_t* dup_range = reinterpret_cast<int64_t*>(c->d_small + 12);
  COUNT_LAUNCH();
  k_dupfix_keys<<<1, 32, 0, s>>>(n, c->key.p, c->d_small, c->dup_list.p, dupcap, dup_range,
                                 c->d_status);
  cudaEventRecord(c->keys_ev, s);  // keys and sorted indices final: the host grow copies them back
  cudaEventRecord(c->ev[8], s);
  // tree: per-particle node counts and their scans
  COUNT_LAUNCH();
  k_node_counts<<<grid_for(n), kThreads, 0, s>>>(n, c->key.p, c->lev.p, c->lcpn.p, c->cstart.p,
                                                  c->cend.p, c->d_status,
                                                  reinterpret_cast<int*>(c->d_small + 2),
                                                  c->lvlcnt.p);
  exclusive_scan2<int32_t>(c->cstart.p, c->sstart.p, c->cend.p, c->send.p, n, c->scan_tmp.p, s);
  // the host needs the node count M (grid sizes, allocations), the box, the
  // level counts and the status: one kernel writes them to mapped host memory
  COUNT_LAUNCH();
  k_grow_summary<<<1, 64, 0, s>>>(n, c->sstart.p, c->cstart.p, c->d_box, c->d_small, c->d_status,
                                  c->lvlcnt.p, c->d_sum);
  if (!cuda_ok(c, cudaEventRecord(c->sum_ev, s), "grow summary")) return PEPCG_ERR_CUDA;
  cudaEventRecord(c->ev[9], s);
  // the particles into key order run while the host waits for the summary
  if (q_ready && !cuda_ok(c, cudaStreamWaitEvent(s, q_ready, 0), "charges")) return PEPCG_ERR_CUDA;
  COUNT_LAUNCH();
  k_gather<<<grid_for(n), kThreads, 0, s>>>(n, vin, c->packed.p, q_ready ? dq : nullptr, c->x.p,
                                            c->y.p, c->z.p, c->q.p, c->perm.p);
  COUNT_LAUNCH();
  k_dupfix_coords<<<148 * 2, kThreads, 0, s>>>(n, c->key.p, c->orig_key.p, c->x.p, c->y.p, c->z.p,
                                               c->d_small, dupcap, dup_range, c->d_box,
                                               c->prm.curve);
  cudaEventRecord(c->ev[2], s);
  if (!cuda_ok(c, cudaEventSynchronize(c->sum_ev), "grow (keys/sort)")) return PEPCG_ERR_CUDA;
  const Ctx::GrowSummary& gs = *c->h_sum;
  for (int k = 0; k < 9; ++k) c->box[k] = gs.box[k];
  for (int k = 0; k <= kMaxLevel; ++k) c->boxlength2[k] = gs.box[9 + k];
  for (int k = 0; k <= kMaxLevel; ++k) c->lvl_host[k] = gs.lvl[k];
  c->dup_count = (int64_t)gs.dup_count;
  c->max_level = gs.max_level;
  if (gs.status) {
    // the gather and the fix were queued behind the summary: let them finish
    // before the caller reuses the buffers
    cudaStreamSynchronize(s);
    return status_to_code(c, gs.status);
  }
  const int64_t M = (int64_t)gs.starts_before_last + gs.starts_last;
  // every particle starts at most kMaxLevel + 1 nodes
  if (M < 2 || M > (int64_t)(kMaxLevel + 1) * n || M >= (int64_t)INT32_MAX) {
    c->err = "node count out of range";
    return PEPCG_ERR_NODE_POOL;
  }
  if (!ensure(c, c->nc4, M, "nc4") || !ensure(c, c->meta, M, "meta") ||
      !ensure(c, c->fwd, M, "fwd") || !ensure(c, c->fwdf, M, "fwdf") ||
      !ensure(c, c->mom, kMomStride * M, "mom") ||
      !ensure(c, c->mom32, 4 * kMom32Stride * M, "mom32") ||
      !ensure(c, c->parent, M, "parent") || !ensure(c, c->nchild, M, "nchild") ||
      !ensure(c, c->twiglist, M, "twiglist") || !ensure(c, c->first_part, M, "first_part") ||
      !ensure(c, c->nleaves, M, "nleaves") || !ensure(c, c->fpo2rpo, M, "fpo2rpo") ||
      !ensure(c, c->rpo2fpo, M, "rpo2fpo") || !ensure(c, c->nkey, M, "nkey") ||
      !ensure(c, c->child8, 2 * M, "child8"))
    return PEPCG_ERR_OOM;
  COUNT_LAUNCH();
  k_build_nodes<<<grid_for(n), kThreads, 0, s>>>(n, M, c->key.p, c->lev.p, c->lcpn.p, c->sstart.p,
                                                  c->send.p, c->x.p, c->y.p, c->z.p, c->q.p,
                                                  c->nc4.p, c->meta.p, c->fpo2rpo.p, c->rpo2fpo.p,
                                                  c->first_part.p, c->nleaves.p, c->nkey.p,
                                                  c->leafnode.p);
  // the level lists' per-block counts come from k_link: its blocks are the
  // level lists' blocks of 256 nodes
  const unsigned gM = (unsigned)((M + kThreads - 1) / kThreads);
  const size_t nlb = (size_t)(kMaxLevel + 1) * gM;
  const int64_t ntw = M - n;
  if (!ensure(c, c->lvlblk, 2 * nlb, "level blocks") ||
      !ensure(c, c->drec, M, "level records") || !ensure(c, c->lvlpos, M, "level positions") ||
      !ensure(c, c->dmom, kDmomStride * ntw, "dmom") ||
      !ensure(c, c->tinfo, ntw, "twig info") || !ensure(c, c->tcounts, 2 * ntw, "twig counts") ||
      // block sums of the paired scans below
      !ensure(c, c->scan_tmp, 2 * (std::max<int64_t>((int64_t)nlb, ntw) / kScanTile + 2), "scan_tmp"))
    return PEPCG_ERR_OOM;
  int32_t* bt = c->lvlblk.p;
  int32_t* ba = c->lvlblk.p + nlb;
  COUNT_LAUNCH();
  k_link<<<gM, kThreads, 0, s>>>(M, c->meta.p, c->rpo2fpo.p, c->fpo2rpo.p, c->fwd.p, c->fwdf.p,
                                 c->parent.p, c->nchild.p, c->child8.p, bt, ba, (int)gM);
  cudaEventRecord(c->ev[3], s);
  // twigs by level, then one launch per level, sized by the level's twig
  // count; the deepest twig level is one above the deepest leaf level
  {
    exclusive_scan2<int32_t>(bt, bt, ba, ba, (int64_t)nlb, c->scan_tmp.p, s);
    COUNT_LAUNCH();
    int32_t* cc = c->tcounts.p;
    int32_t* tcn = c->tcounts.p + ntw;
    k_level_scatter<<<gM, kThreads, 0, s>>>(M, c->meta.p, bt, ba, (int)gM, c->twiglist.p,
                                            c->nc4.p, c->drec.p, c->lvlpos.p, c->child8.p,
                                            c->nchild.p, c->tinfo.p, cc, tcn);
    exclusive_scan2<int32_t>(cc, cc, tcn, tcn, ntw, c->scan_tmp.p, s);
    float4* m32 = reinterpret_cast<float4*>(c->mom32.p);
    for (int L = c->max_level - 1; L >= 0; --L) {
      const int64_t cnt = c->lvl_host[L];
      if (cnt <= 0) continue;
      COUNT_LAUNCH();
      k_upward_level<<<grid_for(cnt, kUpThreads), kUpThreads, 0, s>>>(
          L, c->lvlcnt.p, c->twiglist.p, c->tinfo.p, cc, tcn, c->nleaves.p, c->drec.p, c->dmom.p, c->nc4.p,
          c->mom.p, m32);
    }
  }
  cudaEventRecord(c->ev[4], s);
  if (!cuda_ok(c, cudaGetLastError(), "grow kernels")) return PEPCG_ERR_CUDA;
  c->n = n;
  c->nnodes = M;
  c->ntwig = M - n;

  c->has_tree = true;
  return PEPCG_OK;
}

// The local key sort alone (slsort_keys at one rank, sl_pepc/mpi_pepckeys.c:
// 151-167 -> pepckeys_sort_radix, sort_radix.c:122-151): the LSD passes of the
// grow, then the replay of the reference's order on runs of equal keys.
namespace {
__global__ void k_sortkeys_load(int64_t n, const int64_t* __restrict__ in,
                                uint64_t* __restrict__ k, int32_t* __restrict__ v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    k[i] = (uint64_t)in[i];
    v[i] = (int32_t)i;
  }
}

__global__ void k_sortkeys_store(int64_t n, const uint64_t* __restrict__ k,
                                 const int32_t* __restrict__ v, int64_t* __restrict__ kout,
                                 int64_t* __restrict__ pout) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (kout) kout[i] = (int64_t)k[i];
    if (pout) pout[i] = (int64_t)v[i];
  }
}
}  // namespace

int sort_keys_device(Ctx* c, int64_t n, const int64_t* d_in, int64_t* d_kout, int64_t* d_pout) {
  cudaStream_t s = c->stream;
  if (n < 0 || n > (int64_t)INT32_MAX / 4) {
    c->err = "pepcg_sort_keys: n out of range";
    return PEPCG_ERR_BAD_ARG;
  }
  if (n == 0) return PEPCG_OK;
  const int64_t nblk_sort = (n + kSortChunk - 1) / kSortChunk;
  if (!ensure(c, c->skey, n, "skey") || !ensure(c, c->skey_alt, n, "skey_alt") ||
      !ensure(c, c->sval, n, "sval") || !ensure(c, c->sval_alt, n, "sval_alt") ||
      !ensure(c, c->hist, kMaxDigits * nblk_sort + 1, "hist") ||
      !ensure(c, c->scan_tmp, 2 * ((kMaxDigits * nblk_sort + n) / 2048 + 64), "scan_tmp") ||
      !ensure(c, c->cstart, n, "cstart") || !ensure(c, c->cend, n, "cend") ||
      !ensure(c, c->sstart, n, "sstart") || !ensure(c, c->send, n, "send") ||
      !ensure(c, c->tiepre, n + 1, "tiepre"))
    return PEPCG_ERR_OOM;
  unsigned long long* npair = c->d_small + 11;
  if (!cuda_ok(c, cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), s), "memset status") ||
      !cuda_ok(c, cudaMemsetAsync(npair, 0, sizeof(unsigned long long), s), "memset"))
    return PEPCG_ERR_CUDA;
  COUNT_LAUNCH();
  k_sortkeys_load<<<grid_for(n), kThreads, 0, s>>>(n, d_in, c->skey.p, c->sval.p);
  lsd_sort(c, n, false, s);
  count_pairs_launch(n, c->skey.p, npair, s);
  if (!tie_order_launch(c, tie_args(c, n, npair), s)) return PEPCG_ERR_CUDA;
  COUNT_LAUNCH();
  k_sortkeys_store<<<grid_for(n), kThreads, 0, s>>>(n, c->skey.p, c->sval.p, d_kout, d_pout);
  uint32_t st = 0;
  if (!cuda_ok(c, cudaGetLastError(), "sort kernels") ||
      !cuda_ok(c, cudaMemcpyAsync(&st, c->d_status, 4, cudaMemcpyDeviceToHost, s), "status") ||
      !cuda_ok(c, cudaStreamSynchronize(s), "sort"))
    return PEPCG_ERR_CUDA;
  return st ? status_to_code(c, st) : PEPCG_OK;
}

// Tree export in the reference's insertion (forward preorder) order.
namespace {
__global__ void k_export(int64_t M, const int32_t* __restrict__ fpo2rpo,
                         const int32_t* __restrict__ rpo2fpo, const int2* __restrict__ meta,
                         const int2* __restrict__ fwd, const int32_t* __restrict__ parent,
                         const int64_t* __restrict__ nkey, const double4* __restrict__ nc4,
                         const double* __restrict__ mom,
                         int64_t* okey, int32_t* olevel, int64_t* oleaves, int64_t* odesc,
                         int64_t* oparent, int64_t* ofirst, int64_t* onext, double* omom,
                         const int32_t* __restrict__ first_part, int64_t n) {
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < M;
       f += (int64_t)gridDim.x * blockDim.x) {
    int64_t u = fpo2rpo[f];
    int2 mu = meta[u];
    const bool leaf = mu.y & kLeafFlag;
    const int64_t size = (int64_t)mu.x - u;
    okey[f] = nkey[u];
    olevel[f] = mu.y & 0xff;
    oleaves[f] = 0;  // filled below from the particle range
    odesc[f] = size - 1;
    oparent[f] = parent[u] < 0 ? -1 : rpo2fpo[parent[u]];
    ofirst[f] = leaf ? -1 : f + 1;
    // next sibling: the node after the subtree in forward preorder, if it has the same parent
    int64_t after = f + size;
    int64_t nxt = -1;
    if (after < M) {
      int64_t ua = fpo2rpo[after];
      if (parent[ua] == parent[u]) nxt = after;
    }
    onext[f] = nxt;
    double4 a = nc4[u];
    double* o = omom + 15 * f;
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    if (leaf) {
      o[4] = fabs(a.w);
      for (int k = 5; k < 15; ++k) o[k] = 0.0;
    } else {
      const double* m = mom + kMomStride * u;
      o[4] = m[kMomAbs];
      for (int k = 0; k < 9; ++k) o[5 + k] = m[k];
      o[14] = m[kMomBmax];
    }
    // leaves = particles in the node's range: from the first particle of this
    // node to the first particle of the node after the subtree
    int64_t p0 = first_part[u];
    int64_t p1 = after < M ? (int64_t)first_part[fpo2rpo[after]] : n;
    oleaves[f] = p1 - p0;
  }
}
}  // namespace

int export_tree(Ctx* c, int64_t* key, int32_t* level, int64_t* leaves, int64_t* desc,
                int64_t* parent, int64_t* first_child, int64_t* next_sibling, double* mom15) {
  const int64_t M = c->nnodes;
  cudaStream_t s = c->stream;
  size_t bytes = M * (8 * 6 + 4 + 15 * 8);
  char* d = nullptr;
  if (!cuda_ok(c, cudaMallocAsync((void**)&d, bytes, s), "export alloc")) return PEPCG_ERR_OOM;
  int64_t* dk = (int64_t*)d;
  int64_t* dl = dk + M;
  int64_t* dd = dl + M;
  int64_t* dp = dd + M;
  int64_t* df = dp + M;
  int64_t* dn = df + M;
  double* dm = (double*)(dn + M);
  int32_t* dlev = (int32_t*)(dm + 15 * M);
  COUNT_LAUNCH();
  k_export<<<grid_for(M), kThreads, 0, s>>>(M, c->fpo2rpo.p, c->rpo2fpo.p, c->meta.p, c->fwd.p,
                                            c->parent.p, c->nkey.p, c->nc4.p, c->mom.p,
                                            dk, dlev, dl, dd, dp, df, dn, dm, c->first_part.p, c->n);
  bool ok = true;
  auto cp = [&](void* h, const void* dv, size_t b) {
    if (h) ok = ok && cuda_ok(c, cudaMemcpyAsync(h, dv, b, cudaMemcpyDeviceToHost, s), "export");
  };
  cp(key, dk, 8 * M);
  cp(level, dlev, 4 * M);
  cp(leaves, dl, 8 * M);
  cp(desc, dd, 8 * M);
  cp(parent, dp, 8 * M);
  cp(first_child, df, 8 * M);
  cp(next_sibling, dn, 8 * M);
  cp(mom15, dm, 8 * 15 * M);
  cudaFreeAsync(d, s);
  if (!ok || !cuda_ok(c, cudaStreamSynchronize(s), "export")) return PEPCG_ERR_CUDA;
  return PEPCG_OK;
}

}  // namespace pepcg

// ---------------------------------------------------------------------------
// Allocation-free key sort.
//
// Some callers cannot allocate device memory at the time they need the sort:
// a Fortran or C frontend that runs inside another code's memory pool with
// cudaMalloc forbidden, code that must not change the device's memory
// footprint between steps, or a caller that runs where allocating would
// synchronise the device.  pepcg_sort_keys_noalloc serves them: it runs the
// same LSD radix sort passes as pepcg_grow_tree (k_sort_hist /
// k_sort_scatter / the exclusive scans above) with every scratch buffer taken
// from the file-scope array below, and never calls cudaMalloc, cudaFree or an
// allocating library routine.
//
// Limits and sharing:
//  * at most kNoAllocMaxKeys keys per call (larger n is rejected);
//  * the array lives on every GPU that loads this library until the process
//    exits (about 24.3 MB per device);
//  * all calls share the array, and it keeps the last call's contents; every
//    scratch word a call reads is written by that same call first, so nothing
//    needs clearing, but calls that overlap on the GPU (two streams, two host
//    threads, or a call issued before the previous one finished) race on it;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (host code only holds a host-side stand-in for the
//    symbol) and keeps it for the life of the process; make that first call
//    before any stream capture on the device.  A device reset between calls
//    would leave the kept address stale, so it is not supported;
//  * keys are ordered as unsigned 64-bit values and equal keys keep their
//    input order (the LSD passes are stable); pepcg_grow_tree additionally
//    puts equal keys in the reference's order (tieorder.cu).
// ---------------------------------------------------------------------------
namespace pepcg {
namespace {

constexpr int64_t kNoAllocMaxKeys = int64_t(1) << 20;
constexpr int64_t kNoAllocBlocks = kNoAllocMaxKeys / kSortChunk;  // 256
// byte offsets inside the scratch array
constexpr size_t kNaKeysA = 0;
constexpr size_t kNaKeysB = kNaKeysA + 8 * kNoAllocMaxKeys;
constexpr size_t kNaValsA = kNaKeysB + 8 * kNoAllocMaxKeys;
constexpr size_t kNaValsB = kNaValsA + 4 * kNoAllocMaxKeys;
constexpr size_t kNaHist = kNaValsB + 4 * kNoAllocMaxKeys;
constexpr size_t kNaHistBytes = ((4 * (256 * kNoAllocBlocks + 1) + 255) / 256) * 256;
constexpr size_t kNaScan = kNaHist + kNaHistBytes;
constexpr size_t kNaScanBytes = 4 * 1024;
constexpr size_t kNaBytes = kNaScan + kNaScanBytes;

static __device__ __align__(256) unsigned char g_sort_scratch[kNaBytes];

__global__ void k_noalloc_load(int64_t n, const int64_t* __restrict__ in, uint64_t* __restrict__ k,
                               int32_t* __restrict__ v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    k[i] = (uint64_t)in[i];
    v[i] = (int32_t)i;
  }
}

__global__ void k_noalloc_store(int64_t n, const uint64_t* __restrict__ k,
                                const int32_t* __restrict__ v, int64_t* __restrict__ kout,
                                int64_t* __restrict__ pout) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    kout[i] = (int64_t)k[i];
    pout[i] = (int64_t)v[i];
  }
}

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {};

}  // namespace
}  // namespace pepcg

extern "C" int pepcg_sort_keys_noalloc(int64_t n, const int64_t* d_keys_in, int64_t* d_keys_out,
                                       int64_t* d_perm_out, void* stream) {
  using namespace pepcg;
  if (n < 0 || n > kNoAllocMaxKeys) {
    set_static_error("pepcg_sort_keys_noalloc: n = " + std::to_string(n) +
                     " is outside 0.." + std::to_string(kNoAllocMaxKeys) +
                     " (the size of the library's static sort scratch)");
    return PEPCG_ERR_BAD_ARG;
  }
  if (n == 0) return PEPCG_OK;
  if (!d_keys_in || !d_keys_out || !d_perm_out) {
    set_static_error("pepcg_sort_keys_noalloc: null pointer");
    return PEPCG_ERR_BAD_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    set_static_error(std::string("pepcg_sort_keys_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return PEPCG_ERR_CUDA;
  }
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_sort_scratch);
      if (e != cudaSuccess || p == nullptr) {
        set_static_error(std::string("pepcg_sort_keys_noalloc: cudaGetSymbolAddress: ") +
                         cudaGetErrorString(e));
        return PEPCG_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = p;
    }
    base = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint64_t* kin = reinterpret_cast<uint64_t*>(base + kNaKeysA);
  uint64_t* kout = reinterpret_cast<uint64_t*>(base + kNaKeysB);
  int32_t* vin = reinterpret_cast<int32_t*>(base + kNaValsA);
  int32_t* vout = reinterpret_cast<int32_t*>(base + kNaValsB);
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + kNaHist);
  uint32_t* tmp = reinterpret_cast<uint32_t*>(base + kNaScan);
  const int nb = (int)((n + kSortChunk - 1) / kSortChunk);
  COUNT_LAUNCH();
  k_noalloc_load<<<grid_for(n), kThreads, 0, s>>>(n, d_keys_in, kin, vin);
  for (int shift = 0; shift < 64; shift += 8) {
    sort_pass<8>(n, kin, vin, kout, vout, shift, hist, tmp, s);
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  COUNT_LAUNCH();
  k_noalloc_store<<<grid_for(n), kThreads, 0, s>>>(n, kin, vin, d_keys_out, d_perm_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_static_error(std::string("pepcg_sort_keys_noalloc: launch: ") + cudaGetErrorString(e));
    return PEPCG_ERR_CUDA;
  }
  return PEPCG_OK;
}
