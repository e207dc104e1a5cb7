// tieorder.cu -- the reference's order of equal keys, on the device.
//
// The grow sorts keys with a stable LSD radix sort (grow.cu).  For distinct
// keys that order is the only sorted order, so it equals the reference's.
// Equal keys are another matter.  The reference's local sort
// (sl_pepc/src/core/sort_radix.c:33-119, rs_rec_ip, called from
// sort_radix_ip :122-151 with rhigh 63, rlow 0, width 10) is an in-place MSD
// radix sort: one pass per 10-bit class digit from the top, each pass moving
// the elements into their class regions by cycle-leader exchanges, then a
// recursion into every class of more than 256 elements and a stable insertion
// sort (sort_insert.c) below that.  Equal keys leave it in the order those
// exchanges put them in, which is not their input order, and
// domain_decompose (module_domains.f90:276-307) then shifts the colliding
// keys of the particles in that order.
//
// k_tie_order replays the reference's class passes, only where they decide the
// order of equal keys, and rewrites the permutation on the runs of equal keys.
// It is one block: it returns at once when the sorted keys have no equal
// neighbours (the count comes from k_sorted_keys or k_count_pairs), so the grow
// pays one empty launch.  With ties, the replay covers:
//  * the first class pass over all n elements (every tie lies in it);
//  * then, level by level, only the class ranges that hold two equal keys:
//    ranges of more than 256 elements get the next class pass, smaller ones
//    the insertion sort (stable, so it keeps the order the passes left), and
//    after the last digit (bits 3..0) the range is sorted.
//
// One class pass over a range, as the reference runs it.  Call a position
// foreign when the element there does not belong to the class region that
// contains the position.  The reference visits the regions in class order;
// in region i it takes each foreign element still there and follows a chain:
// carry the element to its class region j, put it on the first foreign slot
// of region j not yet used, pick up the element that was there, and go on
// until an element of class i comes back to fill the slot the chain started
// from.  Elements already in their region never move, and every position
// ahead of a region's fill pointer still holds its original element, so the
// pass depends only on the classes of the foreign slots in position order.
// The replay lists those (fc, fp), lets one thread follow the chains over the
// list (a shared-memory fill pointer per class; the class list in shared memory
// when it fits), recording for each foreign slot the slot whose element moves
// into it (src), and then moves the elements in parallel.  The chains are a
// sequential dependency by nature: the first pass over n elements costs about
// n dependent steps of one thread (tens of ms per million elements), paid
// only by grows whose keys collide.

#include <algorithm>
#include <mutex>

#include "internal.cuh"

namespace pepcg {
namespace {

constexpr int kTieThreads = 1024;
constexpr int kTieMaxClasses = 1024;
constexpr int kTieSmallRange = 256;  // sr_ip_threshold: insertion sort at or below
constexpr int kTieInts = 5 * kTieMaxClasses + 2 + 32 + 8 + 6;  // shared ints (multiple of 4)
constexpr int kTieStaged = 96 * 1024;  // foreign classes staged in shared memory (uint16)
constexpr size_t kTieSmem = (size_t)kTieInts * 4 + (size_t)kTieStaged * 2;

// exclusive scan over the 1024 threads of the block; total to every thread
__device__ __forceinline__ int tie_scan(int v, int* wsum, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int s = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  total = wsum[31];
  const int pre = warp > 0 ? wsum[warp - 1] : 0;
  __syncthreads();
  return pre + x - v;
}

struct TieShared {
  int* cnt;    // [1024] elements per class
  int* start;  // [1025] class region starts in the range
  int* inp;    // [1024] elements already in their region
  int* fst;    // [1025] first foreign slot of each region in the list
  int* ptr;    // [1024] fill pointer of each region (the walk)
  int* wsum;   // [32]
  int* misc;   // [8]
  uint16_t* sfc;
};

// One class pass of rs_rec_ip (sort_radix.c:33-87) over A[off, off + len):
// the arrangement after the pass replaces it.  shift / ncls: the digit.
__device__ void tie_pass(const TieArgs& a, const TieShared& sh, int off, int len, int shift,
                         int ncls) {
  const int tid = threadIdx.x;
  const uint64_t mask = (uint64_t)ncls - 1;
  for (int c = tid; c < ncls; c += kTieThreads) {
    sh.cnt[c] = 0;
    sh.inp[c] = 0;
  }
  __syncthreads();
  // count the elements of every class (sort_radix.c:55)
  for (int p = tid; p < len; p += kTieThreads) {
    const int c = (int)((a.kb[a.A[off + p]] >> shift) & mask);
    a.cl[off + p] = (uint16_t)c;
    atomicAdd(&sh.cnt[c], 1);
  }
  __syncthreads();
  // class regions (sort_radix.c:58-59)
  {
    int tot;
    const int ex = tie_scan(tid < ncls ? sh.cnt[tid] : 0, sh.wsum, tot);
    if (tid < ncls) sh.start[tid] = ex;
    if (tid == 0) sh.start[ncls] = tot;
  }
  __syncthreads();
  // elements already in their region stay where they are
  for (int p = tid; p < len; p += kTieThreads) {
    const int c = a.cl[off + p];
    if (p >= sh.start[c] && p < sh.start[c + 1]) atomicAdd(&sh.inp[c], 1);
  }
  __syncthreads();
  {
    int tot;
    const int ex = tie_scan(tid < ncls ? sh.cnt[tid] - sh.inp[tid] : 0, sh.wsum, tot);
    if (tid < ncls) sh.fst[tid] = ex;
    if (tid == 0) sh.fst[ncls] = tot;
  }
  __syncthreads();
  const int T = sh.fst[ncls];
  // the foreign slots in position order: region r's are [fst[r], fst[r + 1])
  int run = 0;
  for (int b0 = 0; b0 < len; b0 += kTieThreads) {
    const int p = b0 + tid;
    int c = 0, f = 0;
    if (p < len) {
      c = a.cl[off + p];
      f = (p >= sh.start[c] && p < sh.start[c + 1]) ? 0 : 1;
    }
    int tot;
    const int ex = tie_scan(f, sh.wsum, tot);
    if (f) {
      a.fc[off + run + ex] = (uint16_t)c;
      a.fp[off + run + ex] = p;
    }
    run += tot;
  }
  __syncthreads();
  const bool staged = T <= kTieStaged;
  if (staged)
    for (int q = tid; q < T; q += kTieThreads) sh.sfc[q] = a.fc[off + q];
  for (int c = tid; c < ncls; c += kTieThreads) sh.ptr[c] = sh.fst[c];
  __syncthreads();
  // the chains (sort_radix.c:62-84), in the reference's order: regions in
  // class order, each region's remaining foreign slots in position order
  if (tid == 0) {
    const uint16_t* fcl = staged ? sh.sfc : a.fc + off;
    int32_t* src = a.src + off;
    int steps = 0;
    bool bad = false;
    for (int i = 0; i < ncls && !bad; ++i) {
      const int ei = sh.fst[i + 1];
      while (sh.ptr[i] < ei) {
        const int q0 = sh.ptr[i]++;
        int qprev = q0;
        int j = fcl[q0];
        while (j != i) {
          const int q = sh.ptr[j]++;
          // every step fills one foreign slot: the chains end within T steps
          if (q >= sh.fst[j + 1] || ++steps > T) {
            bad = true;
            break;
          }
          src[q] = qprev;
          qprev = q;
          j = fcl[q];
        }
        if (bad) break;
        src[q0] = qprev;
      }
    }
    if (bad) atomicOr(a.status, ST_SORT_REPLAY);
  }
  __syncthreads();
  if (*a.status & ST_SORT_REPLAY) return;
  // move the elements: foreign slot q receives the element of slot src[q]
  for (int q = tid; q < T; q += kTieThreads) {
    const int p = a.fp[off + q];
    a.B[off + p] = a.A[off + a.fp[off + a.src[off + q]]];
  }
  __syncthreads();
  for (int q = tid; q < T; q += kTieThreads) {
    const int p = a.fp[off + q];
    a.A[off + p] = a.B[off + p];
  }
  __syncthreads();
}

// sort_insert_bmask_kernel (sort_insert.c): stable insertion sort of a range
// whose elements share every key bit above the ones still to sort.
__device__ void tie_insertion_sort(const TieArgs& a, int r0, int r1) {
  for (int i = r0 + 1; i < r1; ++i) {
    const int32_t e = a.A[i];
    const uint64_t k = a.kb[e];
    int j = i - 1;
    while (j >= r0 && a.kb[a.A[j]] > k) {
      a.A[j + 1] = a.A[j];
      --j;
    }
    a.A[j + 1] = e;
  }
}

__global__ void __launch_bounds__(kTieThreads, 1) k_tie_order(TieArgs a) {
  if (*a.ndup == 0) return;
  extern __shared__ __align__(16) int tsm[];
  TieShared sh;
  sh.cnt = tsm;
  sh.start = sh.cnt + kTieMaxClasses;
  sh.inp = sh.start + kTieMaxClasses + 1;
  sh.fst = sh.inp + kTieMaxClasses;
  sh.ptr = sh.fst + kTieMaxClasses + 1;
  sh.wsum = sh.ptr + kTieMaxClasses;
  sh.misc = sh.wsum + 32;
  sh.sfc = reinterpret_cast<uint16_t*>(tsm + kTieInts);
  const int tid = threadIdx.x;
  const int n = (int)a.n;
  // keys by input index, the input arrangement, and dpre[i] = the number of
  // equal neighbours (i', i' + 1) with i' < i in the sorted keys
  for (int i = tid; i < n; i += kTieThreads) {
    a.kb[a.sval[i]] = a.skey[i];
    a.A[i] = i;
  }
  {
    int run = 0;
    for (int b0 = 0; b0 < n; b0 += kTieThreads) {
      const int i = b0 + tid;
      const int f = (i + 1 < n && a.skey[i] == a.skey[i + 1]) ? 1 : 0;
      int tot;
      const int ex = tie_scan(f, sh.wsum, tot);
      if (i < n) a.dpre[i] = run + ex;
      run += tot;
    }
    if (tid == 0) a.dpre[n] = run;
  }
  int2* cur = a.seg;
  int2* nxt = a.seg + a.segcap;
  if (tid == 0) cur[0] = make_int2(0, n);  // sort_radix_ip passes the whole array
  __syncthreads();
  int ncur = 1;
  // rhigh = 63 - 10 L, width min(10, rhigh + 1): digits 63..54, ..., 13..4, 3..0
  for (int L = 0; L < 7 && ncur > 0; ++L) {
    const int rhigh = 63 - 10 * L;
    const int width = min(10, rhigh + 1);
    const int shift = rhigh - width + 1;
    const int ncls = 1 << width;
    if (tid == 0) sh.misc[0] = 0;
    __syncthreads();
    for (int s = 0; s < ncur; ++s) {
      const int2 sg = cur[s];
      tie_pass(a, sh, sg.x, sg.y, shift, ncls);
      if (*a.status & ST_SORT_REPLAY) return;
      // the classes that still hold equal keys (sort_radix.c:88-116); after
      // the last digit there is nothing left to sort
      if (shift > 0 && tid < ncls) {
        const int r0 = sg.x + sh.start[tid], r1 = sg.x + sh.start[tid + 1];
        if (r1 - r0 >= 2 && a.dpre[r1 - 1] - a.dpre[r0] > 0) {
          if (r1 - r0 > kTieSmallRange) {
            const int k = atomicAdd(&sh.misc[0], 1);
            if (k < a.segcap) nxt[k] = make_int2(r0, r1 - r0);
            else atomicOr(a.status, ST_SORT_REPLAY);
          } else {
            tie_insertion_sort(a, r0, r1);
          }
        }
      }
      __syncthreads();
    }
    ncur = min(sh.misc[0], (int)a.segcap);
    int2* t = cur;
    cur = nxt;
    nxt = t;
    __syncthreads();
    if (*a.status & ST_SORT_REPLAY) return;
  }
  // every run of equal keys now stands in the reference's order in A
  for (int i = tid; i < n; i += kTieThreads) {
    const bool tie = (a.dpre[i + 1] - a.dpre[i]) > 0 || (i > 0 && a.dpre[i] - a.dpre[i - 1] > 0);
    if (!tie) continue;
    a.sval[i] = a.A[i];
  }
}

__global__ void k_count_pairs(int64_t n, const uint64_t* __restrict__ skey,
                              unsigned long long* npair) {
  unsigned long long c = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i + 1 < n;
       i += (int64_t)gridDim.x * blockDim.x)
    c += skey[i] == skey[i + 1];
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(npair, c);
}

}  // namespace

int64_t tie_segcap(int64_t n) { return n / (kTieSmallRange + 1) + 2; }

bool tie_order_launch(Ctx* c, const TieArgs& a, cudaStream_t s) {
  static std::mutex mu;
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
      if (!cuda_ok(c, cudaFuncSetAttribute(k_tie_order, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kTieSmem), "tie order smem"))
        return false;
      configured[dev] = true;
    }
  }
  COUNT_LAUNCH();
  k_tie_order<<<1, kTieThreads, kTieSmem, s>>>(a);
  return true;
}

void count_pairs_launch(int64_t n, const uint64_t* skey, unsigned long long* npair,
                        cudaStream_t s) {
  COUNT_LAUNCH();
  k_count_pairs<<<std::min<int64_t>((n + 255) / 256, 148 * 8), 256, 0, s>>>(n, skey, npair);
}

}  // namespace pepcg
