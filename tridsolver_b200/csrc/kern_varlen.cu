// Variable-length packed batch (sm_100a): length-bucketed work queues,
// persistent launches.
//
// System s occupies rows [offsets[s], offsets[s+1]) of every array (unit
// stride, int64 offsets).  The preparation sorts the systems into length
// classes, each served by persistent CTAs looping over its list:
//   * at most 256 rows: the short queue, in system order; one warp per
//     system (partitioned Thomas of partition.cuh, the rows-per-lane chunk M
//     picked from the length: 2/4/8, the length buckets), each warp
//     software-pipelined: lane 0 claims the next system while the current one
//     is staged, and the next system's copies go out as soon as the current
//     one's rows are in registers (varlen_short_kernel);
//   * 257 .. 4096 rows: the one-CTA buckets (launch_xcta_varlen,
//     kern_xcta.cu): bucket W lists the systems that need W = ceil(n/512)
//     warps at 16 rows per lane; one persistent launch per bucket, CTA = W
//     warps solving one system at a time, every row read once;
//   * 4097 .. 8192 rows: one CTA of 4 warps per system (varlen_long_kernel):
//     the first half of the system's rows is requested into L2 at once,
//     every warp reduces its 256-row blocks to block rows in shared memory,
//     one warp solves the block system, every warp stages its blocks again
//     (from L2 where they are still there) and finishes them.
// Nothing waits on another CTA.  Rows reach each warp's shared-memory regions
// by coalesced cp.async (row q of the 32*M at q + q/M, conflict-free for the
// lane-per-chunk reads) and leave by coalesced stores.
//
// Three preparation launches (launch_varlen_prep) classify the systems,
// write the short queue (a prefix scan keeps system order) and append the
// others to their lists.  Malformed offsets (decreasing or past `total`) and
// systems longer than 8192 rows are skipped and recorded in the device error
// word (bits 4 and 8).  Every system lands in at most one queue or list, so
// no table index can pass nsys whatever the offsets hold.
//
// Measured on B200 (FP64, 120 M unknowns, lengths log-uniform): 8 .. 256
// rows 3.46 TB/s, 257 .. 1024 4.4-4.7, 1025 .. 4096 4.26, 4097 .. 8192 3.18,
// the whole 8 .. 8192 range 3.48 TB/s algorithmic (200,000 systems: 3.63 TB/s).
// Before the classes (every
// system past 256 rows as 256-row block items reduced, published and
// finished by a second queue across SMs, 72 B moved per unknown) the same
// ranges ran at 1.9, 2.3 and 2.4 TB/s, and 8 .. 8192 at 2.25.
#include <mutex>

#include "partition.cuh"
#include "tma.cuh"

namespace tridb200 {

constexpr int kVLBlock = 256;            // rows per block of a long system (M = 8)
constexpr int kVLShort = kVarlenShort;   // longest system of the short queue
constexpr int kVLMid = 512 * kVarlenCtaBuckets;  // longest system of the one-CTA buckets
constexpr int kVLMaxBlocks = 32;         // longest solvable system: 32 blocks
constexpr int kVLWarps = 8;              // warps per CTA of the short queue
constexpr int kVLBatch = 4;              // short-queue items claimed per atomic
constexpr int kVLLongWarps = 4;          // warps per CTA of the long systems (four CTAs per SM)
constexpr int kVLRegion = 32 * (8 + 1);  // elements per staged array and warp
constexpr int kVLLists = kVarlenCtaBuckets + 1;  // the one-CTA buckets, then the long list
static_assert(kVLLists <= kVarlenClaims && 64 + 4 * (kVarlenClaims + kVLLists) <= 256,
              "list and claim counters fit the 256-byte control block");
constexpr unsigned kErrBadOffsets = 4u;
constexpr unsigned kErrTooLong = 8u;

__device__ __forceinline__ bool vl_bad(int64_t lo, int64_t hi, int64_t total) {
  return hi < lo || lo < 0 || hi > total;
}

// Class of system s: 1 .. kVarlenCtaBuckets the one-CTA bucket (warps of 512
// rows), kClsLong, kClsShort, or nothing to solve (empty, malformed, too long).
enum : int {
  kClsEmpty = 0,
  kClsLong = kVarlenCtaBuckets + 1,  // its list index is kClsLong - 1
  kClsShort,
  kClsTooLong,
  kClsBad
};

__device__ __forceinline__ int vl_class(const int64_t *offsets, int64_t total, int64_t s) {
  const int64_t lo = offsets[s], hi = offsets[s + 1];
  if (vl_bad(lo, hi, total)) return kClsBad;
  const int64_t len = hi - lo;
  if (len == 0) return kClsEmpty;
  if (len <= kVLShort) return kClsShort;
  if (len <= kVLMid) return (int)((len + 511) / 512);
  if (len <= (int64_t)kVLBlock * kVLMaxBlocks) return kClsLong;
  return kClsTooLong;
}

// Preparation, three short launches over the systems (256 per CTA):
//   count: short systems per CTA of systems -> bsum;
//   scan : one CTA, exclusive prefix of bsum; the short total; clears the
//          queue's claim counter and the lists' counters;
//   fill : per system, the short queue entry at its prefix (system order),
//          or its list entry (appended), or its error bit.
constexpr int kPrepThreads = 256;

// inclusive sum over the CTA of v (blockDim.x == kPrepThreads); returns it
__device__ __forceinline__ int64_t vl_cta_scan(int64_t v, int64_t *warp_tot) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) warp_tot[w] = v;
  __syncthreads();
  int64_t add = 0;
  for (int k = 0; k < w; ++k) add += warp_tot[k];
  __syncthreads();
  return v + add;
}

__global__ void __launch_bounds__(kPrepThreads) varlen_prep_count(const int64_t *__restrict__ offsets,
                                                                  int64_t nsys, int64_t total,
                                                                  int64_t *__restrict__ bsum) {
  pdl_enter();
  __shared__ int64_t wt[kPrepThreads / 32];
  const int64_t s = (int64_t)blockIdx.x * kPrepThreads + threadIdx.x;
  const int64_t v = (s < nsys && vl_class(offsets, total, s) == kClsShort) ? 1 : 0;
  const int64_t c = vl_cta_scan(v, wt);
  if (threadIdx.x == kPrepThreads - 1) bsum[blockIdx.x] = c;
}

// ctl[0]: short systems in the queue; ctl[1]: the queue's claim counter
__global__ void __launch_bounds__(1024) varlen_prep_scan(int64_t *__restrict__ bsum, int64_t nblocks,
                                                         int64_t *__restrict__ ctl,
                                                         unsigned *__restrict__ list_count) {
  pdl_enter();
  __shared__ int64_t wt[32];
  const int tid = threadIdx.x;
  const int64_t per = (nblocks + 1023) / 1024;
  const int64_t b0 = tid * per, b1 = (b0 + per < nblocks) ? b0 + per : nblocks;
  int64_t acc = 0;
  for (int64_t b = b0; b < b1; ++b) acc += bsum[b];
  // exclusive prefix of the threads' sums (shuffles within warps, then the
  // warp totals)
  const int64_t incl = vl_cta_scan(acc, wt);
  if (tid == 1023) {
    ctl[0] = incl;
    ctl[1] = 0;
    for (int k = 0; k < kVLLists; ++k) {
      list_count[k] = 0u;
      list_count[kVarlenClaims + k] = 0u;  // the lists' claim counters
    }
  }
  int64_t run = incl - acc;
  for (int64_t b = b0; b < b1; ++b) {
    const int64_t v = bsum[b];
    bsum[b] = run;
    run += v;
  }
}

// lists: kVLLists lists of nsys entries each (a system is listed at most
// once, so no list passes nsys); the short queue holds at most nsys entries
__global__ void __launch_bounds__(kPrepThreads) varlen_prep_fill(
    const int64_t *__restrict__ offsets, int64_t nsys, int64_t total,
    const int64_t *__restrict__ bsum, int *__restrict__ item_sys, int *__restrict__ lists,
    unsigned *__restrict__ list_count, unsigned *__restrict__ err) {
  pdl_enter();
  __shared__ int64_t wt[kPrepThreads / 32];
  const int64_t s = (int64_t)blockIdx.x * kPrepThreads + threadIdx.x;
  const int cls = s < nsys ? vl_class(offsets, total, s) : kClsEmpty;
  const int64_t v = cls == kClsShort ? 1 : 0;
  const int64_t r = bsum[blockIdx.x] + vl_cta_scan(v, wt) - v;
  // list appends aggregated per warp: the lanes bound for one list take
  // consecutive slots from a single atomic of their leader (one atomic per
  // list and warp instead of one per system)
  const int li = (s < nsys && cls >= 1 && cls <= kClsLong) ? cls - 1 : -1;
  const unsigned grp = __match_any_sync(0xffffffffu, li);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(grp) - 1;
  unsigned base = 0;
  if (li >= 0 && lane == leader) base = atomicAdd(&list_count[li], (unsigned)__popc(grp));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (li >= 0) lists[(int64_t)li * nsys + base + __popc(grp & ((1u << lane) - 1u))] = (int)s;
  if (s >= nsys) return;
  if (cls == kClsShort) {
    item_sys[r] = (int)s;
  } else if (cls == kClsBad) {
    atomicOr(err, kErrBadOffsets);
  } else if (cls == kClsTooLong) {
    atomicOr(err, kErrTooLong);
  }
}

// The work space of one solve, carved from one buffer.
struct VLSpace {
  int64_t *ctl;          // [0] short systems, [1] claim counter
  unsigned *list_count;  // kVLLists counters; kVarlenClaims on, their claim counters
  int64_t *bsum;         // ceil(nsys/256) per-CTA prefixes
  int *item_sys;         // the short queue, nsys entries
  int *lists;            // kVLLists lists of nsys entries
};

static inline size_t vl_al(size_t x) { return (x + 255) & ~(size_t)255; }

// bytes of the work space for nsys systems; with base and sp given, also its
// carving
static size_t vl_space(int64_t nsys, unsigned char *base, VLSpace *sp) {
  const size_t nb = (size_t)((nsys + kPrepThreads - 1) / kPrepThreads);
  size_t at = 0;
  const size_t o_ctl = at;
  at += 256;  // ctl (2 x int64), then the list counters at +64, their claim counters at +128
  const size_t o_bsum = at;
  at += vl_al(sizeof(int64_t) * nb);
  const size_t o_items = at;
  at += vl_al(sizeof(int) * (size_t)nsys);
  const size_t o_lists = at;
  at += vl_al(sizeof(int) * kVLLists * (size_t)nsys);
  if (base && sp) {
    sp->ctl = (int64_t *)(base + o_ctl);
    sp->list_count = (unsigned *)(base + o_ctl + 64);
    sp->bsum = (int64_t *)(base + o_bsum);
    sp->item_sys = (int *)(base + o_items);
    sp->lists = (int *)(base + o_lists);
  }
  return at;
}

static cudaError_t launch_varlen_prep(const int64_t *offsets, int64_t nsys, int64_t total,
                                      const VLSpace &sp, unsigned *err, cudaStream_t st) {
  const int64_t nb = (nsys + kPrepThreads - 1) / kPrepThreads;
  if (nb > 0x7fffffff) return cudaErrorInvalidValue;
  cudaError_t e = launch_pdl(varlen_prep_count, dim3((unsigned)nb), dim3(kPrepThreads), 0, st,
                             offsets, nsys, total, sp.bsum);
  if (e != cudaSuccess) return e;
  e = launch_pdl(varlen_prep_scan, dim3(1), dim3(1024), 0, st, sp.bsum, nb, sp.ctl,
                 sp.list_count);
  if (e != cudaSuccess) return e;
  return launch_pdl(varlen_prep_fill, dim3((unsigned)nb), dim3(kPrepThreads), 0, st, offsets,
                    nsys, total, (const int64_t *)sp.bsum, sp.item_sys, sp.lists, sp.list_count,
                    err);
}

template <typename T>
struct VLArgs {
  const T *a, *b, *c;
  T *d;
  const int64_t *offsets;
  const int *item_sys;        // the short queue (systems in system order)
  const int64_t *nitems;      // its length
  unsigned long long *queue;  // its claim counter
  int m2max, m4max;           // length buckets: 2 rows per lane up to m2max, 4 up to m4max
};

__device__ __forceinline__ void vl_cp_async(void *dst, const void *src, bool valid, int bytes) {
  const unsigned dd = (unsigned)__cvta_generic_to_shared(dst);
  const int sz = valid ? bytes : 0;  // 0: zero-fill, nothing read
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dd), "l"(src), "r"(sz)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dd), "l"(src), "r"(sz)
                 : "memory");
}

// rows rb .. rb+32M-1 of a system (clipped to len) into the warp's four
// regions (issue only; vl_read waits)
template <typename T, int M>
__device__ __forceinline__ void vl_issue(const VLArgs<T> &A, T *reg, int64_t lo, int64_t rb,
                                         int64_t len, int lane) {
  const T *src[4] = {A.a + lo, A.b + lo, A.c + lo, A.d + lo};
  __syncwarp();  // the previous item's reads of the regions are done
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int q = j * kWarp + lane;
    const int64_t r = rb + q;
    const bool in = r < len;
    const int sq = q + q / M;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      vl_cp_async(reg + k * kVLRegion + sq, in ? src[k] + r : src[k], in, (int)sizeof(T));
  }
}

// wait for vl_issue's copies, then this lane's rows rb+lane*M+j, transposed
template <typename T, int M>
__device__ __forceinline__ void vl_read(const T *reg, int64_t rb, int64_t len, int lane,
                                        T (&al)[M], T (&be)[M], T (&ga)[M], T (&de)[M]) {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncwarp();
  const int ts = lane * (M + 1);
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int64_t r = rb + lane * M + j;
    const bool in = r < len;
    al[j] = (in && r > 0) ? reg[ts + j] : T(0);
    be[j] = in ? reg[kVLRegion + ts + j] : T(1);
    ga[j] = (r < len - 1) ? reg[2 * kVLRegion + ts + j] : T(0);
    de[j] = reg[3 * kVLRegion + ts + j];  // zero-filled past len
  }
}

// this lane's solution rows through the warp's store region (the fifth),
// coalesced to d; the four staging regions may already hold the next item's
// copies in flight
template <typename T, int M>
__device__ __forceinline__ void vl_store(const VLArgs<T> &A, T *reg, int64_t lo, int64_t rb,
                                         int64_t len, int lane, const T (&x)[M]) {
  T *rd = reg + 4 * kVLRegion;
  const int ts = lane * (M + 1);
#pragma unroll
  for (int j = 0; j < M; ++j) rd[ts + j] = x[j];  // d slots read only by this lane
  __syncwarp();
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int q = j * kWarp + lane;
    if (rb + q < len) A.d[lo + rb + q] = rd[q + q / M];
  }
  __syncwarp();  // the store region is reused by the warp's next item
}

// ------------------------------------------------------------ short queue --
// One short system as a warp sees it.
struct VLItem {
  int64_t s;    // system, -1: nothing to do
  int64_t lo;   // first row of the system
  int64_t len;  // rows of the system
  int m;        // rows per lane of the staging: 2, 4 or 8
};

template <typename T>
__device__ __forceinline__ VLItem vl_item(const VLArgs<T> &A, int64_t it, int64_t nitems) {
  VLItem d = {-1, 0, 0, 8};
  if (it >= nitems) return d;
  const int64_t s = A.item_sys[it];
  d.s = s;
  d.lo = A.offsets[s];
  d.len = A.offsets[s + 1] - d.lo;
  d.m = d.len <= A.m2max ? 2 : (d.len <= A.m4max ? 4 : 8);
  return d;
}

template <typename T>
__device__ __forceinline__ void vl_issue_item(const VLArgs<T> &A, T *reg, const VLItem &d,
                                              int lane) {
  if (d.s < 0) return;
  if (d.m == 2)
    vl_issue<T, 2>(A, reg, d.lo, 0, d.len, lane);
  else if (d.m == 4)
    vl_issue<T, 4>(A, reg, d.lo, 0, d.len, lane);
  else
    vl_issue<T, 8>(A, reg, d.lo, 0, d.len, lane);
}

// a whole short system: rows already staged; the next item's copies go out
// as soon as the rows are in registers
template <typename T, int M>
__device__ __forceinline__ void vl_short_solve(const VLArgs<T> &A, T *reg, const VLItem &cur,
                                               const VLItem &nxt, int lane) {
  T al[M], be[M], ga[M], de[M];
  vl_read<T, M>(reg, 0, cur.len, lane, al, be, ga, de);
  vl_issue_item(A, reg, nxt, lane);
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  T xF, xL;
  warp_interface_solve(F, L, xF, xL, lane);
  chunk_backsub<T, M>(al, ga, de, xF, xL);
  vl_store<T, M>(A, reg, cur.lo, 0, cur.len, lane, de);
}

// The short queue, software-pipelined per warp: lane 0 claims the next item
// while the current one is staged; once the current item's rows are in
// registers the next item's copies are issued into the same staging
// regions, so they are in flight while the current item is solved and
// stored (stores go through a fifth region).
template <typename T>
__global__ void __launch_bounds__(kVLWarps * 32, 2) varlen_short_kernel(VLArgs<T> A) {
  extern __shared__ __align__(16) unsigned char vl_dyn[];
  const int lane = threadIdx.x & (kWarp - 1);
  T *reg = reinterpret_cast<T *>(vl_dyn) + (size_t)(threadIdx.x / kWarp) * 5 * kVLRegion;
  const int64_t nitems = *A.nitems;
  // items are claimed kVLBatch at a time (consecutive queue entries, so
  // consecutive systems in memory), and the batch after the current one is
  // requested as soon as the current one is taken: its atomic's result is
  // read only kVLBatch items later, so the claim latency is hidden
  unsigned long long first = 0, pending = 0;
  if (lane == 0) {
    first = atomicAdd(A.queue, (unsigned long long)kVLBatch);
    pending = atomicAdd(A.queue, (unsigned long long)kVLBatch);
  }
  int64_t base = (int64_t)__shfl_sync(0xffffffffu, first, 0);
  int k = 0;
  int64_t it = base;
  VLItem cur = vl_item(A, it, nitems);
  vl_issue_item(A, reg, cur, lane);
  while (it < nitems) {
    int64_t nit;
    if (k + 1 < kVLBatch) {
      nit = base + ++k;
    } else {
      base = (int64_t)__shfl_sync(0xffffffffu, pending, 0);
      k = 0;
      nit = base;
      if (lane == 0) pending = atomicAdd(A.queue, (unsigned long long)kVLBatch);
    }
    const VLItem nxt = vl_item(A, nit, nitems);
    if (cur.m == 2)
      vl_short_solve<T, 2>(A, reg, cur, nxt, lane);
    else if (cur.m == 4)
      vl_short_solve<T, 4>(A, reg, cur, nxt, lane);
    else
      vl_short_solve<T, 8>(A, reg, cur, nxt, lane);
    it = nit;
    cur = nxt;
  }
}

// ----------------------------------------------------------- long systems --
// Systems of 4097 .. 8192 rows (17 .. 32 blocks of 256): one CTA of
// kVLLongWarps warps per system, four CTAs per SM, each looping over the
// long systems' list (four 4-warp CTAs per SM measured ahead of two of 8
// warps by 2-7% on 4097..8192-row mixes, 5% behind on uniform 8192-row
// batches, whose four systems per SM crowd L2 before their second pass; one
// CTA of 16 warps and three or two 4-warp CTAs per SM were slower).  Thread
// 0 first asks L2 for the first half of the system (one bulk prefetch per
// array: the whole system measured 8% slower on uniform 8192-row batches,
// whose 592 CTAs' systems then exceed L2 before their second pass, and no
// prefetch 1% slower on 4097..8192-row mixes); every
// warp reduces its blocks (warp w: blocks w, w+4, ...) to their block rows
// in shared memory; warp 0 solves the block system (lane t = block t); every
// warp then stages its blocks again -- from L2, a few microseconds after
// the first read -- and finishes them from their two boundary unknowns
// (warp_block_finish).  In both passes a warp requests its next block as
// soon as the current one is in registers.  The second pass costs the chunk
// reductions again and reads of rows that L2 still holds, the rest from
// DRAM: four CTAs per SM keep more rows in flight than L2 holds.
template <typename T>
__device__ __forceinline__ void vl_prefetch_rows(const T *p, int64_t n) {
  // the 16-byte aligned interior of the rows, one bulk prefetch
  const uintptr_t b = ((uintptr_t)p + 15) & ~(uintptr_t)15;
  const uintptr_t e = (uintptr_t)(p + n) & ~(uintptr_t)15;
  if (e > b)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b), "r"((uint32_t)(e - b))
                 : "memory");
}

template <typename T>
__global__ void __launch_bounds__(kVLLongWarps * 32, 4)
    varlen_long_kernel(VLArgs<T> A, const int *__restrict__ list, const unsigned *__restrict__ count,
                       unsigned *__restrict__ claim) {
  extern __shared__ __align__(16) unsigned char vll_dyn[];
  __shared__ T brow[kVLMaxBlocks * 8];  // block rows; then the block unknowns at [8t], [8t+1]
  __shared__ unsigned s_next;
  const int lane = threadIdx.x & (kWarp - 1);
  const int w = threadIdx.x / kWarp;
  T *reg = reinterpret_cast<T *>(vll_dyn) + (size_t)w * 5 * kVLRegion;
  const int64_t cnt = (int64_t)*count;
  // systems claimed one at a time (lengths differ by up to 2x)
  if (threadIdx.x == 0) s_next = atomicAdd(claim, 1u);
  __syncthreads();
  for (int64_t i = s_next; i < cnt;) {
    const int s = list[i];
    const int64_t lo = A.offsets[s];
    const int64_t len = A.offsets[s + 1] - lo;
    const int nblk = (int)((len + kVLBlock - 1) / kVLBlock);
    if (threadIdx.x == 0) {
      const int64_t half = len / 2;
      vl_prefetch_rows(A.a + lo, half);
      vl_prefetch_rows(A.b + lo, half);
      vl_prefetch_rows(A.c + lo, half);
      vl_prefetch_rows(A.d + lo, half);
    }
    // ---- the warp's blocks reduced to their block rows; once a block's
    // rows are in registers the warp's next block is requested, so its
    // copies are in flight while this one is reduced
    if (w < nblk) vl_issue<T, 8>(A, reg, lo, (int64_t)w * kVLBlock, len, lane);
    for (int blk = w; blk < nblk; blk += kVLLongWarps) {
      const int64_t rb = (int64_t)blk * kVLBlock;
      T al[8], be[8], ga[8], de[8], bF[3], bL[3];
      vl_read<T, 8>(reg, rb, len, lane, al, be, ga, de);
      if (blk + kVLLongWarps < nblk)
        vl_issue<T, 8>(A, reg, lo, rb + kVLLongWarps * kVLBlock, len, lane);
      Row<T> F, L, FB, LB;
      chunk_reduce<T, 8>(al, be, ga, de, F, L);
      warp_block_basis(F, L, lane, bF, bL);
      block_rows(F, L, bF, bL, lane, FB, LB);
      if (lane == 0) {
        T *q = brow + 8 * blk;
        q[0] = FB.a; q[1] = FB.b; q[2] = FB.c; q[3] = FB.d;
        q[4] = LB.a; q[5] = LB.b; q[6] = LB.c; q[7] = LB.d;
      }
    }
    // the warp's first block of the second pass, requested before the wait
    if (w < nblk) vl_issue<T, 8>(A, reg, lo, (int64_t)w * kVLBlock, len, lane);
    __syncthreads();
    // ---- the block system (2 rows per block, lane t = block t)
    if (w == 0) {
      Row<T> RF{T(0), T(1), T(0), T(0)}, RL{T(0), T(1), T(0), T(0)};
      if (lane < nblk) {
        const T *q = brow + 8 * lane;
        RF = {q[0], q[1], q[2], q[3]};
        RL = {q[4], q[5], q[6], q[7]};
      }
      T f, l;
      warp_interface_solve(RF, RL, f, l, lane);
      __syncwarp();
      if (lane < nblk) {
        brow[8 * lane] = f;
        brow[8 * lane + 1] = l;
      }
    }
    __syncthreads();
    // ---- the warp's blocks again (L2), back-substituted from their two
    // boundary unknowns
    for (int blk = w; blk < nblk; blk += kVLLongWarps) {
      const int64_t rb = (int64_t)blk * kVLBlock;
      T al[8], be[8], ga[8], de[8];
      vl_read<T, 8>(reg, rb, len, lane, al, be, ga, de);
      if (blk + kVLLongWarps < nblk)
        vl_issue<T, 8>(A, reg, lo, rb + kVLLongWarps * kVLBlock, len, lane);
      Row<T> F, L;
      chunk_reduce<T, 8>(al, be, ga, de, F, L);
      T xF, xL;
      warp_block_finish(F, L, brow[8 * blk], brow[8 * blk + 1], lane, xF, xL);
      chunk_backsub<T, 8>(al, ga, de, xF, xL);
      vl_store<T, 8>(A, reg, lo, rb, len, lane, de);
    }
    if (threadIdx.x == 0) s_next = atomicAdd(claim, 1u);
    __syncthreads();  // brow is rewritten by the next system; s_next is seen
    i = s_next;
    __syncthreads();  // every thread has read s_next
  }
}

// ---------------------------------------------------------------- launches --
template <typename T>
static int varlen_smem_bytes() {
  return kVLWarps * 5 * kVLRegion * (int)sizeof(T);  // both kernels: 8 warps of 5 regions
}

// CTAs of `kern` resident on the whole device at once (sets the
// shared-memory attribute on the first call per device)
template <typename K>
static cudaError_t persistent_grid(K kern, int threads, int smem, int &grid, bool (&attr)[64]) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr[dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr[dev] = true;
  }
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  grid = sms * per_sm;
  return cudaSuccess;
}

// Everything after the preparation: the one-CTA buckets, the long systems,
// the short queue (one stream, in that order).
template <typename T>
static cudaError_t launch_varlen_work(const VLArgs<T> &A, const VLSpace &sp, int64_t nsys,
                                      cudaStream_t st) {
  static bool attr_short[64] = {}, attr_long[64] = {};
  const int smem = varlen_smem_bytes<T>();
  cudaError_t e =
      launch_xcta_varlen<T>(A.a, A.b, A.c, A.d, A.offsets, sp.lists, nsys, sp.list_count, st);
  if (e != cudaSuccess) return e;
  int grid = 0;
  const int lsmem = kVLLongWarps * 5 * kVLRegion * (int)sizeof(T);
  e = persistent_grid(varlen_long_kernel<T>, kVLLongWarps * 32, lsmem, grid, attr_long);
  if (e != cudaSuccess) return e;

  // the long systems and the short queue keep the plain launch (under
  // programmatic launch the long class measured 9% slower)
  varlen_long_kernel<T><<<(unsigned)grid, kVLLongWarps * 32, lsmem, st>>>(
      A, sp.lists + (size_t)(kClsLong - 1) * nsys, sp.list_count + (kClsLong - 1),
      sp.list_count + kVarlenClaims + (kClsLong - 1));
  e = persistent_grid(varlen_short_kernel<T>, kVLWarps * 32, smem, grid, attr_short);
  if (e != cudaSuccess) return e;
  varlen_short_kernel<T><<<(unsigned)grid, kVLWarps * 32, smem, st>>>(A);
  return cudaGetLastError();
}

template <typename T>
static VLArgs<T> varlen_args(const T *a, const T *b, const T *c, T *d, const int64_t *offsets,
                             const VLSpace &sp) {
  VLArgs<T> A;
  A.a = a;
  A.b = b;
  A.c = c;
  A.d = d;
  A.offsets = offsets;
  A.item_sys = sp.item_sys;
  A.nitems = sp.ctl;
  A.queue = (unsigned long long *)(sp.ctl + 1);
  varlen_buckets((int)sizeof(T), A.m2max, A.m4max);
  return A;
}

template <typename T>
cudaError_t launch_varlen(const T *a, const T *b, const T *c, T *d, const int64_t *offsets,
                          int64_t nsys, int64_t total, unsigned *err, cudaStream_t st) {
  const Scratch sc(vl_space(nsys, nullptr, nullptr), 0, st);
  unsigned char *w = (unsigned char *)sc.get();
  if (!w) return cudaErrorMemoryAllocation;
  VLSpace sp;
  vl_space(nsys, w, &sp);
  cudaError_t e = launch_varlen_prep(offsets, nsys, total, sp, err, st);
  if (e != cudaSuccess) return e;
  return launch_varlen_work<T>(varlen_args(a, b, c, d, offsets, sp), sp, nsys, st);
}

template cudaError_t launch_varlen<float>(const float *, const float *, const float *, float *,
                                          const int64_t *, int64_t, int64_t, unsigned *,
                                          cudaStream_t);
template cudaError_t launch_varlen<double>(const double *, const double *, const double *, double *,
                                           const int64_t *, int64_t, int64_t, unsigned *,
                                           cudaStream_t);

}  // namespace tridb200

using namespace tridb200;

template <typename T>
static tridStatus_t varlen_entry(const T *a, const T *b, const T *c, T *d, const int64_t *offsets,
                                 int64_t nsys, int64_t total) {
  if (nsys < 0 || total < 0 || !offsets || (total > 0 && (!a || !b || !c || !d)))
    return TRID_STATUS_INVALID_VALUE;
  if (nsys == 0 || total == 0) return TRID_STATUS_SUCCESS;
  if (nsys >= ((int64_t)1 << 31)) return TRID_STATUS_INVALID_VALUE;  // int item tables
  unsigned *err = device_error_flags();
  if (!err) return TRID_STATUS_ALLOC_FAILED;
  const cudaError_t e = launch_varlen<T>(a, b, c, d, offsets, nsys, total, err, current_stream());
  if (e == cudaErrorMemoryAllocation) return TRID_STATUS_ALLOC_FAILED;
  return e == cudaSuccess ? TRID_STATUS_SUCCESS : TRID_STATUS_EXECUTION_FAILED;
}

static_assert(sizeof(long long) == sizeof(int64_t), "int64 offsets");
extern "C" tridStatus_t tridDmtsvVarlenBatch(const double *a, const double *b, const double *c,
                                             double *d, const long long *offsets, long long nsys,
                                             long long total) {
  return varlen_entry<double>(a, b, c, d, (const int64_t *)offsets, nsys, total);
}
extern "C" tridStatus_t tridSmtsvVarlenBatch(const float *a, const float *b, const float *c,
                                             float *d, const long long *offsets, long long nsys,
                                             long long total) {
  return varlen_entry<float>(a, b, c, d, (const int64_t *)offsets, nsys, total);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the variable-length solve.
//
// Some callers cannot allocate device memory: code that runs under another
// component's allocator or memory budget, where a driver allocation would
// steal memory the pool has reserved (or fail), and latency-critical loops
// where the implicit device synchronisation of cudaMalloc/cudaFree is not
// acceptable.  tridDmtsvVarlenBatchNoAlloc serves them: its work space (the
// preparation's prefixes, the short queue, the class lists, their counters
// and an error word) lives in the fixed array below, which every GPU that
// loads this library holds until the process exits.  Nothing is allocated
// per call.
// ---------------------------------------------------------------------------
namespace tridb200 {

constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;  // 32 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[64];  // device address of g_noalloc_scratch, per device

// Device address of the static array on the current device.  The host-side
// name g_noalloc_scratch is only a stand-in, never a device address, so the
// address is looked up once per device (with that device current) and cached.
static void *noalloc_scratch_address() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    g_noalloc_ptr[dev] = p;
  }
  return g_noalloc_ptr[dev];
}

// The allocation-free solve's error word (the first bytes of the static
// array) on the current device, or nullptr when no allocation-free solve has
// run there yet (the word is then still zero).  Read and cleared by
// tridGetDeviceErrors.
unsigned *noalloc_error_word() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  return (unsigned *)g_noalloc_ptr[dev];
}

// The static array: the error word (its own 256 bytes), then the work space
// of vl_space.  False when a solve of nsys systems does not fit.
static bool noalloc_fits(int64_t nsys) {
  return 256 + vl_space(nsys, nullptr, nullptr) <= kNoAllocScratchBytes;
}

}  // namespace tridb200

extern "C" tridStatus_t tridDmtsvVarlenBatchNoAlloc(const double *a, const double *b,
                                                    const double *c, double *d,
                                                    const long long *offsets, long long nsys,
                                                    long long total) {
  using namespace tridb200;
  if (nsys < 0 || total < 0 || !offsets || (total > 0 && (!a || !b || !c || !d)))
    return TRID_STATUS_INVALID_VALUE;
  if (nsys == 0 || total == 0) return TRID_STATUS_SUCCESS;
  if (nsys >= ((int64_t)1 << 31) || total > ((int64_t)1 << 46)) return TRID_STATUS_INVALID_VALUE;
  if (!noalloc_fits(nsys)) return TRID_STATUS_INVALID_VALUE;  // too large
  unsigned char *w = (unsigned char *)noalloc_scratch_address();
  if (!w) return TRID_STATUS_EXECUTION_FAILED;
  const cudaStream_t st = current_stream();
  unsigned *err = (unsigned *)w;
  VLSpace sp;
  vl_space(nsys, w + 256, &sp);
  // the preparation rewrites the prefixes, the queue and the lists and clears
  // the counters, so whatever the previous call left in the array does not
  // matter
  const int64_t *off = (const int64_t *)offsets;
  if (launch_varlen_prep(off, nsys, total, sp, err, st) != cudaSuccess ||
      launch_varlen_work<double>(varlen_args(a, b, c, d, off, sp), sp, nsys, st) != cudaSuccess)
    return TRID_STATUS_EXECUTION_FAILED;
  return TRID_STATUS_SUCCESS;
}
