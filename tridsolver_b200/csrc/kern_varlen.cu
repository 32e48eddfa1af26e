// Variable-length packed batch (sm_100a): length-bucketed work, persistent
// launches.
//
// System s occupies rows [offsets[s], offsets[s+1]) of every array (unit
// stride, int64 offsets).  Three length classes:
//   * 257 .. 4096 rows: the one-CTA buckets (launch_xcta_varlen,
//     kern_xcta.cu): bucket W holds the systems that need W = ceil(n/512)
//     warps at 16 rows per lane; one persistent launch per bucket, CTA = W
//     warps solving one system at a time with every row read once.  (In the
//     block items below they moved 72 bytes per FP64 unknown at 1.9-2.3
//     TB/s algorithmic; 300-row systems at 1.4.)
//   * at most 256 rows, and 4097 .. 8192 rows: two work queues in system
//     order, served by the same persistent warps one after the other:
//   * the reduce queue: a system of at most 256 rows is one item, solved
//     whole by one warp with the partitioned Thomas of partition.cuh, the
//     rows-per-lane chunk M picked from the length (2/4/8: the length
//     buckets); a longer system (up to 32 blocks of 256 rows = 8192 rows)
//     gives one item per block: the warp reduces its block to the block's two
//     boundary rows (warp_block_basis / block_rows), publishes them and counts
//     the block done on the system's counter; the warp that completes the
//     count solves the system's block system (2 rows per block, one warp
//     interface solve), publishes the block boundary unknowns and marks the
//     system solved.  Nothing waits in this phase.
//   * the finish queue (taken once the reduce queue is empty): one item per
//     block of a long system; the warp reduces the block again and
//     back-substitutes from the block's boundary unknowns.  Its system was
//     marked solved long ago except for the last few systems, whose reduce
//     items are held by running warps; for those the warp polls the mark a
//     bounded number of times (a timeout is recorded in the device error
//     word and the block skipped).
// Items map to their system through per-item tables built beforehand.
// Rows reach each warp's shared-memory regions by coalesced cp.async (row q
// of the 32*M at q + q/M, conflict-free for the lane-per-chunk reads) and
// leave by coalesced stores.  Long systems move their rows twice (reduce,
// finish): 72 bytes per FP64 unknown, like the blocked partition of
// kern_general.cu.
//
// Three preparation launches (launch_varlen_prep) turn offsets into the
// prefix sums and item tables of both queues and the one-CTA bucket lists,
// and clear the queues and the per-system counters.
// Malformed offsets (decreasing or past `total`) and systems longer than
// 8192 rows are skipped and recorded in the device error word (bits 4 and 8).
// The item tables hold `cap` = nsys + total/256 + 1 entries, which bounds the
// items of any offsets that increase monotonically.  Offsets that do not
// (e.g. 0, T, 0, T, ...: every other system valid and T rows long) can ask
// for more; a system whose items would end past `cap` is skipped whole
// (its table entries read -1) and recorded as malformed (bit 4), so no table,
// block-row or queue access ever leaves the scratch.
#include <mutex>

#include "partition.cuh"
#include "tma.cuh"

namespace tridb200 {

constexpr int kVLBlock = 256;   // rows per block of a long system (M = 8)
constexpr int kVLShort = kVarlenShort;  // longest system solved as one item
// systems of kVLShort+1 .. kVLMid rows go to the one-CTA buckets
constexpr int kVLMid = 512 * kVarlenCtaBuckets;
constexpr int kVLMaxBlocks = 32;
constexpr int kVLWarps = 8;     // warps per CTA
constexpr int kVLRegion = 32 * (8 + 1);  // elements per staged array and warp
constexpr unsigned kErrBadOffsets = 4u;
constexpr unsigned kErrTooLong = 8u;
constexpr unsigned kVLSolved = 0x80000000u;  // sys_count flag: block solution published
constexpr uint32_t kVLMaxIdle = 1u << 22;    // finish-queue polls after the reduce queue ran dry

__device__ __forceinline__ bool vl_bad(int64_t lo, int64_t hi, int64_t total) {
  return hi < lo || lo < 0 || hi > total;
}

// a system for the one-CTA buckets (launch_xcta_varlen, kern_xcta.cu)
__device__ __forceinline__ bool vl_mid(int64_t len) { return len > kVLShort && len <= kVLMid; }
// a system for the long-system CTAs (varlen_long_kernel)
__device__ __forceinline__ bool vl_long(int64_t len) {
  return len > kVLMid && len <= (int64_t)kVLBlock * kVLMaxBlocks;
}

// reduce items of a system of len rows (none for the CTA classes)
__device__ __forceinline__ int64_t vl_items(int64_t len) {
  if (len <= kVLShort) return 1;
  if (vl_mid(len) || vl_long(len)) return 0;
  return (len + kVLBlock - 1) / kVLBlock;
}

// finish items: one per block of a long system that can be solved
__device__ __forceinline__ int64_t vl_fitems(int64_t len) {
  if (len <= kVLShort || vl_mid(len) || vl_long(len)) return 0;
  const int64_t nb = (len + kVLBlock - 1) / kVLBlock;
  return nb <= kVLMaxBlocks ? nb : 0;
}

// Preparation, three short launches over the systems (256 per CTA):
//   count: reduce and finish items per CTA of systems -> bsum;
//   scan : one CTA, exclusive prefix of bsum; totals; clears both queues;
//   fill : per system, its prefixes item_off/fitem_off (CTA scan + the CTA's
//          prefix), its counter cleared, and the system index written into
//          the item tables item_sys/fitem_sys for each of its items.
constexpr int kPrepThreads = 256;

// Items of system s, each count clamped to cap + 1 so that the prefix sums
// stay far from int64 overflow whatever the offsets hold (a system with more
// than cap items is skipped by the fill anyway).
__device__ __forceinline__ void vl_counts(const int64_t *offsets, int64_t nsys, int64_t total,
                                          int64_t cap, int64_t s, int64_t &ni, int64_t &nf) {
  ni = nf = 0;
  if (s >= nsys) return;
  int64_t len = offsets[s + 1] - offsets[s];
  if (vl_bad(offsets[s], offsets[s + 1], total)) len = 0;
  ni = vl_items(len > 0 ? len : 1);
  nf = vl_fitems(len);
  if (ni > cap + 1) ni = cap + 1;
  if (nf > cap + 1) nf = cap + 1;
}

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
                                                                  int64_t cap,
                                                                  int64_t *__restrict__ bsum) {
  __shared__ int64_t wt[kPrepThreads / 32];
  const int64_t s = (int64_t)blockIdx.x * kPrepThreads + threadIdx.x;
  int64_t ni, nf;
  vl_counts(offsets, nsys, total, cap, s, ni, nf);
  const int64_t ci = vl_cta_scan(ni, wt);
  const int64_t cf = vl_cta_scan(nf, wt);
  if (threadIdx.x == kPrepThreads - 1) {
    bsum[2 * blockIdx.x] = ci;
    bsum[2 * blockIdx.x + 1] = cf;
  }
}

__global__ void __launch_bounds__(1024) varlen_prep_scan(int64_t *__restrict__ bsum, int64_t nblocks,
                                                         int64_t nsys, int64_t *__restrict__ item_off,
                                                         int64_t *__restrict__ fitem_off,
                                                         unsigned long long *__restrict__ queue,
                                                         unsigned *__restrict__ mid_count) {
  __shared__ int64_t part[1024], fpart[1024];
  const int tid = threadIdx.x;
  const int64_t per = (nblocks + 1023) / 1024;
  const int64_t b0 = tid * per, b1 = (b0 + per < nblocks) ? b0 + per : nblocks;
  int64_t acc = 0, facc = 0;
  for (int64_t b = b0; b < b1; ++b) {
    acc += bsum[2 * b];
    facc += bsum[2 * b + 1];
  }
  part[tid] = acc;
  fpart[tid] = facc;
  __syncthreads();
  if (tid == 0) {
    int64_t run = 0, frun = 0;
    for (int k = 0; k < 1024; ++k) {
      const int64_t v = part[k], fv = fpart[k];
      part[k] = run;
      fpart[k] = frun;
      run += v;
      frun += fv;
    }
    item_off[nsys] = run;
    fitem_off[nsys] = frun;
    queue[0] = 0ull;
    queue[1] = 0ull;
    for (int k = 0; k <= kVarlenCtaBuckets; ++k) mid_count[k] = 0u;
  }
  __syncthreads();
  int64_t run = part[tid], frun = fpart[tid];
  for (int64_t b = b0; b < b1; ++b) {
    const int64_t v = bsum[2 * b], fv = bsum[2 * b + 1];
    bsum[2 * b] = run;
    bsum[2 * b + 1] = frun;
    run += v;
    frun += fv;
  }
}

__global__ void __launch_bounds__(kPrepThreads) varlen_prep_fill(
    const int64_t *__restrict__ offsets, int64_t nsys, int64_t total, int64_t cap,
    const int64_t *__restrict__ bsum, int64_t *__restrict__ item_off,
    int64_t *__restrict__ fitem_off, int *__restrict__ item_sys, int *__restrict__ fitem_sys,
    unsigned *__restrict__ sys_count, int *__restrict__ mid_list, unsigned *__restrict__ mid_count,
    unsigned *__restrict__ err) {
  __shared__ int64_t wt[kPrepThreads / 32];
  const int64_t s = (int64_t)blockIdx.x * kPrepThreads + threadIdx.x;
  int64_t ni, nf;
  vl_counts(offsets, nsys, total, cap, s, ni, nf);
  const int64_t ri = bsum[2 * blockIdx.x] + vl_cta_scan(ni, wt) - ni;
  const int64_t rf = bsum[2 * blockIdx.x + 1] + vl_cta_scan(nf, wt) - nf;
  if (s >= nsys) return;
  item_off[s] = ri;
  fitem_off[s] = rf;
  sys_count[s] = 0u;
  // A system whose items end past the tables' capacity (only non-monotone
  // offsets get there) is skipped whole: its entries below cap read -1.
  const bool fits = ri + ni <= cap && rf + nf <= cap;
  if (!fits) atomicOr(err, kErrBadOffsets);
  const int tag = fits ? (int)s : -1;
  for (int64_t k = ri; k < ri + ni && k < cap; ++k) item_sys[k] = tag;
  for (int64_t k = rf; k < rf + nf && k < cap; ++k) fitem_sys[k] = tag;
  // a system for the one-CTA buckets: listed in bucket ceil(len/512) - 1
  // (each bucket holds up to nsys entries; a system is listed once)
  // and a long system in the list after them
  const int64_t lo = offsets[s], hi = offsets[s + 1];
  if (!vl_bad(lo, hi, total) && (vl_mid(hi - lo) || vl_long(hi - lo))) {
    const int wb = vl_mid(hi - lo) ? (int)((hi - lo + 511) / 512) - 1 : kVarlenCtaBuckets;
    const unsigned pos = atomicAdd(&mid_count[wb], 1u);
    mid_list[(int64_t)wb * nsys + pos] = (int)s;
  }
}

// Capacity of the item tables: enough for any monotone offsets
// (sum over systems of max(1, ceil(len/256)) <= nsys + total/256).
static inline int64_t varlen_cap(int64_t nsys, int64_t total) {
  return nsys + total / kVLBlock + 1;
}

// the three preparation launches; bsum holds 2*ceil(nsys/256) int64, the
// item tables cap = varlen_cap(nsys, total) entries each, mid_list
// (kVarlenCtaBuckets+1)*nsys ints, mid_count kVarlenCtaBuckets+1 counters
static cudaError_t launch_varlen_prep(const int64_t *offsets, int64_t nsys, int64_t total,
                                      int64_t *bsum, int64_t *item_off, int64_t *fitem_off,
                                      int *item_sys, int *fitem_sys, unsigned *sys_count,
                                      unsigned long long *queue, int *mid_list,
                                      unsigned *mid_count, unsigned *err, cudaStream_t st) {
  const int64_t nb = (nsys + kPrepThreads - 1) / kPrepThreads;
  if (nb > 0x7fffffff) return cudaErrorInvalidValue;
  const int64_t cap = varlen_cap(nsys, total);
  varlen_prep_count<<<(unsigned)nb, kPrepThreads, 0, st>>>(offsets, nsys, total, cap, bsum);
  varlen_prep_scan<<<1, 1024, 0, st>>>(bsum, nb, nsys, item_off, fitem_off, queue, mid_count);
  varlen_prep_fill<<<(unsigned)nb, kPrepThreads, 0, st>>>(offsets, nsys, total, cap, bsum,
                                                          item_off, fitem_off, item_sys,
                                                          fitem_sys, sys_count, mid_list,
                                                          mid_count, err);
  return cudaGetLastError();
}

template <typename T>
struct VLArgs {
  const T *a, *b, *c;
  T *d;
  const int64_t *offsets;
  const int64_t *item_off;   // reduce-queue prefix, nsys+1
  const int64_t *fitem_off;  // finish-queue prefix, nsys+1
  const int *item_sys;       // system of every reduce item (-1: skipped)
  const int *fitem_sys;      // system of every finish item (-1: skipped)
  int64_t nsys;
  int64_t total;
  int64_t cap;               // entries of item_sys / fitem_sys / block rows
  int m2max, m4max;          // length buckets: 2 rows per lane up to m2max, 4 up to m4max
  unsigned *sys_count;
  unsigned long long *queue;  // [0] reduce queue, [1] finish queue
  T *rows;       // per reduce item: the block's 8 row values; later its 2 unknowns
  unsigned *err;
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

__device__ __forceinline__ unsigned vl_load_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// One work item as a warp sees it: the rows of system s to stage (a whole
// short system, or block `blk` of a long one) and the rows per lane m.
struct VLItem {
  int64_t s;    // system, -1: nothing to do
  int64_t lo;   // first row of the system
  int64_t len;  // rows of the system
  int blk;      // block of a long system, -1: the whole (short) system
  int m;        // rows per lane of the staging: 2, 4 or 8
};

template <typename T>
__device__ __forceinline__ void vl_issue_item(const VLArgs<T> &A, T *reg, const VLItem &d,
                                              int lane) {
  if (d.s < 0) return;
  const int64_t rb = d.blk < 0 ? 0 : (int64_t)d.blk * kVLBlock;
  if (d.m == 2)
    vl_issue<T, 2>(A, reg, d.lo, rb, d.len, lane);
  else if (d.m == 4)
    vl_issue<T, 4>(A, reg, d.lo, rb, d.len, lane);
  else
    vl_issue<T, 8>(A, reg, d.lo, rb, d.len, lane);
}

// reduce-queue item `it` (every lane computes the same descriptor); records
// malformed offsets and over-long systems once
template <typename T>
__device__ __forceinline__ VLItem vl_reduce_item(const VLArgs<T> &A, int64_t it, int64_t nitems,
                                                 int lane) {
  VLItem d = {-1, 0, 0, -1, 8};
  if (it >= nitems) return d;
  const int64_t s = A.item_sys[it];
  if (s < 0) return d;  // skipped by the preparation (past cap)
  const int64_t lo = A.offsets[s], hi = A.offsets[s + 1];
  if (vl_bad(lo, hi, A.total)) {
    if (lane == 0) atomicOr(A.err, kErrBadOffsets);
    return d;
  }
  const int64_t len = hi - lo;
  if (len == 0) return d;
  if (len <= kVLShort) {
    d.m = len <= A.m2max ? 2 : (len <= A.m4max ? 4 : 8);
  } else {
    const int64_t nblk = (len + kVLBlock - 1) / kVLBlock;
    if (nblk > kVLMaxBlocks) {
      if (lane == 0 && it == A.item_off[s]) atomicOr(A.err, kErrTooLong);
      return d;
    }
    d.blk = (int)(it - A.item_off[s]);
  }
  d.s = s;
  d.lo = lo;
  d.len = len;
  return d;
}

template <typename T>
__device__ __forceinline__ VLItem vl_finish_item(const VLArgs<T> &A, int64_t fi, int64_t nf) {
  VLItem d = {-1, 0, 0, -1, 8};
  if (fi >= nf) return d;
  const int64_t s = A.fitem_sys[fi];
  if (s < 0) return d;
  d.s = s;
  d.lo = A.offsets[s];
  d.len = A.offsets[s + 1] - d.lo;
  d.blk = (int)(fi - A.fitem_off[s]);
  return d;
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

__device__ __forceinline__ unsigned vl_add_acq_rel(unsigned *p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v)
               : "memory");
  return old;
}

__device__ __forceinline__ void vl_or_release(unsigned *p, unsigned v) {
  asm volatile("red.release.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Both queues are software-pipelined per warp: lane 0 claims the next item
// while the current one is staged; once the current item's rows are in
// registers the next item's copies are issued into the same staging
// regions, so they are in flight while the current item is solved and
// stored (stores go through a fifth region).
template <typename T>
__global__ void __launch_bounds__(kVLWarps * 32, 2) varlen_kernel(VLArgs<T> A) {
  extern __shared__ __align__(16) unsigned char vl_dyn[];
  const int lane = threadIdx.x & (kWarp - 1);
  T *reg = reinterpret_cast<T *>(vl_dyn) + (size_t)(threadIdx.x / kWarp) * 5 * kVLRegion;
  // the prefixes can pass cap only for non-monotone offsets; the systems past
  // it were skipped by the preparation
  const int64_t nitems = A.item_off[A.nsys] < A.cap ? A.item_off[A.nsys] : A.cap;
  const int64_t nf = A.fitem_off[A.nsys] < A.cap ? A.fitem_off[A.nsys] : A.cap;
  // ---- reduce queue ----
  unsigned long long claim = 0;
  if (lane == 0) claim = atomicAdd(&A.queue[0], 1ull);
  int64_t it = (int64_t)__shfl_sync(0xffffffffu, claim, 0);
  VLItem cur = vl_reduce_item(A, it, nitems, lane);
  vl_issue_item(A, reg, cur, lane);
  while (it < nitems) {
    if (lane == 0) claim = atomicAdd(&A.queue[0], 1ull);
    const int64_t nit = (int64_t)__shfl_sync(0xffffffffu, claim, 0);
    const VLItem nxt = vl_reduce_item(A, nit, nitems, lane);
    if (cur.s < 0) {
      vl_issue_item(A, reg, nxt, lane);
    } else if (cur.blk < 0) {
      if (cur.m == 2)
        vl_short_solve<T, 2>(A, reg, cur, nxt, lane);
      else if (cur.m == 4)
        vl_short_solve<T, 4>(A, reg, cur, nxt, lane);
      else
        vl_short_solve<T, 8>(A, reg, cur, nxt, lane);
    } else {
      // one block of a long system: chunk reduction + block basis, its two
      // block rows published, the block counted done
      const int64_t s = cur.s;
      const int nblk = (int)((cur.len + kVLBlock - 1) / kVLBlock);
      T al[8], be[8], ga[8], de[8], bF[3], bL[3];
      vl_read<T, 8>(reg, (int64_t)cur.blk * kVLBlock, cur.len, lane, al, be, ga, de);
      vl_issue_item(A, reg, nxt, lane);
      Row<T> F, L, FB, LB;
      chunk_reduce<T, 8>(al, be, ga, de, F, L);
      warp_block_basis(F, L, lane, bF, bL);
      block_rows(F, L, bF, bL, lane, FB, LB);
      // the block rows published by lane 0 before it counts the block done
      // (release); the warp that completes the count acquires every block's
      T *rw = A.rows + ((int64_t)A.item_off[s] + cur.blk) * 8;
      unsigned done = 0;
      if (lane == 0) {
        rw[0] = FB.a; rw[1] = FB.b; rw[2] = FB.c; rw[3] = FB.d;
        rw[4] = LB.a; rw[5] = LB.b; rw[6] = LB.c; rw[7] = LB.d;
        done = vl_add_acq_rel(&A.sys_count[s], 1u);
      }
      done = __shfl_sync(0xffffffffu, done, 0);
      if (done == (unsigned)(nblk - 1)) {
        __syncwarp();  // lane 0's acquire orders the block rows for the whole warp
        // the block system of s: lane t holds block t's two rows
        T *rs = A.rows + (int64_t)A.item_off[s] * 8;
        Row<T> RF{T(0), T(1), T(0), T(0)}, RL{T(0), T(1), T(0), T(0)};
        if (lane < nblk) {
          const T *q = rs + (int64_t)lane * 8;
          RF = {__ldcg(q + 0), __ldcg(q + 1), __ldcg(q + 2), __ldcg(q + 3)};
          RL = {__ldcg(q + 4), __ldcg(q + 5), __ldcg(q + 6), __ldcg(q + 7)};
        }
        T fB, lB;
        int span = 1;
        while (span < nblk) span <<= 1;
        warp_interface_solve(RF, RL, fB, lB, lane, span);
        __syncwarp();  // all block rows read before they are overwritten
        if (lane < nblk) {
          rs[(int64_t)lane * 8 + 0] = fB;  // block t's boundary unknowns
          rs[(int64_t)lane * 8 + 1] = lB;
        }
        __syncwarp();
        if (lane == 0) vl_or_release(&A.sys_count[s], kVLSolved);  // cumulative release
      }
    }
    it = nit;
    cur = nxt;
  }
  // ---- finish queue: every block of a long system again, back-substituted
  // from its boundary unknowns once the system's mark is set ----
  if (lane == 0) claim = atomicAdd(&A.queue[1], 1ull);
  int64_t fi = (int64_t)__shfl_sync(0xffffffffu, claim, 0);
  cur = vl_finish_item(A, fi, nf);
  vl_issue_item(A, reg, cur, lane);
  while (fi < nf) {
    if (lane == 0) claim = atomicAdd(&A.queue[1], 1ull);
    const int64_t nfi = (int64_t)__shfl_sync(0xffffffffu, claim, 0);
    const VLItem nxt = vl_finish_item(A, nfi, nf);
    if (cur.s < 0) {
      vl_issue_item(A, reg, nxt, lane);
    } else {
      const int64_t s = cur.s;
      T al[8], be[8], ga[8], de[8], bF[3], bL[3];
      vl_read<T, 8>(reg, (int64_t)cur.blk * kVLBlock, cur.len, lane, al, be, ga, de);
      vl_issue_item(A, reg, nxt, lane);
      Row<T> F, L;
      chunk_reduce<T, 8>(al, be, ga, de, F, L);
      warp_block_basis(F, L, lane, bF, bL);
      // the system's reduce items were all taken by running warps before the
      // finish queue opened: its mark comes; poll a bounded number of times
      int ok = 0;
      if (lane == 0) {
        for (uint32_t k = 0; k < kVLMaxIdle; ++k) {
          if (vl_load_acquire(&A.sys_count[s]) & kVLSolved) {
            ok = 1;
            break;
          }
          __nanosleep(128);
        }
        if (!ok) atomicOr(A.err, kErrWaitTimeout);
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      __syncwarp();  // lane 0's acquire orders the boundary unknowns for the warp
      if (ok) {
        const T *bs = A.rows + ((int64_t)A.item_off[s] + cur.blk) * 8;
        const T f = __ldcg(bs), l = __ldcg(bs + 1);
        const T xF = bF[0] + f * bF[1] + l * bF[2];
        const T xL = bL[0] + f * bL[1] + l * bL[2];
        chunk_backsub<T, 8>(al, ga, de, xF, xL);
        vl_store<T, 8>(A, reg, cur.lo, (int64_t)cur.blk * kVLBlock, cur.len, lane, de);
      }
    }
    fi = nfi;
    cur = nxt;
  }
}

// Systems of 4097 .. 8192 rows (17 .. 32 blocks of 256): one CTA of
// kVLLongWarps warps per system, two CTAs per SM, each looping over the
// long systems' list.  Thread 0 first asks L2 for the whole system (one bulk
// prefetch per array, so its DRAM reads are all in flight at once); every
// warp reduces its blocks (warp w: blocks w, w+8, ...) to their block rows
// in shared memory; warp 0 solves the block system (lane t = block t); every
// warp then stages its blocks again -- from L2, a few microseconds after
// the first read -- and finishes them.  DRAM moves each input once (40 bytes
// per FP64 unknown); the second pass costs L2 reads and the chunk
// reductions again.
constexpr int kVLLongWarps = 8;

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
__global__ void __launch_bounds__(kVLLongWarps * 32, 2)
    varlen_long_kernel(VLArgs<T> A, const int *__restrict__ list, const unsigned *__restrict__ count) {
  extern __shared__ __align__(16) unsigned char vll_dyn[];
  __shared__ T brow[kVLMaxBlocks * 8];  // block rows; then the block unknowns at [8t], [8t+1]
  const int lane = threadIdx.x & (kWarp - 1);
  const int w = threadIdx.x / kWarp;
  T *reg = reinterpret_cast<T *>(vll_dyn) + (size_t)w * 5 * kVLRegion;
  const int64_t cnt = (int64_t)*count;
  for (int64_t i = blockIdx.x; i < cnt; i += gridDim.x) {
    const int s = list[i];
    const int64_t lo = A.offsets[s];
    const int64_t len = A.offsets[s + 1] - lo;
    const int nblk = (int)((len + kVLBlock - 1) / kVLBlock);
    if (threadIdx.x == 0) {
      vl_prefetch_rows(A.a + lo, len);
      vl_prefetch_rows(A.b + lo, len);
      vl_prefetch_rows(A.c + lo, len);
      vl_prefetch_rows(A.d + lo, len);
    }
    // ---- the warp's blocks reduced to their block rows
    for (int blk = w; blk < nblk; blk += kVLLongWarps) {
      const int64_t rb = (int64_t)blk * kVLBlock;
      vl_issue<T, 8>(A, reg, lo, rb, len, lane);
      T al[8], be[8], ga[8], de[8], bF[3], bL[3];
      vl_read<T, 8>(reg, rb, len, lane, al, be, ga, de);
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
      vl_issue<T, 8>(A, reg, lo, rb, len, lane);
      T al[8], be[8], ga[8], de[8];
      vl_read<T, 8>(reg, rb, len, lane, al, be, ga, de);
      Row<T> F, L;
      chunk_reduce<T, 8>(al, be, ga, de, F, L);
      T xF, xL;
      warp_block_finish(F, L, brow[8 * blk], brow[8 * blk + 1], lane, xF, xL);
      chunk_backsub<T, 8>(al, ga, de, xF, xL);
      vl_store<T, 8>(A, reg, lo, rb, len, lane, de);
    }
    __syncthreads();  // brow is rewritten by the next system
  }
}

template <typename T>
static cudaError_t launch_varlen_long(const VLArgs<T> &A, const int *list, const unsigned *count,
                                      cudaStream_t st) {
  const int smem = kVLLongWarps * 5 * kVLRegion * (int)sizeof(T);
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  static int per_sm[64];
  if (per_sm[dev] == 0) {
    e = cudaFuncSetAttribute(varlen_long_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
    if (e != cudaSuccess) return e;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, varlen_long_kernel<T>,
                                                      kVLLongWarps * 32, smem) != cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      nb = 1;
    }
    per_sm[dev] = nb;
  }
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  varlen_long_kernel<T><<<(unsigned)(sms * per_sm[dev]), kVLLongWarps * 32, smem, st>>>(A, list,
                                                                                       count);
  return cudaGetLastError();
}

template <typename T>
static int varlen_smem_bytes() {
  return kVLWarps * 5 * kVLRegion * (int)sizeof(T);
}

// Residency of the persistent kernel on the current device (sets the
// shared-memory attribute once per device).
template <typename T>
static cudaError_t varlen_grid(int &grid) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  static bool attr_set[64] = {};
  if (!attr_set[dev]) {
    e = cudaFuncSetAttribute(varlen_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             varlen_smem_bytes<T>());
    if (e != cudaSuccess) return e;
    attr_set[dev] = true;
  }
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, varlen_kernel<T>, kVLWarps * 32,
                                                    varlen_smem_bytes<T>()) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  grid = sms * per_sm;
  return cudaSuccess;
}

template <typename T>
cudaError_t launch_varlen(const T *a, const T *b, const T *c, T *d, const int64_t *offsets,
                          int64_t nsys, int64_t total, unsigned *err, cudaStream_t st) {
  // scratch: item_off and fitem_off (nsys+1 each), sys_count, queues, block
  // rows (8 per item), item_sys and fitem_sys (one int per item each)
  const int64_t max_items = varlen_cap(nsys, total);
  const size_t b_off = sizeof(int64_t) * (size_t)(nsys + 1);
  const size_t b_cnt = sizeof(unsigned) * (size_t)(nsys + 1);
  const size_t b_q = 64;
  const size_t b_rows = sizeof(T) * 8 * (size_t)max_items;
  const size_t b_map = sizeof(int) * (size_t)max_items;
  const size_t b_bsum = sizeof(int64_t) * 2 * (size_t)((nsys + kPrepThreads - 1) / kPrepThreads);
  const size_t b_mid = sizeof(int) * (kVarlenCtaBuckets + 1) * (size_t)nsys;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t at_bsum = 2 * al(b_off) + al(b_cnt) + al(b_q) + al(b_rows) + 2 * al(b_map);
  const size_t at_mid = at_bsum + al(b_bsum);
  unsigned char *w = (unsigned char *)scratch(at_mid + al(b_mid) + 256, 0);
  if (!w) return cudaErrorMemoryAllocation;
  int64_t *bsum = (int64_t *)(w + at_bsum);
  int *mid_list = (int *)(w + at_mid);
  unsigned *mid_count = (unsigned *)(w + at_mid + al(b_mid));
  VLArgs<T> A;
  A.a = a;
  A.b = b;
  A.c = c;
  A.d = d;
  A.offsets = offsets;
  A.nsys = nsys;
  A.total = total;
  A.cap = max_items;
  varlen_buckets((int)sizeof(T), A.m2max, A.m4max);
  A.item_off = (int64_t *)w;
  A.fitem_off = (int64_t *)(w + al(b_off));
  A.sys_count = (unsigned *)(w + 2 * al(b_off));
  A.queue = (unsigned long long *)(w + 2 * al(b_off) + al(b_cnt));
  A.rows = (T *)(w + 2 * al(b_off) + al(b_cnt) + al(b_q));
  A.item_sys = (const int *)(w + 2 * al(b_off) + al(b_cnt) + al(b_q) + al(b_rows));
  A.fitem_sys = A.item_sys + al(b_map) / sizeof(int);
  A.err = err;
  int grid = 0;
  cudaError_t e = varlen_grid<T>(grid);
  if (e != cudaSuccess) return e;
  e = launch_varlen_prep(offsets, nsys, total, bsum, (int64_t *)A.item_off,
                         (int64_t *)A.fitem_off, (int *)A.item_sys, (int *)A.fitem_sys,
                         A.sys_count, A.queue, mid_list, mid_count, err, st);
  if (e != cudaSuccess) return e;
  e = launch_xcta_varlen<T>(a, b, c, d, offsets, mid_list, nsys, mid_count, st);
  if (e != cudaSuccess) return e;
  e = launch_varlen_long<T>(A, mid_list + (size_t)kVarlenCtaBuckets * nsys,
                            mid_count + kVarlenCtaBuckets, st);
  if (e != cudaSuccess) return e;
  varlen_kernel<T><<<dim3((unsigned)grid), dim3(kVLWarps * 32), varlen_smem_bytes<T>(), st>>>(A);
  return cudaGetLastError();
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
// item prefix sums, per-system counters, work queue, block rows and an error
// word) lives in the fixed array below, which every GPU that loads this
// library holds until the process exits.  Nothing is allocated per call.
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

// Bytes of work space a solve of nsys systems / total rows needs (0 when it
// does not fit in the static array).
static size_t noalloc_layout(int64_t nsys, int64_t total, size_t off[6]) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const int64_t max_items = varlen_cap(nsys, total);
  size_t at = 0;
  off[0] = at;  // error word (read and cleared by tridGetDeviceErrors)
  at += 256;
  off[1] = at;  // item_off and fitem_off, nsys+1 int64 each
  at += 2 * al(sizeof(int64_t) * (size_t)(nsys + 1));
  off[2] = at;  // sys_count, nsys+1 unsigned
  at += al(sizeof(unsigned) * (size_t)(nsys + 1));
  off[3] = at;  // queue
  at += 256;
  off[4] = at;  // block rows, 8 per item; then item_sys and fitem_sys; then
                // the preparation's per-CTA sums
  at += al(sizeof(double) * 8 * (size_t)max_items) + 2 * al(sizeof(int) * (size_t)max_items);
  at += al(sizeof(int64_t) * 2 * (size_t)((nsys + kPrepThreads - 1) / kPrepThreads));
  off[5] = at;  // the CTA classes: counters, then kVarlenCtaBuckets+1 lists of nsys
  at += 256 + al(sizeof(int) * (kVarlenCtaBuckets + 1) * (size_t)nsys);
  return at <= kNoAllocScratchBytes ? at : 0;
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
  size_t off[6];
  if (noalloc_layout(nsys, total, off) == 0) return TRID_STATUS_INVALID_VALUE;  // too large
  unsigned char *w = (unsigned char *)noalloc_scratch_address();
  if (!w) return TRID_STATUS_EXECUTION_FAILED;
  const cudaStream_t st = current_stream();
  VLArgs<double> A;
  A.a = a;
  A.b = b;
  A.c = c;
  A.d = d;
  A.offsets = (const int64_t *)offsets;
  A.nsys = nsys;
  A.total = total;
  A.cap = varlen_cap(nsys, total);
  varlen_buckets((int)sizeof(double), A.m2max, A.m4max);
  A.err = (unsigned *)(w + off[0]);
  A.item_off = (int64_t *)(w + off[1]);
  A.fitem_off = (int64_t *)(w + off[1] + (off[2] - off[1]) / 2);
  A.sys_count = (unsigned *)(w + off[2]);
  A.queue = (unsigned long long *)(w + off[3]);
  A.rows = (double *)(w + off[4]);
  int64_t *bsum = nullptr;
  {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const int64_t max_items = A.cap;
    A.item_sys = (const int *)(w + off[4] + al(sizeof(double) * 8 * (size_t)max_items));
    A.fitem_sys = A.item_sys + al(sizeof(int) * (size_t)max_items) / sizeof(int);
    bsum = (int64_t *)(w + off[4] + al(sizeof(double) * 8 * (size_t)max_items) +
                       2 * al(sizeof(int) * (size_t)max_items));
  }
  // the preparation rewrites the prefix sums and clears the queues and counters,
  // so whatever the previous call left in the array does not matter
  int grid = 0;
  if (varlen_grid<double>(grid) != cudaSuccess) return TRID_STATUS_EXECUTION_FAILED;
  unsigned *mid_count = (unsigned *)(w + off[5]);
  int *mid_list = (int *)(w + off[5] + 256);
  if (launch_varlen_prep(A.offsets, nsys, total, bsum, (int64_t *)A.item_off,
                         (int64_t *)A.fitem_off, (int *)A.item_sys, (int *)A.fitem_sys,
                         A.sys_count, A.queue, mid_list, mid_count, A.err, st) != cudaSuccess)
    return TRID_STATUS_EXECUTION_FAILED;
  if (launch_xcta_varlen<double>(a, b, c, d, A.offsets, mid_list, nsys, mid_count, st) !=
          cudaSuccess ||
      launch_varlen_long<double>(A, mid_list + (size_t)kVarlenCtaBuckets * nsys,
                                 mid_count + kVarlenCtaBuckets, st) != cudaSuccess)
    return TRID_STATUS_EXECUTION_FAILED;
  varlen_kernel<double><<<dim3((unsigned)grid), dim3(kVLWarps * 32), varlen_smem_bytes<double>(),
                          st>>>(A);
  return cudaGetLastError() == cudaSuccess ? TRID_STATUS_SUCCESS : TRID_STATUS_EXECUTION_FAILED;
}
