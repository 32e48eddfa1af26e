// Variable-length packed batch: one persistent launch (sm_100a).
//
// System s occupies rows [offsets[s], offsets[s+1]) of every array (unit
// stride, int64 offsets).  Work items:
//   * a system of at most 256 rows is one item, solved whole by one warp with
//     the partitioned Thomas of partition.cuh; the rows-per-lane chunk M is
//     picked per item from the length (2/4/8: the length buckets);
//   * a longer system (up to 32 blocks of 256 rows = 8192 rows) is one item
//     per block.  A warp reduces its block to the block's two boundary rows
//     (warp_block_basis / block_rows), publishes them, and counts the block
//     done on the system's atomic counter; the warp that completes the count
//     solves the system's block system (2 rows per block, one warp interface
//     solve) and then finishes every block of the system (back-substitution
//     from the block's boundary unknowns).  Nothing ever waits on another
//     warp: completion is detected by the counter, never polled.
// Warps take items from one atomic queue in system order.
//
// varlen_prep (one CTA) turns offsets into the item prefix sums and clears
// the queue and the per-system counters.  Malformed offsets (decreasing or
// past `total`) and systems longer than 8192 rows are skipped and recorded in
// the device error word (bits 4 and 8).
#include <mutex>

#include "partition.cuh"

namespace tridb200 {

constexpr int kVLBlock = 256;   // rows per block of a long system (M = 8)
constexpr int kVLShort = 256;   // longest system solved as one item
constexpr int kVLMaxBlocks = 32;
constexpr unsigned kErrBadOffsets = 4u;
constexpr unsigned kErrTooLong = 8u;

__device__ __forceinline__ int64_t vl_items(int64_t len) {
  if (len <= kVLShort) return 1;
  return (len + kVLBlock - 1) / kVLBlock;
}

// Exclusive prefix of items per system into item_off[0..nsys]; clears queue
// and counters.  One CTA of 1024 threads.
__global__ void __launch_bounds__(1024) varlen_prep(const int64_t *__restrict__ offsets, int64_t nsys,
                                                    int64_t total, int64_t *__restrict__ item_off,
                                                    unsigned *__restrict__ sys_count,
                                                    unsigned long long *__restrict__ queue) {
  __shared__ int64_t part[1024];
  const int tid = threadIdx.x;
  const int64_t per = (nsys + 1023) / 1024;
  const int64_t s0 = tid * per, s1 = (s0 + per < nsys) ? s0 + per : nsys;
  int64_t acc = 0;
  for (int64_t s = s0; s < s1; ++s) {
    int64_t len = offsets[s + 1] - offsets[s];
    if (len < 0 || offsets[s] < 0 || offsets[s + 1] > total) len = 0;
    acc += vl_items(len > 0 ? len : 1);
    sys_count[s] = 0u;
  }
  part[tid] = acc;
  __syncthreads();
  if (tid == 0) {
    int64_t run = 0;
    for (int k = 0; k < 1024; ++k) {
      const int64_t v = part[k];
      part[k] = run;
      run += v;
    }
    item_off[nsys] = run;
    *queue = 0ull;
  }
  __syncthreads();
  int64_t run = part[tid];
  for (int64_t s = s0; s < s1; ++s) {
    item_off[s] = run;
    int64_t len = offsets[s + 1] - offsets[s];
    if (len < 0 || offsets[s] < 0 || offsets[s + 1] > total) len = 0;
    run += vl_items(len > 0 ? len : 1);
  }
}

template <typename T>
struct VLArgs {
  const T *a, *b, *c;
  T *d;
  const int64_t *offsets;
  const int64_t *item_off;
  int64_t nsys;
  int64_t total;
  unsigned *sys_count;
  unsigned long long *queue;
  T *rows;       // block rows: item index * 8
  unsigned *err;
};

template <typename T, int M>
__device__ __forceinline__ void vl_load(const VLArgs<T> &A, int64_t lo, int64_t len, int64_t r0,
                                        T (&al)[M], T (&be)[M], T (&ga)[M], T (&de)[M]) {
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int64_t r = r0 + j;
    if (r < len) {
      al[j] = (r == 0) ? T(0) : A.a[lo + r];
      be[j] = A.b[lo + r];
      ga[j] = (r == len - 1) ? T(0) : A.c[lo + r];
      de[j] = A.d[lo + r];
    } else {
      al[j] = T(0);
      be[j] = T(1);
      ga[j] = T(0);
      de[j] = T(0);
    }
  }
}

template <typename T, int M>
__device__ __forceinline__ void vl_short(const VLArgs<T> &A, int64_t lo, int64_t len, int lane) {
  T al[M], be[M], ga[M], de[M];
  const int64_t r0 = (int64_t)lane * M;
  vl_load<T, M>(A, lo, len, r0, al, be, ga, de);
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  T xF, xL;
  warp_interface_solve(F, L, xF, xL, lane);
  chunk_backsub<T, M>(al, ga, de, xF, xL);
#pragma unroll
  for (int j = 0; j < M; ++j)
    if (r0 + j < len) A.d[lo + r0 + j] = de[j];
}

// one block of a long system: chunk reduction + block basis
template <typename T>
__device__ __forceinline__ void vl_block(const VLArgs<T> &A, int64_t lo, int64_t len, int blk,
                                         int lane, T (&al)[8], T (&ga)[8], T (&de)[8], Row<T> &F,
                                         Row<T> &L, T (&bF)[3], T (&bL)[3]) {
  T be[8];
  vl_load<T, 8>(A, lo, len, (int64_t)blk * kVLBlock + lane * 8, al, be, ga, de);
  chunk_reduce<T, 8>(al, be, ga, de, F, L);
  warp_block_basis(F, L, lane, bF, bL);
}

template <typename T>
__global__ void __launch_bounds__(256, 2) varlen_kernel(VLArgs<T> A) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t nitems = A.item_off[A.nsys];
  for (;;) {
    unsigned long long it = 0;
    if (lane == 0) it = atomicAdd(A.queue, 1ull);
    it = __shfl_sync(0xffffffffu, it, 0);
    if ((int64_t)it >= nitems) break;
    // system of this item: last s with item_off[s] <= it
    int64_t lo_s = 0, hi_s = A.nsys;  // item_off[lo_s] <= it < item_off[hi_s]
    while (hi_s - lo_s > 1) {
      const int64_t mid = (lo_s + hi_s) / 2;
      if (A.item_off[mid] <= (int64_t)it) lo_s = mid; else hi_s = mid;
    }
    const int64_t s = lo_s;
    const int64_t lo = A.offsets[s], hi = A.offsets[s + 1];
    const int64_t len = hi - lo;
    if (len < 0 || lo < 0 || hi > A.total) {
      if (lane == 0) atomicOr(A.err, kErrBadOffsets);
      continue;
    }
    if (len == 0) continue;
    if (len <= kVLShort) {
      if (len <= 64)
        vl_short<T, 2>(A, lo, len, lane);
      else if (len <= 128)
        vl_short<T, 4>(A, lo, len, lane);
      else
        vl_short<T, 8>(A, lo, len, lane);
      continue;
    }
    const int nblk = (int)((len + kVLBlock - 1) / kVLBlock);
    if (nblk > kVLMaxBlocks) {
      if (lane == 0 && it == (unsigned long long)A.item_off[s]) atomicOr(A.err, kErrTooLong);
      continue;
    }
    const int blk = (int)((int64_t)it - A.item_off[s]);
    T al[8], ga[8], de[8], bF[3], bL[3];
    Row<T> F, L, FB, LB;
    vl_block<T>(A, lo, len, blk, lane, al, ga, de, F, L, bF, bL);
    block_rows(F, L, bF, bL, lane, FB, LB);
    T *rw = A.rows + ((int64_t)A.item_off[s] + blk) * 8;
    if (lane == 0) {
      rw[0] = FB.a; rw[1] = FB.b; rw[2] = FB.c; rw[3] = FB.d;
      rw[4] = LB.a; rw[5] = LB.b; rw[6] = LB.c; rw[7] = LB.d;
    }
    __threadfence();  // publish the block rows before counting the block done
    unsigned done = 0;
    if (lane == 0) done = atomicAdd(&A.sys_count[s], 1u);
    done = __shfl_sync(0xffffffffu, done, 0);
    if (done != (unsigned)(nblk - 1)) continue;
    __threadfence();  // every block's rows are visible to this warp now
    // the block system of s: lane t holds block t's two rows
    const T *rs = A.rows + (int64_t)A.item_off[s] * 8;
    Row<T> RF{T(0), T(1), T(0), T(0)}, RL{T(0), T(1), T(0), T(0)};
    if (lane < nblk) {
      const T *q = rs + (int64_t)lane * 8;
      RF = {__ldcg(q + 0), __ldcg(q + 1), __ldcg(q + 2), __ldcg(q + 3)};
      RL = {__ldcg(q + 4), __ldcg(q + 5), __ldcg(q + 6), __ldcg(q + 7)};
    }
    T fB, lB;
    warp_interface_solve(RF, RL, fB, lB, lane);
    // finish every block of s
    for (int t = 0; t < nblk; ++t) {
      vl_block<T>(A, lo, len, t, lane, al, ga, de, F, L, bF, bL);
      const T f = __shfl_sync(0xffffffffu, fB, t);
      const T l = __shfl_sync(0xffffffffu, lB, t);
      const T xF = bF[0] + f * bF[1] + l * bF[2];
      const T xL = bL[0] + f * bL[1] + l * bL[2];
      chunk_backsub<T, 8>(al, ga, de, xF, xL);
      const int64_t r0 = (int64_t)t * kVLBlock + lane * 8;
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (r0 + j < len) A.d[lo + r0 + j] = de[j];
    }
  }
}

template <typename T>
cudaError_t launch_varlen(const T *a, const T *b, const T *c, T *d, const int64_t *offsets,
                          int64_t nsys, int64_t total, unsigned *err, cudaStream_t st) {
  // scratch: item_off (nsys+1), sys_count (nsys), queue, block rows
  const int64_t max_items = nsys + total / kVLBlock + 1;
  const size_t b_off = sizeof(int64_t) * (size_t)(nsys + 1);
  const size_t b_cnt = sizeof(unsigned) * (size_t)(nsys + 1);
  const size_t b_q = 64;
  const size_t b_rows = sizeof(T) * 8 * (size_t)max_items;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  unsigned char *w = (unsigned char *)scratch(al(b_off) + al(b_cnt) + al(b_q) + al(b_rows), 0);
  if (!w) return cudaErrorMemoryAllocation;
  VLArgs<T> A;
  A.a = a;
  A.b = b;
  A.c = c;
  A.d = d;
  A.offsets = offsets;
  A.nsys = nsys;
  A.total = total;
  A.item_off = (int64_t *)w;
  A.sys_count = (unsigned *)(w + al(b_off));
  A.queue = (unsigned long long *)(w + al(b_off) + al(b_cnt));
  A.rows = (T *)(w + al(b_off) + al(b_cnt) + al(b_q));
  A.err = err;
  varlen_prep<<<1, 1024, 0, st>>>(offsets, nsys, total, (int64_t *)A.item_off, A.sys_count, A.queue);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, varlen_kernel<T>, 256, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  varlen_kernel<T><<<dim3((unsigned)(sms * per_sm)), dim3(256), 0, st>>>(A);
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
  if (nsys > ((int64_t)1 << 40)) return TRID_STATUS_INVALID_VALUE;
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

// Bytes of work space a solve of nsys systems / total rows needs (0 when it
// does not fit in the static array).
static size_t noalloc_layout(int64_t nsys, int64_t total, size_t off[5]) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const int64_t max_items = nsys + total / kVLBlock + 1;
  size_t at = 0;
  off[0] = at;  // error word
  at += 256;
  off[1] = at;  // item_off, nsys+1 int64
  at += al(sizeof(int64_t) * (size_t)(nsys + 1));
  off[2] = at;  // sys_count, nsys+1 unsigned
  at += al(sizeof(unsigned) * (size_t)(nsys + 1));
  off[3] = at;  // queue
  at += 256;
  off[4] = at;  // block rows, 8 per item
  at += al(sizeof(double) * 8 * (size_t)max_items);
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
  if (nsys > ((int64_t)1 << 40) || total > ((int64_t)1 << 46)) return TRID_STATUS_INVALID_VALUE;
  size_t off[5];
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
  A.err = (unsigned *)(w + off[0]);
  A.item_off = (int64_t *)(w + off[1]);
  A.sys_count = (unsigned *)(w + off[2]);
  A.queue = (unsigned long long *)(w + off[3]);
  A.rows = (double *)(w + off[4]);
  // varlen_prep rewrites the prefix sums and clears the queue and counters,
  // so whatever the previous call left in the array does not matter
  varlen_prep<<<1, 1024, 0, st>>>(A.offsets, nsys, total, (int64_t *)A.item_off, A.sys_count,
                                   A.queue);
  if (cudaGetLastError() != cudaSuccess) return TRID_STATUS_EXECUTION_FAILED;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, varlen_kernel<double>, 256, 0) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  varlen_kernel<double><<<dim3((unsigned)(sms * per_sm)), dim3(256), 0, st>>>(A);
  return cudaGetLastError() == cudaSuccess ? TRID_STATUS_SUCCESS : TRID_STATUS_EXECUTION_FAILED;
}
