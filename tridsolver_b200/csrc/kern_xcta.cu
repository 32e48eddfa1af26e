// Axis-0 systems of one CTA (sm_100a): the blocked partition of
// kern_general.cu kept inside one CTA, so systems of up to 4096 rows are
// solved in one launch without re-reading anything.
//
// CTA = one system, W <= 16 warps; warp w owns block w (32 chunks of M rows,
// M = 4, 8 or 16).
// Every warp reduces its chunks (chunk_reduce) and its block
// (warp_block_basis + block_rows); the 2W block rows meet in shared memory,
// warp 0 solves the block system (one warp interface solve, lane = block),
// and every warp finishes its block from its two boundary unknowns.  A
// system of one block skips the block level.
//
// Modes:
//   kXFwd / kXFwdInc : x = A^{-1} d into d / added into u;
//   kXAdj            : the adjoint for a given solution u and cotangent w
//                      (transposed system solved in place, gradients formed
//                      in the same pass);
//   kXFused          : forward and adjoint of the linear loss <w, x> in one
//                      pass: reads a, b, c, d, w once and writes x, da, db,
//                      dc, dd (10 values per unknown instead of 5 + 9); the
//                      transposed chunk reductions reuse the forward pivots.
#include "partition.cuh"

namespace tridb200 {

// XArgs (trid_internal.cuh): d = forward RHS (unused by kXAdj); w = adjoint
// cotangent (kXAdj, kXFused); usol = forward solution (kXAdj); x = solution
// (kXFwd, kXFused) or u (+=, kXFwdInc); ga..gd = gradients, each may be null.
constexpr int kXFwd = kXcFwd, kXFwdInc = kXcFwdInc, kXAdj = kXcAdj, kXFused = kXcFused;

// Solve the system held in (al, be, ga, de) across the CTA; the solution
// overwrites de.  Whole CTA must call it (barriers inside).
// The part of cta_solve after the chunk reduction (F, L: this thread's
// interface rows; al/ga/de: its reduced chunk).
template <typename T, int M>
__device__ __forceinline__ void cta_solve_rows(const Row<T> &F, const Row<T> &L, T (&al)[M],
                                               T (&ga)[M], T (&de)[M], int w, int lane, int nw,
                                               T *sm);

template <typename T, int M>
__device__ __forceinline__ void cta_solve(T (&al)[M], const T (&be)[M], T (&ga)[M], T (&de)[M],
                                          int w, int lane, int nw, T *sm) {
  Row<T> F, L;
  T rp[M];
  chunk_reduce_cont<T, M>(al, be, ga, de, F, L, rp);
  cta_solve_rows<T, M>(F, L, al, ga, de, w, lane, nw, sm);
}

template <typename T, int M>
__device__ __forceinline__ void cta_solve_rows(const Row<T> &F, const Row<T> &L, T (&al)[M],
                                               T (&ga)[M], T (&de)[M], int w, int lane, int nw,
                                               T *sm) {
  if (nw == 1) {  // one block: the warp's interface system is the whole system
    T xF, xL;
    warp_interface_solve(F, L, xF, xL, lane);
    chunk_backsub<T, M>(al, ga, de, xF, xL);
    return;
  }
  T bF[3], bL[3];
  warp_block_basis(F, L, lane, bF, bL);
  Row<T> FB, LB;
  block_rows(F, L, bF, bL, lane, FB, LB);
  // sm layout: [0, 8*16) block rows, [128, 128 + 2*16) block unknowns
  if (lane == 0) {
    T *q = sm + 8 * w;
    q[0] = FB.a; q[1] = FB.b; q[2] = FB.c; q[3] = FB.d;
    q[4] = LB.a; q[5] = LB.b; q[6] = LB.c; q[7] = LB.d;
  }
  __syncthreads();
  if (w == 0) {
    Row<T> RF{T(0), T(1), T(0), T(0)}, RL{T(0), T(1), T(0), T(0)};
    if (lane < nw) {
      const T *q = sm + 8 * lane;
      RF = {q[0], q[1], q[2], q[3]};
      RL = {q[4], q[5], q[6], q[7]};
    }
    T f, l;
    int span = 1;  // lanes with block rows, rounded up to a power of two
    while (span < nw) span <<= 1;
    warp_interface_solve(RF, RL, f, l, lane, span);
    if (lane < nw) {
      sm[128 + 2 * lane] = f;
      sm[128 + 2 * lane + 1] = l;
    }
  }
  __syncthreads();
  const T f = sm[128 + 2 * w], l = sm[128 + 2 * w + 1];
  const T xF = bF[0] + f * bF[1] + l * bF[2];
  const T xL = bL[0] + f * bL[1] + l * bL[2];
  chunk_backsub<T, M>(al, ga, de, xF, xL);
  __syncthreads();  // sm is reused by the caller's next solve
}

// Staging: every array of the system is copied into shared memory with
// coalesced 4/8-byte cp.async (row r of a warp's 32*M rows at q + q/M, one
// pad element per M rows, so that the transposed reads -- lane L takes rows
// L*M .. L*M+M-1 -- hit 32 distinct banks), and results leave the same way:
// written transposed into the warp's region, stored coalesced.
template <int M>
__device__ __forceinline__ int pidx(int q) {
  return q + q / M;
}

template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int sz = valid ? (int)sizeof(T) : 0;  // 0: zero-fill, nothing read
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(sz)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(sz)
                 : "memory");
}

template <typename T, int M>
struct Stage {
  T *base;  // dynamic shared memory
  int nw;   // warps of the CTA
  static constexpr int R = 32 * (M + 1);  // elements per warp region
  __device__ T *region(int k, int w) const { return base + ((size_t)k * nw + w) * R; }
  // element of system row r in staged array k (any warp's region)
  __device__ T &row(int k, int r) const {
    const int wr = r / (32 * M);
    return region(k, wr)[pidx<M>(r - wr * 32 * M)];
  }
};

// FULL: n is a whole number of warp blocks (no row past n anywhere)
template <typename T, int M, bool FULL = false>
__device__ __forceinline__ void stage_in(const Stage<T, M> &S, int k, int w, int lane, const T *p,
                                         int n) {
  T *reg = S.region(k, w);
  const int wb = w * 32 * M;
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int q = j * kWarp + lane;
    const bool in = FULL || wb + q < n;
    cp_async_elem(reg + pidx<M>(q), in ? p + wb + q : p, in);
  }
}

// v (rows lane*M + j of warp w) -> region k -> coalesced store to p (ADD: +=)
template <typename T, int M, bool ADD, bool FULL = false>
__device__ __forceinline__ void stage_out(const Stage<T, M> &S, int k, int w, int lane,
                                          const T (&v)[M], T *p, int n) {
  T *reg = S.region(k, w);
#pragma unroll
  for (int j = 0; j < M; ++j) reg[lane * (M + 1) + j] = v[j];
  __syncwarp();
  const int wb = w * 32 * M;
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int q = j * kWarp + lane;
    if (FULL || wb + q < n) {
      if (ADD)
        p[wb + q] += reg[pidx<M>(q)];
      else
        p[wb + q] = reg[pidx<M>(q)];
    }
  }
}

// Warm L2 with the system `dist` CTAs ahead (half a resident set ahead: its
// rows arrive well before their CTA starts, without crowding L2): one bulk
// prefetch per array, so that DRAM keeps streaming while the resident CTAs
// compute.  Needs 16-byte aligned rows of a
// whole number of 16-byte units.
template <typename T>
__device__ __forceinline__ void prefetch_system_l2(const T *p, int n) {
  const uint32_t bytes = (uint32_t)n * sizeof(T);
  if (((uintptr_t)p & 15) == 0 && (bytes & 15) == 0)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// One system of n rows whose arrays start at off[] (rows past n are
// identity rows), solved by the whole CTA: the body of the strided-batch
// kernel below and of the variable-length batch's one-CTA systems
// (kern_varlen.cu).  prefetch() runs on every thread once the system's
// copies are issued.  n <= blockDim.x / 32 * 32 * M.
template <typename T, int M, int MODE, bool FULL, typename PF>
__device__ __forceinline__ void xcta_system(const XArgs<T> &A, const int64_t (&off)[5], const int n,
                                            PF &&prefetch) {
  extern __shared__ __align__(16) unsigned char xcta_dyn[];
  __shared__ T sm[128 + 32 + 2 * 16];
  const int lane = threadIdx.x & (kWarp - 1);
  const int w = threadIdx.x / kWarp;
  const int nw = blockDim.x / kWarp;
  const int r0 = w * kWarp * M + lane * M;
  const Stage<T, M> S{reinterpret_cast<T *>(xcta_dyn), nw};
  // staged arrays: 0 a, 1 b, 2 c, 3 d (forward modes) or the solution
  // (kXAdj), 4 w (kXAdj, kXFused)
  constexpr bool kHasW = (MODE == kXAdj || MODE == kXFused);
  stage_in<T, M, FULL>(S, 0, w, lane, A.a + off[kA], n);
  stage_in<T, M, FULL>(S, 1, w, lane, A.b + off[kB], n);
  stage_in<T, M, FULL>(S, 2, w, lane, A.c + off[kC], n);
  if (MODE == kXAdj)
    stage_in<T, M, FULL>(S, 3, w, lane, A.usol + off[kU], n);
  else
    stage_in<T, M, FULL>(S, 3, w, lane, A.d + off[kD], n);
  if (kHasW) stage_in<T, M, FULL>(S, 4, w, lane, A.w + off[kD], n);
  prefetch();
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();  // neighbouring rows are read across warp regions

  const T *ra = S.region(0, w) + lane * (M + 1);
  const T *rb = S.region(1, w) + lane * (M + 1);
  const T *rc = S.region(2, w) + lane * (M + 1);
  const T *rd = S.region(3, w) + lane * (M + 1);

  T gsol[M];  // the adjoint solution
  T xs[M];    // the forward solution
  if (MODE == kXAdj) {
    // transposed rows: sub-diagonal c_{r-1}, super-diagonal a_{r+1}
    const T *rw = S.region(4, w) + lane * (M + 1);
    T ta[M], be[M], tg[M];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int r = r0 + j;
      const bool in = FULL || r < n;
      ta[j] = (in && r > 0) ? (j > 0 ? rc[j - 1] : S.row(2, r - 1)) : T(0);
      tg[j] = (r + 1 < n) ? (j < M - 1 ? ra[j + 1] : S.row(0, r + 1)) : T(0);
      be[j] = in ? rb[j] : T(1);
      gsol[j] = rw[j];  // zero-filled past n
    }
    cta_solve<T, M>(ta, be, tg, gsol, w, lane, nw, sm);
#pragma unroll
    for (int j = 0; j < M; ++j) xs[j] = rd[j];
  } else {
    // forward rows
    T al[M], be[M], ga[M], rp[M];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int r = r0 + j;
      const bool in = FULL || r < n;
      al[j] = (in && r > 0) ? ra[j] : T(0);
      be[j] = in ? rb[j] : T(1);
      ga[j] = (r < n - 1) ? rc[j] : T(0);
      xs[j] = rd[j];  // zero-filled past n
    }
    if (MODE == kXFused) {
      Row<T> F, L;
      chunk_reduce_cont<T, M>(al, be, ga, xs, F, L, rp);
      // the transposed reduction needs b only at the chunk's first and last
      // rows, where it stays in this thread's own b slots (read by this
      // thread alone); the interior pivots wait in the other slots, so that
      // neither occupies registers meanwhile
      T *rbw = S.region(1, w) + lane * (M + 1);
#pragma unroll
      for (int j = 1; j <= M - 2; ++j) rbw[j] = rp[j];
      cta_solve_rows<T, M>(F, L, al, ga, xs, w, lane, nw, sm);
      // x into this thread's own slots of region 3 (d was read by this
      // thread alone): the neighbours x_{r-1}, x_{r+1} and the outgoing x
      T *rx = S.region(3, w) + lane * (M + 1);
#pragma unroll
      for (int j = 0; j < M; ++j) rx[j] = xs[j];
      // x leaves now (coalesced from the warp's own region), its stores
      // overlapping the transposed solve
      __syncwarp();
      {
        const T *reg = S.region(3, w);
        const int wb = w * 32 * M;
#pragma unroll
        for (int j = 0; j < M; ++j) {
          const int q = j * kWarp + lane;
          if (FULL || wb + q < n) A.x[off[kD] + wb + q] = reg[pidx<M>(q)];
        }
      }
      // the transposed system: rows (c_{r-1}, b_r, a_{r+1}); its chunk
      // interiors have the forward pivots
      const T *rw = S.region(4, w) + lane * (M + 1);
      T ta[M], tg[M], tb[M], tp[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const int r = r0 + j;
        const bool in = FULL || r < n;
        ta[j] = (in && r > 0) ? (j > 0 ? rc[j - 1] : S.row(2, r - 1)) : T(0);
        tg[j] = (r + 1 < n) ? (j < M - 1 ? ra[j + 1] : S.row(0, r + 1)) : T(0);
        gsol[j] = rw[j];  // zero-filled past n
        // interior b unused; rows past n are identity rows (staged b is 0 there)
        tb[j] = ((j == 0 || j == M - 1) && in) ? rbw[j] : T(1);
        tp[j] = (j >= 1 && j <= M - 2) ? rbw[j] : T(0);
      }
      chunk_reduce_given<T, M>(ta, tb, tg, gsol, F, L, tp);
      cta_solve_rows<T, M>(F, L, ta, tg, gsol, w, lane, nw, sm);
    } else {
      cta_solve<T, M>(al, be, ga, xs, w, lane, nw, sm);
    }
  }

  if (MODE == kXFwd) {
    stage_out<T, M, false, FULL>(S, 3, w, lane, xs, A.x + off[kD], n);
    return;
  }
  if (MODE == kXFwdInc) {
    stage_out<T, M, true, FULL>(S, 3, w, lane, xs, A.x + off[kU], n);
    return;
  }
  // gradients: x_{r-1} and x_{r+1} from the staged solution (region 3)
  __syncthreads();
  if (MODE == kXFused) {
    const T *rx = S.region(3, w) + lane * (M + 1);
#pragma unroll
    for (int j = 0; j < M; ++j) xs[j] = rx[j];
  }
  const T xprev = (r0 > 0 && r0 - 1 < n) ? S.row(3, r0 - 1) : T(0);
  const T xnext = (r0 + M < n) ? S.row(3, r0 + M) : T(0);
  T v[M];
  if (A.ga) {
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const T xm = (j > 0) ? xs[j - 1] : xprev;
      v[j] = (r0 + j > 0) ? -gsol[j] * xm : T(0);
    }
    stage_out<T, M, false, FULL>(S, 0, w, lane, v, A.ga + off[kA], n);
  }
  if (A.gb) {
#pragma unroll
    for (int j = 0; j < M; ++j) v[j] = -gsol[j] * xs[j];
    stage_out<T, M, false, FULL>(S, 1, w, lane, v, A.gb + off[kB], n);
  }
  if (A.gc) {
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const T xp = (j < M - 1) ? xs[j + 1] : xnext;
      v[j] = (r0 + j + 1 < n) ? -gsol[j] * xp : T(0);
    }
    stage_out<T, M, false, FULL>(S, 2, w, lane, v, A.gc + off[kC], n);
  }
  if (A.gd) stage_out<T, M, false, FULL>(S, 4, w, lane, gsol, A.gd + off[kD], n);
}

// The strided-batch kernel: CTA = system blockIdx.x; thread 0 warms L2 with
// the system `dist` CTAs ahead.  Register use bounded by its launch bounds
// (MAXW warps, MINB CTAs per SM).
template <typename T, int M, int MODE, int MAXW, int MINB, bool FULL>
__global__ void __launch_bounds__(MAXW * 32, MINB) xcta_kernel(Geom g, XArgs<T> A, int dist) {
  int64_t off[5];
  system_offsets(g, (int64_t)blockIdx.x, off);
  const int n = g.n;
  xcta_system<T, M, MODE, FULL>(A, off, n, [&] {
    if (dist > 0 && threadIdx.x == 0 && blockIdx.x + (int64_t)dist < g.nsys) {
      constexpr bool kHasW = (MODE == kXAdj || MODE == kXFused);
      int64_t po[5];
      system_offsets(g, blockIdx.x + (int64_t)dist, po);
      prefetch_system_l2(A.a + po[kA], n);
      prefetch_system_l2(A.b + po[kB], n);
      prefetch_system_l2(A.c + po[kC], n);
      prefetch_system_l2(MODE == kXAdj ? A.usol + po[kU] : A.d + po[kD], n);
      if (kHasW) prefetch_system_l2(A.w + po[kD], n);
    }
  });
}

template <typename T, int M, int MODE, auto kern>
static cudaError_t launch_xcta_k(int max_warps, const Geom &g, const XArgs<T> &A, int warps,
                                 cudaStream_t st) {
  constexpr int kArrays = (MODE == kXAdj || MODE == kXFused) ? 5 : 4;
  const size_t smem = (size_t)kArrays * warps * Stage<T, M>::R * sizeof(T);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 64) return cudaErrorNotSupported;
  static bool attr_set[64] = {};  // per device, per kernel (one instantiation each)
  if (!attr_set[dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kArrays * max_warps * Stage<T, M>::R * (int)sizeof(T));
    if (e != cudaSuccess) return e;
    attr_set[dev] = true;
  }
  // prefetch distance: half the CTAs resident on the whole GPU at once (16,384
  // systems of 1024 rows: the forward and forward+adjoint passes both run
  // fastest there; the full resident count is 2-6% slower, twice it 26-47%,
  // a quarter 2-14%, none 11-34%)
  int per_sm = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, warps * kWarp, smem) !=
          cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    per_sm = 0;
    cudaGetLastError();
  }
  kern<<<(unsigned)g.nsys, warps * kWarp, smem, st>>>(g, A, per_sm * sms / 2);
  return cudaGetLastError();
}

template <typename T, int M, int MODE, int MAXW, int MINB = 1, bool FULL = false>
static cudaError_t launch_xcta_m(const Geom &g, const XArgs<T> &A, int warps, cudaStream_t st) {
  return launch_xcta_k<T, M, MODE, xcta_kernel<T, M, MODE, MAXW, MINB, FULL>>(MAXW, g, A, warps,
                                                                            st);
}

template <typename T, int MODE>
cudaError_t launch_xcta(const Geom &g, const XArgs<T> &A, int chunk, cudaStream_t st) {
  // rows per thread M (chunk, or by length: 16 above 256 rows -- fewer warps
  // per system beat shorter chains on B200 at every length measured, 512 to
  // 4096 -- else 8 or 4); at most 16 warps, so n <= 512*M
  const int n = g.n;
  if (n > 4096 || g.nsys > 0x7fffffff) return cudaErrorNotSupported;
  if constexpr (MODE == kXFwd || MODE == kXFwdInc) {
    // 12 rows per lane (384 per warp) where that pads fewer rows than 16
    // and takes at most four warps: the kernel is issue-bound on row slots
    // (warps x 32 x M), not on the system's rows, e.g. 700 rows fill 768
    // slots instead of 1024 (B200, same box: 257 rows 4.04 -> 4.72 TB/s, 700
    // 4.64 -> 5.21, 1100 4.86 -> 5.49; with five 12-row warps, 1700 and 1920
    // rows ran 14-20% slower than four 16-row warps, so those keep 16)
    const int w12 = (n + 383) / 384, w16 = (n + 511) / 512;
    if (chunk == 0 && n > 256 && w12 <= 4 && w12 * 384 < w16 * 512) {
      const bool full12 = n == w12 * 384;
      if (w12 <= 2)
        return full12 ? launch_xcta_m<T, 12, MODE, 2, 6, true>(g, A, w12, st)
                      : launch_xcta_m<T, 12, MODE, 2, 6>(g, A, w12, st);
      return full12 ? launch_xcta_m<T, 12, MODE, 4, 3, true>(g, A, w12, st)
                    : launch_xcta_m<T, 12, MODE, 4, 3>(g, A, w12, st);
    }
  }
  int M = chunk;
  if (M != 4 && M != 8 && M != 16) M = (n > 256) ? 16 : (n > 128 ? 8 : 4);
  while (n > 512 * M) M *= 2;
  const int warps = (n + 32 * M - 1) / (32 * M);
  if (M == 4) return launch_xcta_m<T, 4, MODE, 16>(g, A, warps, st);
  if (M == 8)
    return warps <= 8 ? launch_xcta_m<T, 8, MODE, 8>(g, A, warps, st)
                      : launch_xcta_m<T, 8, MODE, 16>(g, A, warps, st);
  // forward modes up to 3072 rows (six warps): registers capped near 170
  // (6 CTAs per SM up to two warps, 3 up to four, 2 up to six; uncapped the
  // 3..6-warp CTAs take 254 registers and fit once or twice per SM); the
  // adjoint modes spill under such caps and measured slower.  Systems of
  // whole warp blocks (n = 512 * warps) drop every row guard.
  const bool full = n == warps * 32 * 16;
  if constexpr (MODE == kXFwd || MODE == kXFwdInc) {
    if (warps <= 2)
      return full ? launch_xcta_m<T, 16, MODE, 2, 6, true>(g, A, warps, st)
                  : launch_xcta_m<T, 16, MODE, 2, 6>(g, A, warps, st);
    if (warps <= 4)
      return full ? launch_xcta_m<T, 16, MODE, 4, 3, true>(g, A, warps, st)
                  : launch_xcta_m<T, 16, MODE, 4, 3>(g, A, warps, st);
    if (warps <= 6)
      return full ? launch_xcta_m<T, 16, MODE, 6, 2, true>(g, A, warps, st)
                  : launch_xcta_m<T, 16, MODE, 6, 2>(g, A, warps, st);
  }
  if constexpr (MODE == kXFused) {  // (the adjoint measured slower without guards)
    if (full) return launch_xcta_m<T, 16, MODE, 8, 1, true>(g, A, warps, st);
  }
  return launch_xcta_m<T, 16, MODE, 8>(g, A, warps, st);
}

// ------------------------------------------- variable-length batch buckets --
// Systems of 257 .. 4096 rows of a variable-length batch (kern_varlen.cu),
// bucketed by the warps they need at 16 rows per lane (W = ceil(n / 512),
// bucket W-1 of lists / counts): one persistent launch per bucket, CTA = W
// warps, each CTA looping over the bucket's systems (every row read once,
// as in the strided batch), thread 0 warming L2 with its next system.
template <typename T>
__device__ __forceinline__ void prefetch_rows_l2(const T *p, int n) {
  // the 16-byte aligned interior of the rows, one bulk prefetch
  const uintptr_t b = ((uintptr_t)p + 15) & ~(uintptr_t)15;
  const uintptr_t e = (uintptr_t)(p + n) & ~(uintptr_t)15;
  if (e > b)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b), "r"((uint32_t)(e - b))
                 : "memory");
}

template <typename T, int M, int MAXW, int MINB>
__global__ void __launch_bounds__(MAXW * 32, MINB)
    xcta_varlen_kernel(XArgs<T> A, const int64_t *__restrict__ offsets,
                       const int *__restrict__ list, const unsigned *__restrict__ count,
                       unsigned *__restrict__ claim) {
  pdl_enter();
  // systems are claimed one at a time (a bucket's lengths differ by up to 2x,
  // so a fixed split leaves CTAs idle at the end); the next one is claimed
  // when the current one starts, so that its rows can be warmed in L2
  __shared__ unsigned s_next;
  const int64_t cnt = (int64_t)*count;
  if (threadIdx.x == 0) s_next = atomicAdd(claim, 1u);
  __syncthreads();
  int64_t i = s_next;
  while (i < cnt) {
    __syncthreads();  // every thread has read s_next
    if (threadIdx.x == 0) s_next = atomicAdd(claim, 1u);
    const int s = list[i];
    const int64_t lo = offsets[s];
    const int n = (int)(offsets[s + 1] - lo);
    const int64_t off[5] = {lo, lo, lo, lo, lo};
    xcta_system<T, M, kXFwd, false>(A, off, n, [&] {
      const int64_t nxt = s_next;  // thread 0's own claim
      if (threadIdx.x == 0 && nxt < cnt) {
        const int s2 = list[nxt];
        const int64_t lo2 = offsets[s2];
        const int n2 = (int)(offsets[s2 + 1] - lo2);
        prefetch_rows_l2(A.a + lo2, n2);
        prefetch_rows_l2(A.b + lo2, n2);
        prefetch_rows_l2(A.c + lo2, n2);
        prefetch_rows_l2(A.d + lo2, n2);
      }
    });
    __syncthreads();  // the staged regions are refilled for the next system; s_next is seen
    i = s_next;
  }
}

template <typename T, int M, int MAXW, int MINB>
static cudaError_t launch_xcta_varlen_w(const XArgs<T> &A, const int64_t *offsets, const int *list,
                                        const unsigned *count, unsigned *claim, int W, int dev,
                                        int sms, cudaStream_t st) {
  auto kern = xcta_varlen_kernel<T, M, MAXW, MINB>;
  const size_t smem = (size_t)4 * W * Stage<T, M>::R * sizeof(T);
  static bool attr_set[64] = {};
  static int per_sm[64][9] = {};  // resident CTAs per SM by W, per device
  if (!attr_set[dev]) {
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               4 * MAXW * Stage<T, M>::R * (int)sizeof(T));
    if (e != cudaSuccess) return e;
    attr_set[dev] = true;
  }
  if (per_sm[dev][W] == 0) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, W * kWarp, smem) != cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      nb = 1;
    }
    per_sm[dev][W] = nb;
  }
  return launch_pdl(kern, dim3((unsigned)(sms * per_sm[dev][W])), dim3(W * kWarp), (size_t)smem,
                    st, A, offsets, list, count, claim);
}

template <typename T>
cudaError_t launch_xcta_varlen(const T *a, const T *b, const T *c, T *d, const int64_t *offsets,
                               const int *lists, int64_t list_stride, unsigned *counts,
                               cudaStream_t st) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const XArgs<T> A{a, b, c, d, nullptr, nullptr, d, nullptr, nullptr, nullptr, nullptr};
  // register caps as for the strided batch: near 170 registers up to six
  // warps (6, 3 and 2 CTAs per SM for 2, 4 and 6 warps).  (Buckets at 12
  // rows per lane where that pads fewer rows, as the strided batch chooses,
  // measured no gain here: 300-row systems +8%, 1025..4096 rows -2%, the
  // 8..8192 mix -0.7%, three more launches against the padding saved.)
  for (int W = kVarlenCtaBuckets; W >= 1; --W) {
    const int *list = lists + (size_t)(W - 1) * (size_t)list_stride;
    const unsigned *cnt = counts + W - 1;
    unsigned *clm = counts + kVarlenClaims + W - 1;
    if (W <= 2)
      e = launch_xcta_varlen_w<T, 16, 2, 6>(A, offsets, list, cnt, clm, W, dev, sms, st);
    else if (W <= 4)
      e = launch_xcta_varlen_w<T, 16, 4, 3>(A, offsets, list, cnt, clm, W, dev, sms, st);
    else if (W <= 6)
      e = launch_xcta_varlen_w<T, 16, 6, 2>(A, offsets, list, cnt, clm, W, dev, sms, st);
    else
      e = launch_xcta_varlen_w<T, 16, 8, 1>(A, offsets, list, cnt, clm, W, dev, sms, st);
    if (e != cudaSuccess) return e;
  }

  return cudaSuccess;
}

template cudaError_t launch_xcta_varlen<float>(const float *, const float *, const float *,
                                               float *, const int64_t *, const int *, int64_t,
                                               unsigned *, cudaStream_t);
template cudaError_t launch_xcta_varlen<double>(const double *, const double *, const double *,
                                                double *, const int64_t *, const int *, int64_t,
                                                unsigned *, cudaStream_t);

#define TRID_XCTA_INSTANTIATE(T)                                                               \
  template cudaError_t launch_xcta<T, kXFwd>(const Geom &, const XArgs<T> &, int, cudaStream_t); \
  template cudaError_t launch_xcta<T, kXFwdInc>(const Geom &, const XArgs<T> &, int,            \
                                                cudaStream_t);                                  \
  template cudaError_t launch_xcta<T, kXAdj>(const Geom &, const XArgs<T> &, int, cudaStream_t); \
  template cudaError_t launch_xcta<T, kXFused>(const Geom &, const XArgs<T> &, int, cudaStream_t);
TRID_XCTA_INSTANTIATE(float)
TRID_XCTA_INSTANTIATE(double)

}  // namespace tridb200
