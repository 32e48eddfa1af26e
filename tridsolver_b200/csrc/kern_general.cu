// General partitioned-Thomas kernels (sm_100a): any system length, the
// forward solve and the adjoint solve.
//
// A system is cut into blocks of B = 32*M rows (one warp's 32 chunks).
//  * n <= B  (phase kSingle): chunk reduction, warp interface solve,
//    back-substitution -- the algorithm of partition.cuh.
//  * n >  B  (three launches, see launch_general):
//      kReduce : every block reduces to two rows in its own first/last
//                unknowns (warp_block_basis + block_rows), written to
//                scratch as a tridiagonal system of 2*nblk rows per system;
//      (the block system is solved by the strided-batch dispatcher itself,
//       recursively, as a contiguous batch);
//      kFinish : every block recomputes its chunk reduction, takes its two
//                boundary unknowns from the block solution and
//                back-substitutes.
//    The block pass re-reads a, b, c and the right-hand side, so long
//    systems move 72 bytes per FP64 unknown instead of the 40-byte minimum.
//
// Row modes:
//  * kFwd / kFwdInc: the strided-batch solve (x overwrites d / u += x),
//    a_i x_{i-1} + b_i x_i + c_i x_{i+1} = d_i (trid_cpu.cpp:360-401).
//  * kAdj: the adjoint of that solve for a loss L(x): with the cotangent
//    w = dL/dx and the forward solution u, g = A^{-T} w is the solution of
//    the transposed system c_{i-1} g_{i-1} + b_i g_i + a_{i+1} g_{i+1} = w_i,
//    and dL/dd = g, dL/da_i = -g_i u_{i-1}, dL/db_i = -g_i u_i,
//    dL/dc_i = -g_i u_{i+1} (zero where a_0 / c_{n-1} are unused).  The
//    transposed coefficients are read in place (no shifted copies), and the
//    gradients are formed in the same pass.
//
// Layouts: axis 0 (unit stride, one warp per system block, rows staged in
// shared memory by coalesced copies) and strided axes
// (SB adjacent systems per CTA, thread = (system, chunk), interface rows
// transposed through shared memory so one warp solves one system's block).
#include <string.h>

#include "partition.cuh"

namespace tridb200 {

constexpr int kFwd = kGenFwd, kFwdInc = kGenFwdInc, kAdj = kGenAdj;
constexpr int kSingle = kGenSingle, kReduce = kGenReduce, kFinish = kGenFinish;

// ---------------------------------------------------------------- rows --
template <typename T, int M, int MODE>
__device__ __forceinline__ void load_rows(const GenArgs<T> &A, const int64_t (&off)[5],
                                          const Geom &g, int rbase, bool valid, T (&al)[M],
                                          T (&be)[M], T (&ga)[M], T (&de)[M]) {
  const int n = g.n;
  const int64_t sa = g.stride[kA], sb = g.stride[kB], sc = g.stride[kC], sd = g.stride[kD];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = rbase + j;
    if (valid && r < n) {
      if (MODE == kAdj) {
        al[j] = (r == 0) ? T(0) : A.c[off[kC] + (int64_t)(r - 1) * sc];
        ga[j] = (r == n - 1) ? T(0) : A.a[off[kA] + (int64_t)(r + 1) * sa];
      } else {
        al[j] = (r == 0) ? T(0) : A.a[off[kA] + (int64_t)r * sa];
        ga[j] = (r == n - 1) ? T(0) : A.c[off[kC] + (int64_t)r * sc];
      }
      be[j] = A.b[off[kB] + (int64_t)r * sb];
      de[j] = A.rhs[off[kD] + (int64_t)r * sd];
    } else {
      al[j] = T(0);
      be[j] = T(1);
      ga[j] = T(0);
      de[j] = T(0);
    }
  }
}

template <typename T, int M, int MODE>
__device__ __forceinline__ void store_rows(const GenArgs<T> &A, const int64_t (&off)[5],
                                           const Geom &g, int rbase, const T (&x)[M]) {
  const int n = g.n;
  if (MODE == kFwd) {
    const int64_t sd = g.stride[kD];
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (rbase + j < n) A.out[off[kD] + (int64_t)(rbase + j) * sd] = x[j];
  } else if (MODE == kFwdInc) {
    const int64_t su = g.stride[kU];
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (rbase + j < n) A.out[off[kU] + (int64_t)(rbase + j) * su] += x[j];
  } else {
    // gradients; u shares the geometry of array slot kU
    const int64_t su = g.stride[kU];
    const T *u = A.usol + off[kU];
    T uprev = (rbase > 0 && rbase - 1 < n) ? u[(int64_t)(rbase - 1) * su] : T(0);
    T ucur = (rbase < n) ? u[(int64_t)rbase * su] : T(0);
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int r = rbase + j;
      if (r >= n) break;
      const T unext = (r + 1 < n) ? u[(int64_t)(r + 1) * su] : T(0);
      const T gg = x[j];
      if (A.gd) A.gd[off[kD] + (int64_t)r * g.stride[kD]] = gg;
      if (A.gb) A.gb[off[kB] + (int64_t)r * g.stride[kB]] = -gg * ucur;
      if (A.ga) A.ga[off[kA] + (int64_t)r * g.stride[kA]] = (r > 0) ? -gg * uprev : T(0);
      if (A.gc) A.gc[off[kC] + (int64_t)r * g.stride[kC]] = (r + 1 < n) ? -gg * unext : T(0);
      uprev = ucur;
      ucur = unext;
    }
  }
}

// block-level bookkeeping shared by both layouts (whole warp calls it)
template <typename T, int PHASE>
__device__ __forceinline__ void block_step(const GenArgs<T> &A, int64_t sys, int blk, int64_t nsys,
                                           const Row<T> &F, const Row<T> &L, int lane, T &xF,
                                           T &xL) {
  if (PHASE == kSingle) {
    warp_interface_solve(F, L, xF, xL, lane);
    return;
  }
  T bF[3], bL[3];
  warp_block_basis(F, L, lane, bF, bL);
  const int64_t m = 2 * (int64_t)A.nblk;
  if (PHASE == kReduce) {
    Row<T> FB, LB;
    block_rows(F, L, bF, bL, lane, FB, LB);
    if (sys < nsys) {
      const int64_t plane = nsys * m;
      const int64_t i = sys * m + 2 * (int64_t)blk;
      if (lane == 0) {
        A.red[0 * plane + i] = FB.a;
        A.red[1 * plane + i] = FB.b;
        A.red[2 * plane + i] = FB.c;
        A.red[3 * plane + i] = FB.d;
        A.red[0 * plane + i + 1] = LB.a;
        A.red[1 * plane + i + 1] = LB.b;
        A.red[2 * plane + i + 1] = LB.c;
        A.red[3 * plane + i + 1] = LB.d;
      }
    }
    xF = xL = T(0);
  } else {
    T fB = T(0), lB = T(0);
    if (sys < nsys) {
      fB = A.bsol[sys * m + 2 * (int64_t)blk];
      lB = A.bsol[sys * m + 2 * (int64_t)blk + 1];
    }
    xF = bF[0] + fB * bF[1] + lB * bF[2];
    xL = bL[0] + fB * bL[1] + lB * bL[2];
  }
}

// --------------------------------------------------------------- axis 0 --
// One warp per block of 32*M rows.  The block's rows arrive in the warp's
// own shared-memory regions by coalesced cp.async (row q of the block at
// q + q/M: one pad element per chunk, so that lane L reading its rows
// L*M .. L*M+M-1 hits 32 distinct banks); results leave the same way.  The
// adjoint mode stages a, b, c, w and u; neighbours across the block edge
// (c_{r-1} for the first row, a_{r+1} for the last, u on both sides) are
// single global loads.
template <typename T>
__device__ __forceinline__ void gx_cp_async(T *dst, const T *src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int sz = valid ? (int)sizeof(T) : 0;  // 0: zero-fill, nothing read
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(sz)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(sz)
                 : "memory");
}

template <int M>
__device__ __forceinline__ int gx_pidx(int q) {
  return q + q / M;
}

template <int MODE>
constexpr int gx_regions() {
  return MODE == kAdj ? 5 : 4;
}

// One warp per block of 32*M rows.  FULL: n is a whole number of blocks (no
// row guards).  (An L2 prefetch of the block a resident set ahead measured no
// gain here: 1.763 ms either way for 2048 x 65,536.)
template <typename T, int M, int MODE, int PHASE, bool FULL>
__global__ void __launch_bounds__(128) gen_x_kernel(Geom g, GenArgs<T> A) {
  extern __shared__ __align__(16) unsigned char gx_dyn[];
  constexpr int R = 32 * (M + 1);  // elements per region
  constexpr int NR = gx_regions<MODE>();
  const int lane = threadIdx.x & (kWarp - 1);
  const int wi = threadIdx.x / kWarp;
  const int64_t item = (int64_t)blockIdx.x * (blockDim.x / kWarp) + wi;
  const int64_t sys = item / A.nblk;
  const int blk = (int)(item % A.nblk);
  if (sys >= g.nsys) return;  // uniform per warp; the kernel has no CTA barriers
  int64_t off[5];
  system_offsets(g, sys, off);
  const int n = g.n;
  const int wb = blk * 32 * M;  // first row of the block
  T *reg = reinterpret_cast<T *>(gx_dyn) + (size_t)wi * NR * R;
  T *sa = reg, *sb = reg + R, *sc = reg + 2 * R, *sd = reg + 3 * R, *su = reg + 4 * R;
  const T *pa = A.a + off[kA], *pb = A.b + off[kB], *pc = A.c + off[kC];
  const T *pd = A.rhs + off[kD];
  const T *pu = (MODE == kAdj) ? A.usol + off[kU] : nullptr;
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int q = j * kWarp + lane;
    const int r = wb + q;
    const bool in = FULL || r < n;
    const int s = gx_pidx<M>(q);
    gx_cp_async(sa + s, in ? pa + r : pa, in);
    gx_cp_async(sb + s, in ? pb + r : pb, in);
    gx_cp_async(sc + s, in ? pc + r : pc, in);
    gx_cp_async(sd + s, in ? pd + r : pd, in);
    if (MODE == kAdj) gx_cp_async(su + s, in ? pu + r : pu, in);
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncwarp();

  const int rbase = wb + lane * M;
  const int ts = lane * (M + 1);  // this lane's rows in every region
  T al[M], be[M], ga[M], de[M];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = rbase + j;
    const bool in = FULL || r < n;
    be[j] = in ? sb[ts + j] : T(1);
    de[j] = sd[ts + j];  // zero-filled past n
    if (MODE == kAdj) {
      // transposed rows: sub-diagonal c_{r-1}, super-diagonal a_{r+1}
      T cm = T(0), ap = T(0);
      if (in && r > 0) cm = (j > 0) ? sc[ts + j - 1] : (lane > 0 ? sc[ts - 2] : pc[r - 1]);
      if (r + 1 < n) ap = (j < M - 1) ? sa[ts + j + 1] : (lane < kWarp - 1 ? sa[ts + M + 1] : pa[r + 1]);
      al[j] = cm;
      ga[j] = ap;
    } else {
      al[j] = (in && r > 0) ? sa[ts + j] : T(0);
      ga[j] = (r < n - 1) ? sc[ts + j] : T(0);
    }
  }
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  T xF, xL;
  block_step<T, PHASE>(A, sys, blk, g.nsys, F, L, lane, xF, xL);
  if (PHASE == kReduce) return;
  chunk_backsub<T, M>(al, ga, de, xF, xL);

  // out through this warp's regions: value v_j of this lane's rows into
  // region k, then coalesced stores of rows wb .. wb+32M-1
  auto put = [&](T *rg, const T(&v)[M]) {
#pragma unroll
    for (int j = 0; j < M; ++j) rg[ts + j] = v[j];
  };
  auto flush = [&](const T *rg, T *p, bool add) {
    __syncwarp();
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int q = j * kWarp + lane;
      if (FULL || wb + q < n) {
        if (add)
          p[wb + q] += rg[gx_pidx<M>(q)];
        else
          p[wb + q] = rg[gx_pidx<M>(q)];
      }
    }
  };
  if constexpr (MODE == kFwd || MODE == kFwdInc) {
    put(sd, de);  // d was read only by this lane
    flush(sd, A.out + (MODE == kFwd ? off[kD] : off[kU]), MODE == kFwdInc);
  } else {
  // gradients: g = de; u_{r-1}, u_r, u_{r+1} from the staged u
  T uu[M];
#pragma unroll
  for (int j = 0; j < M; ++j) uu[j] = su[ts + j];
  const T uprev = (rbase > 0 && rbase - 1 < n) ? (lane > 0 ? su[ts - 2] : pu[rbase - 1]) : T(0);
  const T unext = (rbase + M < n) ? (lane < kWarp - 1 ? su[ts + M + 1] : pu[rbase + M]) : T(0);
  __syncwarp();  // every lane has read its neighbours' a, c and u slots
  T v[M];
  if (A.ga) {
#pragma unroll
    for (int j = 0; j < M; ++j)
      v[j] = (rbase + j > 0) ? -de[j] * (j > 0 ? uu[j - 1] : uprev) : T(0);
    put(sa, v);
    flush(sa, A.ga + off[kA], false);
  }
  if (A.gb) {
#pragma unroll
    for (int j = 0; j < M; ++j) v[j] = -de[j] * uu[j];
    put(sb, v);
    flush(sb, A.gb + off[kB], false);
  }
  if (A.gc) {
#pragma unroll
    for (int j = 0; j < M; ++j)
      v[j] = (rbase + j + 1 < n) ? -de[j] * (j < M - 1 ? uu[j + 1] : unext) : T(0);
    put(sc, v);
    flush(sc, A.gc + off[kC], false);
  }
  if (A.gd) {
    put(sd, de);
    flush(sd, A.gd + off[kD], false);
  }
  }
}

// --------------------------------------------------------- strided axes --
// Whole blocks of forward systems whose rows are 16-byte aligned in every
// array: each lane moves its chunk of M rows (64 bytes per array) as 16-byte
// words straight between global memory and registers, with no shared-memory
// staging (the staged kernel above stalls on its shared-memory traffic).
template <typename T, int M>
__device__ __forceinline__ void gx_ld16(const T *p, T (&v)[M], bool nc) {
  constexpr int K = M * (int)sizeof(T) / 16;
  static_assert(K * 16 == M * (int)sizeof(T), "whole 16-byte words");
  const uint4 *q = reinterpret_cast<const uint4 *>(p);
  uint4 w[K];
#pragma unroll
  for (int k = 0; k < K; ++k) w[k] = nc ? __ldg(q + k) : q[k];
  memcpy(v, w, sizeof(w));
}
template <typename T, int M>
__device__ __forceinline__ void gx_st16(T *p, const T (&v)[M]) {
  constexpr int K = M * (int)sizeof(T) / 16;
  uint4 w[K];
  memcpy(w, v, sizeof(w));
  uint4 *q = reinterpret_cast<uint4 *>(p);
#pragma unroll
  for (int k = 0; k < K; ++k) q[k] = w[k];
}

template <typename T, int M, int MODE, int PHASE>
__global__ void __launch_bounds__(128) gen_xv_kernel(Geom g, GenArgs<T> A) {
  static_assert(MODE == kFwd || MODE == kFwdInc, "forward modes");
  const int lane = threadIdx.x & (kWarp - 1);
  const int wi = threadIdx.x / kWarp;
  const int64_t item = (int64_t)blockIdx.x * (blockDim.x / kWarp) + wi;
  const int64_t sys = item / A.nblk;
  const int blk = (int)(item % A.nblk);
  if (sys >= g.nsys) return;  // uniform per warp
  int64_t off[5];
  system_offsets(g, sys, off);
  const int n = g.n;
  const int rbase = blk * 32 * M + lane * M;
  T al[M], be[M], ga[M], de[M];
  gx_ld16<T, M>(A.a + off[kA] + rbase, al, true);
  gx_ld16<T, M>(A.b + off[kB] + rbase, be, true);
  gx_ld16<T, M>(A.c + off[kC] + rbase, ga, true);
  gx_ld16<T, M>(A.rhs + off[kD] + rbase, de, false);  // d may be the output
  if (rbase == 0) al[0] = T(0);
  if (rbase + M == n) ga[M - 1] = T(0);
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  T xF, xL;
  block_step<T, PHASE>(A, sys, blk, g.nsys, F, L, lane, xF, xL);
  if (PHASE == kReduce) return;
  chunk_backsub<T, M>(al, ga, de, xF, xL);
  if constexpr (MODE == kFwdInc) {
    T uo[M];
    gx_ld16<T, M>(A.out + off[kU] + rbase, uo, false);
#pragma unroll
    for (int j = 0; j < M; ++j) uo[j] += de[j];
    gx_st16<T, M>(A.out + off[kU] + rbase, uo);
  } else {
    gx_st16<T, M>(A.out + off[kD] + rbase, de);
  }
}

template <typename T, int M, int SB, int MODE, int PHASE>
__global__ void __launch_bounds__(SB * kWarp) gen_s_kernel(Geom g, GenArgs<T> A) {
  __shared__ T red[8][kWarp][SB + 1];
  __shared__ T sol[2][kWarp][SB + 1];
  const int tid = threadIdx.x;
  const int sl = tid % SB;
  const int t = tid / SB;
  const int64_t ntile = (g.nsys + SB - 1) / SB;
  const int64_t tile = (int64_t)blockIdx.x % ntile;
  const int blk = (int)((int64_t)blockIdx.x / ntile);
  const int64_t sys = tile * SB + sl;
  const bool valid = sys < g.nsys;
  int64_t off[5] = {0, 0, 0, 0, 0};
  if (valid) system_offsets(g, sys, off);
  const int rbase = blk * 32 * M + t * M;
  T al[M], be[M], ga[M], de[M];
  load_rows<T, M, MODE>(A, off, g, rbase, valid, al, be, ga, de);
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  red[0][t][sl] = F.a;
  red[1][t][sl] = F.b;
  red[2][t][sl] = F.c;
  red[3][t][sl] = F.d;
  red[4][t][sl] = L.a;
  red[5][t][sl] = L.b;
  red[6][t][sl] = L.c;
  red[7][t][sl] = L.d;
  __syncthreads();
  {
    const int w = tid / kWarp;
    const int lane = tid & (kWarp - 1);
    const Row<T> F2{red[0][lane][w], red[1][lane][w], red[2][lane][w], red[3][lane][w]};
    const Row<T> L2{red[4][lane][w], red[5][lane][w], red[6][lane][w], red[7][lane][w]};
    T xF, xL;
    block_step<T, PHASE>(A, tile * SB + w, blk, g.nsys, F2, L2, lane, xF, xL);
    sol[0][lane][w] = xF;
    sol[1][lane][w] = xL;
  }
  if (PHASE == kReduce) return;
  __syncthreads();
  chunk_backsub<T, M>(al, ga, de, sol[0][t][sl], sol[1][t][sl]);
  if (valid) store_rows<T, M, MODE>(A, off, g, rbase, de);
}

// -------------------------------------------------------------- launchers --
template <typename T, int M, int MODE, int PHASE>
static cudaError_t go_x(const Geom &g, const GenArgs<T> &A, cudaStream_t st) {
  constexpr int kW = 4;
  const int64_t items = g.nsys * A.nblk;
  const int64_t blocks = (items + kW - 1) / kW;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  const int smem = kW * gx_regions<MODE>() * 32 * (M + 1) * (int)sizeof(T);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 64) return cudaErrorNotSupported;
  if constexpr ((MODE == kFwd || MODE == kFwdInc) && sizeof(T) == 4 && M == 16) {
    // FP32 whole blocks with every array's rows 16-byte aligned in every
    // system (2,048 x 65,536: 0.934 -> 0.778 ms; FP64 8-row chunks measured
    // the same either way, 1.72 against 1.73 ms, and keep the staged kernel)
    bool vec = g.n % (32 * M) == 0;
    const void *ptrs[5] = {A.a, A.b, A.c, A.rhs, A.out};
    const int arr[5] = {kA, kB, kC, kD, MODE == kFwdInc ? kU : kD};
    for (int q = 0; q < 5 && vec; ++q) {
      vec = ((uintptr_t)ptrs[q] & 15) == 0;
      for (int k = 0; k < g.nod && vec; ++k) vec = (g.ocum[arr[q]][k] * (int64_t)sizeof(T)) % 16 == 0;
    }
    if (vec) {
      gen_xv_kernel<T, M, MODE, PHASE><<<dim3((unsigned)blocks), dim3(kW * kWarp), 0, st>>>(g, A);
      return cudaGetLastError();
    }
  }
  // whole blocks (only instantiated for the 256-row blocks of long systems)
  const bool full = M == 8 && g.n % (32 * M) == 0;
  auto kern = full ? gen_x_kernel<T, M, MODE, PHASE, (M == 8)> : gen_x_kernel<T, M, MODE, PHASE, false>;
  static bool attr_set[2][64] = {};  // per variant and device
  if (!attr_set[full][dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr_set[full][dev] = true;
  }
  kern<<<dim3((unsigned)blocks), dim3(kW * kWarp), smem, st>>>(g, A);
  return cudaGetLastError();
}

template <typename T, int M, int SB, int MODE, int PHASE>
static cudaError_t go_s(const Geom &g, const GenArgs<T> &A, cudaStream_t st) {
  const int64_t blocks = ((g.nsys + SB - 1) / SB) * A.nblk;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  gen_s_kernel<T, M, SB, MODE, PHASE><<<dim3((unsigned)blocks), dim3(SB * kWarp), 0, st>>>(g, A);
  return cudaGetLastError();
}

template <typename T, int M, int MODE, int PHASE>
static cudaError_t go(const Geom &g, const GenArgs<T> &A, int axis, int spc, cudaStream_t st) {
  if (axis == 0) return go_x<T, M, MODE, PHASE>(g, A, st);
  switch (spc) {
    case 4: return go_s<T, M, 4, MODE, PHASE>(g, A, st);
    case 8: return go_s<T, M, 8, MODE, PHASE>(g, A, st);
    case 16: return go_s<T, M, 16, MODE, PHASE>(g, A, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T, int MODE, int PHASE>
static cudaError_t go_m(const Geom &g, const GenArgs<T> &A, int axis, int chunk, int spc,
                        cudaStream_t st) {
  switch (chunk) {
    case 2: return go<T, 2, MODE, PHASE>(g, A, axis, spc, st);
    case 4: return go<T, 4, MODE, PHASE>(g, A, axis, spc, st);
    case 8: return go<T, 8, MODE, PHASE>(g, A, axis, spc, st);
    case 16: return go<T, 16, MODE, PHASE>(g, A, axis, spc, st);
    default: return cudaErrorInvalidValue;
  }
}

// One launch of the general family.  axis 0 = unit stride, else strided.
template <typename T, int MODE>
cudaError_t launch_general_phase(const Geom &g, const GenArgs<T> &A, int axis, int chunk, int spc,
                                 int phase, cudaStream_t st) {
  switch (phase) {
    case kSingle: return go_m<T, MODE, kSingle>(g, A, axis, chunk, spc, st);
    case kReduce: return go_m<T, MODE, kReduce>(g, A, axis, chunk, spc, st);
    case kFinish: return go_m<T, MODE, kFinish>(g, A, axis, chunk, spc, st);
    default: return cudaErrorInvalidValue;
  }
}

#define TRID_GEN_INSTANTIATE(T, MODE)                                                         \
  template cudaError_t launch_general_phase<T, MODE>(const Geom &, const GenArgs<T> &, int, int, \
                                                     int, int, cudaStream_t);
TRID_GEN_INSTANTIATE(float, kFwd)
TRID_GEN_INSTANTIATE(float, kFwdInc)
TRID_GEN_INSTANTIATE(float, kAdj)
TRID_GEN_INSTANTIATE(double, kFwd)
TRID_GEN_INSTANTIATE(double, kFwdInc)
TRID_GEN_INSTANTIATE(double, kAdj)

}  // namespace tridb200
