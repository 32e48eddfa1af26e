// Axis-0 systems of one warp (sm_100a), for systems of about 100..2048 rows:
// the partitioned Thomas of partition.cuh with long chunks kept in shared
// memory instead of registers.
//
// CTA = one warp = one system.  The system's arrays are staged in shared
// memory by coalesced cp.async; lane L owns the chunk of rows
// [L*M, L*M + M), M = ceil(n/32), at shared index L*S + j with S = M | 1 (an
// odd stride, so the 32 lanes walking their chunks hit distinct banks).  Each
// lane reduces its chunk in place (downward sweep with the chunk's first
// unknown as a parameter, upward fold), the warp solves the 64 interface
// rows with shuffles (warp_interface_solve), and each lane back-substitutes
// into the staged right-hand side, which then leaves by coalesced stores.
//
// Compared with the one-CTA kernel (kern_xcta.cu) there is no block level,
// no barrier and one interface solve per system, at the price of a longer
// sequential chain per lane; several warps per SM hide it.
//
// Modes (as kern_xcta.cu): forward, forward-add, adjoint (transposed system
// reduced in place in the shifted slots of a and c: row r's sub-diagonal
// c_{r-1} and super-diagonal a_{r+1} are read by row r alone), and fused
// forward + adjoint of <w, x> (the transposed system's reduced coefficients
// go to two extra arrays, since the forward solve needs a and c intact).
#include "partition.cuh"

namespace tridb200 {

namespace {

constexpr int kWFwd = kXcFwd, kWFwdInc = kXcFwdInc, kWAdj = kXcAdj, kWFused = kXcFused;

template <int MODE>
constexpr int xwarp_arrays() {
  return MODE == kWFused ? 7 : (MODE == kWAdj ? 5 : 4);
}

template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

// Walks rows r = lane, lane + 32, ... and their chunk slots L*S + j.
struct SlotWalk {
  int L, j, M, S, q32, r32;
  __device__ SlotWalk(int lane, int M_, int S_, int q, int rm) : M(M_), S(S_), q32(q), r32(rm) {
    L = lane / M;
    j = lane - L * M;
  }
  __device__ int slot() const { return L * S + j; }
  __device__ void next() {
    j += r32;
    L += q32;
    if (j >= M) {
      j -= M;
      ++L;
    }
  }
};

// One lane's chunk of M rows is K sub-chunks of Ms = M/K rows (Ms >= 3),
// reduced together so that K independent recurrences are in flight per lane.
// Original coefficients of a sub-chunk's interior rows are read through rA/rC
// (and pB, pD), reduced ones written to and read back from wA/wC and pD (in
// place where wA == rA).  A sub-chunk's first and last rows arrive as values
// (R0, Rl).  Rows at or past n are identity rows.  Sub-chunk s, row j is at
// offset s*Ms + j of every pointer.
template <typename T, int K>
__device__ __forceinline__ void subchunks_reduce(const T *rA, const T *pB, const T *rC, T *wA,
                                                 T *wC, T *pD, const Row<T> (&R0)[K],
                                                 const Row<T> (&Rl)[K], const int (&nr)[K], int Ms,
                                                 Row<T> (&F)[K], Row<T> (&L)[K]) {
  T ap[K], cp[K], dp[K];
#pragma unroll
  for (int s = 0; s < K; ++s) {
    const int o = s * Ms + 1;
    const bool in = 1 < nr[s];
    const T a1 = in ? rA[o] : T(0), b1 = in ? pB[o] : T(1);
    const T c1 = (2 < nr[s]) ? rC[o] : T(0), d1 = in ? pD[o] : T(0);
    const T r = rcp(b1);
    ap[s] = a1 * r;
    cp[s] = c1 * r;
    dp[s] = d1 * r;
    wA[o] = ap[s];
    wC[o] = cp[s];
    pD[o] = dp[s];
  }
  for (int j = 2; j <= Ms - 2; ++j) {
#pragma unroll
    for (int s = 0; s < K; ++s) {
      const int o = s * Ms + j;
      const bool in = j < nr[s];
      const T aj = in ? rA[o] : T(0), bj = in ? pB[o] : T(1);
      const T cj = (j + 1 < nr[s]) ? rC[o] : T(0), dj = in ? pD[o] : T(0);
      const T r = rcp(bj - aj * cp[s]);
      dp[s] = (dj - aj * dp[s]) * r;
      ap[s] = -(aj * ap[s]) * r;
      cp[s] = cj * r;
      wA[o] = ap[s];
      wC[o] = cp[s];
      pD[o] = dp[s];
    }
  }
  T D[K], A[K], C[K];
#pragma unroll
  for (int s = 0; s < K; ++s) {
    L[s].a = -Rl[s].a * ap[s];
    L[s].b = Rl[s].b - Rl[s].a * cp[s];
    L[s].c = Rl[s].c;
    L[s].d = Rl[s].d - Rl[s].a * dp[s];
    D[s] = dp[s];
    A[s] = ap[s];
    C[s] = cp[s];
  }
  for (int j = Ms - 3; j >= 1; --j) {
#pragma unroll
    for (int s = 0; s < K; ++s) {
      const int o = s * Ms + j;
      const T cj = wC[o];
      D[s] = pD[o] - cj * D[s];
      A[s] = wA[o] - cj * A[s];
      C[s] = -cj * C[s];
    }
  }
#pragma unroll
  for (int s = 0; s < K; ++s) {
    F[s].a = R0[s].a;
    F[s].b = R0[s].b - R0[s].c * A[s];
    F[s].c = -R0[s].c * C[s];
    F[s].d = R0[s].d - R0[s].c * D[s];
  }
}

// Interior unknowns of the K sub-chunks from their first/last unknowns
// (xb[2s] = first, xb[2s+1] = last); the solution overwrites pD.
template <typename T, int K>
__device__ __forceinline__ void subchunks_backsub(const T *wA, const T *wC, T *pD, int Ms,
                                                  const T (&xb)[2 * K]) {
  T x[K];
#pragma unroll
  for (int s = 0; s < K; ++s) x[s] = xb[2 * s + 1];
  for (int j = Ms - 2; j >= 1; --j) {
#pragma unroll
    for (int s = 0; s < K; ++s) {
      const int o = s * Ms + j;
      x[s] = pD[o] - wA[o] * xb[2 * s] - wC[o] * x[s];
      pD[o] = x[s];
    }
  }
#pragma unroll
  for (int s = 0; s < K; ++s) {
    pD[s * Ms] = xb[2 * s];
    pD[s * Ms + Ms - 1] = xb[2 * s + 1];
  }
}

// Solve one system held in shared memory by the warp.  Forward (TRANS false):
// rows (a_r, b_r, c_r, d_r) from sa/sb/sc/sd, reduced in place.  Transposed
// (TRANS true): rows (c_{r-1}, b_r, a_{r+1}, d_r); reduced coefficients go to
// ta/tc at the row's own slot, or in place into the shifted slots when ta is
// null (row r's c_{r-1} and a_{r+1} are read by row r alone, and the slots a
// sub-chunk's first and last rows read are never written).  The solution
// overwrites sd.
template <typename T, int K, bool TRANS>
__device__ __forceinline__ void warp_solve_sm(T *sa, const T *sb, T *sc, T *sd, T *ta, T *tc,
                                              int lane, int n, int M, int S) {
  const int Ms = M / K;
  const int base = lane * S;
  const int r0 = lane * M;
  const int pad = S - M;
  Row<T> R0[K], Rl[K];
  int nr[K];
#pragma unroll
  for (int s = 0; s < K; ++s) {
    const int bs = base + s * Ms;  // slot of the sub-chunk's first row
    const int rs = r0 + s * Ms;    // its system row
    nr[s] = max(0, min(Ms, n - rs));
    R0[s] = {T(0), T(1), T(0), T(0)};
    Rl[s] = {T(0), T(1), T(0), T(0)};
    const int sl = bs + Ms - 1;
    if (!TRANS) {
      if (nr[s] > 0) R0[s] = {rs > 0 ? sa[bs] : T(0), sb[bs], (rs + 1 < n) ? sc[bs] : T(0), sd[bs]};
      if (nr[s] == Ms) Rl[s] = {sa[sl], sb[sl], (rs + Ms < n) ? sc[sl] : T(0), sd[sl]};
    } else {
      if (nr[s] > 0)
        R0[s] = {rs > 0 ? sc[bs - 1 - (s == 0 ? pad : 0)] : T(0), sb[bs],
                 (rs + 1 < n) ? sa[bs + 1] : T(0), sd[bs]};
      if (nr[s] == Ms)
        Rl[s] = {sc[sl - 1], sb[sl], (rs + Ms < n) ? sa[sl + 1 + (s == K - 1 ? pad : 0)] : T(0),
                 sd[sl]};
    }
  }
  const T *rA = TRANS ? sc + base - 1 : sa + base;
  const T *rC = TRANS ? sa + base + 1 : sc + base;
  T *wA = TRANS ? (ta ? ta + base : sc + base - 1) : sa + base;
  T *wC = TRANS ? (tc ? tc + base : sa + base + 1) : sc + base;
  Row<T> F[K], L[K];
  subchunks_reduce<T, K>(rA, sb + base, rC, wA, wC, sd + base, R0, Rl, nr, Ms, F, L);
  // the 2K interface rows of the lane form a small tridiagonal chunk
  // [F_0, L_0, ..., F_{K-1}, L_{K-1}]: reduce it, solve across the warp,
  // back-substitute
  T ma[2 * K], mb[2 * K], mc[2 * K], md[2 * K];
#pragma unroll
  for (int s = 0; s < K; ++s) {
    ma[2 * s] = F[s].a;
    mb[2 * s] = F[s].b;
    mc[2 * s] = F[s].c;
    md[2 * s] = F[s].d;
    ma[2 * s + 1] = L[s].a;
    mb[2 * s + 1] = L[s].b;
    mc[2 * s + 1] = L[s].c;
    md[2 * s + 1] = L[s].d;
  }
  Row<T> F2, L2;
  chunk_reduce<T, 2 * K>(ma, mb, mc, md, F2, L2);
  T xF, xL;
  warp_interface_solve(F2, L2, xF, xL, lane);
  chunk_backsub<T, 2 * K>(ma, mc, md, xF, xL);
  subchunks_backsub<T, K>(wA, wC, sd + base, Ms, md);
}

}  // namespace

template <typename T, int K, int MODE>
__global__ void __launch_bounds__(32) xwarp_kernel(Geom g, XArgs<T> A, int M, int S, int q32,
                                                   int r32) {
  extern __shared__ __align__(16) unsigned char xwarp_dyn[];
  T *sh = reinterpret_cast<T *>(xwarp_dyn);
  const int lane = threadIdx.x;
  const int n = g.n;
  int64_t off[5];
  system_offsets(g, (int64_t)blockIdx.x, off);
  const int R = 32 * S;
  T *sa = sh, *sb = sh + R, *sc = sh + 2 * R, *sd = sh + 3 * R;
  T *sw = sh + 4 * R;  // kWAdj, kWFused
  T *t1 = sh + 5 * R, *t2 = sh + 6 * R;  // kWFused
  {
    const T *pa = A.a + off[kA], *pb = A.b + off[kB], *pc = A.c + off[kC];
    const T *pd = (MODE == kWAdj) ? A.usol + off[kU] : A.d + off[kD];
    const T *pw = (MODE == kWAdj || MODE == kWFused) ? A.w + off[kD] : nullptr;
    SlotWalk it(lane, M, S, q32, r32);
    for (int r = lane; r < n; r += kWarp, it.next()) {
      const int s = it.slot();
      cp_async_elem(sa + s, pa + r);
      cp_async_elem(sb + s, pb + r);
      cp_async_elem(sc + s, pc + r);
      cp_async_elem(sd + s, pd + r);
      if (MODE == kWAdj || MODE == kWFused) cp_async_elem(sw + s, pw + r);
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncwarp();

  if (MODE == kWAdj || MODE == kWFused) {
    warp_solve_sm<T, K, true>(sa, sb, sc, sw, MODE == kWFused ? t1 : nullptr,
                           MODE == kWFused ? t2 : nullptr, lane, n, M, S);
    __syncwarp();
  }
  if (MODE != kWAdj) {
    warp_solve_sm<T, K, false>(sa, sb, sc, sd, nullptr, nullptr, lane, n, M, S);
    __syncwarp();
  }

  SlotWalk it(lane, M, S, q32, r32);
  if (MODE == kWFwd || MODE == kWFwdInc) {
    T *px = (MODE == kWFwd) ? A.x + off[kD] : A.x + off[kU];
    for (int r = lane; r < n; r += kWarp, it.next()) {
      if (MODE == kWFwd)
        px[r] = sd[it.slot()];
      else
        px[r] += sd[it.slot()];
    }
    return;
  }
  // gradients from g (sw) and x (sd)
  const int pad = S - M;
  T *px = (MODE == kWFused) ? A.x + off[kD] : nullptr;
  for (int r = lane; r < n; r += kWarp, it.next()) {
    const int s = it.slot();
    const T gr = sw[s], xr = sd[s];
    if (MODE == kWFused) px[r] = xr;
    if (A.gd) A.gd[off[kD] + r] = gr;
    if (A.gb) A.gb[off[kB] + r] = -gr * xr;
    if (A.ga) A.ga[off[kA] + r] = (r > 0) ? -gr * sd[s - 1 - (it.j == 0 ? pad : 0)] : T(0);
    if (A.gc) A.gc[off[kC] + r] = (r + 1 < n) ? -gr * sd[s + 1 + (it.j == M - 1 ? pad : 0)] : T(0);
  }
}

template <typename T, int K, int MODE>
static cudaError_t launch_xwarp_k(const Geom &g, const XArgs<T> &A, int M, cudaStream_t st) {
  const int S = M | 1;
  constexpr int kArr = xwarp_arrays<MODE>();
  const size_t smem = (size_t)kArr * kWarp * S * sizeof(T);
  if (smem > 227 * 1024) return cudaErrorNotSupported;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static int attr_bytes[64] = {};  // per device: the largest opt-in set so far
  if (dev >= 64) return cudaErrorNotSupported;
  if ((size_t)attr_bytes[dev] < smem) {
    e = cudaFuncSetAttribute(xwarp_kernel<T, K, MODE>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // the whole unified L1/shared array as shared memory: residency is set by
    // how many systems fit, and nothing here is re-read through L1
    e = cudaFuncSetAttribute(xwarp_kernel<T, K, MODE>,
                             cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    attr_bytes[dev] = (int)smem;
  }
  xwarp_kernel<T, K, MODE><<<(unsigned)g.nsys, kWarp, smem, st>>>(g, A, M, S, kWarp / M,
                                                                    kWarp % M);
  return cudaGetLastError();
}

template <typename T, int MODE>
cudaError_t launch_xwarp(const Geom &g, const XArgs<T> &A, cudaStream_t st) {
  // chunk of M = ceil(n/32) rows per lane, as K sub-chunks of at least 3 rows
  // (M rounded up to a multiple of K; the extra rows are identity rows)
  const int M0 = (g.n + kWarp - 1) / kWarp;
  if (M0 < 3 || g.nsys > 0x7fffffff) return cudaErrorNotSupported;
  if (M0 >= 12) return launch_xwarp_k<T, 4, MODE>(g, A, (M0 + 3) / 4 * 4, st);
  if (M0 >= 6) return launch_xwarp_k<T, 2, MODE>(g, A, (M0 + 1) / 2 * 2, st);
  return launch_xwarp_k<T, 1, MODE>(g, A, M0, st);
}

#define TRID_XWARP_INSTANTIATE(T)                                                             \
  template cudaError_t launch_xwarp<T, kXcFwd>(const Geom &, const XArgs<T> &, cudaStream_t);    \
  template cudaError_t launch_xwarp<T, kXcFwdInc>(const Geom &, const XArgs<T> &, cudaStream_t); \
  template cudaError_t launch_xwarp<T, kXcAdj>(const Geom &, const XArgs<T> &, cudaStream_t);    \
  template cudaError_t launch_xwarp<T, kXcFused>(const Geom &, const XArgs<T> &, cudaStream_t);
TRID_XWARP_INSTANTIATE(float)
TRID_XWARP_INSTANTIATE(double)

}  // namespace tridb200
