// Partitioned Thomas ("hybrid Thomas-PCR") building blocks, sm_100a.
//
// A system of n rows is cut into 32 contiguous chunks of M rows (rows past n
// are identity rows a=c=d=0, b=1).  Each thread owns one chunk in registers:
//
//  1. chunk_reduce: eliminate the chunk's interior rows j=1..M-2 with its first
//     unknown F=x_0 kept as a parameter (downward sweep), then fold the
//     interior back (upward recursion, FMAs only) into two interface rows
//        F row:  fa*L_{t-1} + fb*F_t + fc*L_t     = fd
//        L row:  la*F_t     + lb*L_t + lc*F_{t+1} = ld
//     where L_t = x_{M-1} is the chunk's last unknown.  The interior keeps
//     x_j = d'_j - a'_j*F_t - c'_j*x_{j+1}.
//  2. warp_interface_solve: the 64 interface rows of the 32 chunks form a
//     tridiagonal system [F_0, L_0, F_1, L_1, ...].  One step of odd-even
//     elimination removes the F unknowns (one shuffle), parallel cyclic
//     reduction (5 shuffle steps) solves the 32-row L system, and F_t follows
//     from its own row.
//  3. chunk_backsub: interior unknowns from F_t and L_t (FMAs only).
//
// This is the published partition / hybrid Thomas-PCR method; the reference
// implements its own variant in scalar/src/cuda/trid_thomaspcr.hpp:198-318
// (per-thread modified Thomas, trid_thomaspcr_small.h PCR).  Everything is
// register-resident: no shared or global scratch.
#pragma once

#include "trid_internal.cuh"

namespace tridb200 {

template <typename T>
struct Row {
  T a, b, c, d;
};

// Interface rows of one chunk.  On return al/ga/de[j] (1 <= j <= M-2) hold
// a'_j, c'_j, d'_j of  x_j + c'_j x_{j+1} = d'_j - a'_j x_0.
template <typename T, int M>
__device__ __forceinline__ void chunk_reduce(T (&al)[M], const T (&be)[M], T (&ga)[M],
                                             T (&de)[M], Row<T> &F, Row<T> &L) {
  static_assert(M >= 2, "chunks need at least two rows");
  if constexpr (M == 2) {
    F = {al[0], be[0], ga[0], de[0]};
    L = {al[1], be[1], ga[1], de[1]};
  } else {
    // downward sweep, x_0 as parameter
    T r = rcp(be[1]);
    ga[1] *= r;
    de[1] *= r;
    al[1] *= r;
#pragma unroll
    for (int j = 2; j <= M - 2; ++j) {
      r = rcp(be[j] - al[j] * ga[j - 1]);
      de[j] = (de[j] - al[j] * de[j - 1]) * r;
      al[j] = -(al[j] * al[j - 1]) * r;
      ga[j] = ga[j] * r;
    }
    // x_{M-2} = D - A x_0 - C x_{M-1}  ->  L row
    T D = de[M - 2], A = al[M - 2], C = ga[M - 2];
    L.a = -al[M - 1] * A;
    L.b = be[M - 1] - al[M - 1] * C;
    L.c = ga[M - 1];
    L.d = de[M - 1] - al[M - 1] * D;
    // fold upward to x_1 = D - A x_0 - C x_{M-1}  ->  F row
#pragma unroll
    for (int j = M - 3; j >= 1; --j) {
      D = de[j] - ga[j] * D;
      A = al[j] - ga[j] * A;
      C = -ga[j] * C;
    }
    F.a = al[0];
    F.b = be[0] - ga[0] * A;
    F.c = -ga[0] * C;
    F.d = de[0] - ga[0] * D;
  }
}

// chunk_reduce that also returns the reciprocal pivots rp[1..M-2] of the
// chunk's interior block.  A chunk's interior block and its transpose have
// the same pivots (p_j = b_j - a_j c_{j-1} / p_{j-1} either way), so the
// transposed system can reuse them: chunk_reduce_given below.
template <typename T, int M>
__device__ __forceinline__ void chunk_reduce_pivots(T (&al)[M], const T (&be)[M], T (&ga)[M],
                                                    T (&de)[M], Row<T> &F, Row<T> &L,
                                                    T (&rp)[M]) {
  static_assert(M >= 4, "chunks of at least four rows");
  T r = rcp(be[1]);
  rp[1] = r;
  ga[1] *= r;
  de[1] *= r;
  al[1] *= r;
#pragma unroll
  for (int j = 2; j <= M - 2; ++j) {
    r = rcp(be[j] - al[j] * ga[j - 1]);
    rp[j] = r;
    de[j] = (de[j] - al[j] * de[j - 1]) * r;
    al[j] = -(al[j] * al[j - 1]) * r;
    ga[j] = ga[j] * r;
  }
  T D = de[M - 2], A = al[M - 2], C = ga[M - 2];
  L.a = -al[M - 1] * A;
  L.b = be[M - 1] - al[M - 1] * C;
  L.c = ga[M - 1];
  L.d = de[M - 1] - al[M - 1] * D;
#pragma unroll
  for (int j = M - 3; j >= 1; --j) {
    D = de[j] - ga[j] * D;
    A = al[j] - ga[j] * A;
    C = -ga[j] * C;
  }
  F.a = al[0];
  F.b = be[0] - ga[0] * A;
  F.c = -ga[0] * C;
  F.d = de[0] - ga[0] * D;
}

// 2^-e for the binary exponent e of x (x normal), else 1: multiplying by it
// is exact and brings |x| into [1, 2)
__device__ __forceinline__ double pow2_inv_exponent(double x) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(x);
  const unsigned e = (unsigned)(bits >> 52) & 0x7ffu;
  if (e == 0u || e >= 0x7feu) return 1.0;
  return __longlong_as_double((long long)((unsigned long long)(2046u - e) << 52));
}
__device__ __forceinline__ float pow2_inv_exponent(float x) {
  const unsigned bits = __float_as_uint(x);
  const unsigned e = (bits >> 23) & 0xffu;
  if (e == 0u || e >= 0xfeu) return 1.0f;
  return __uint_as_float((254u - e) << 23);
}

// chunk_reduce_pivots with the pivots from the continuant recurrence
//   q_1 = b_1, q_0 = 1,  q_j = b_j q_{j-1} - (a_j c_{j-1}) q_{j-2},
//   p_j = q_j / q_{j-1}  (the leading minors of the chunk's interior block),
// so that the serial chain carries one multiply-add per row and the
// reciprocals 1/p_j = q_{j-1} / q_j do not wait on each other; the pair
// (q_{j-1}, q_j) is rescaled by a power of two every 4 rows to stay in range.
// Mathematically the same pivots as the Thomas recurrence
// p_j = b_j - a_j c_{j-1} / p_{j-1}.
template <typename T, int M>
__device__ __forceinline__ void chunk_reduce_cont(T (&al)[M], const T (&be)[M], T (&ga)[M],
                                                  T (&de)[M], Row<T> &F, Row<T> &L,
                                                  T (&rp)[M]) {
  static_assert(M >= 4, "chunks of at least four rows");
  T qm2 = T(1), qm1 = be[1];
  rp[1] = rcp(be[1]);
#pragma unroll
  for (int j = 2; j <= M - 2; ++j) {
    const T q = be[j] * qm1 - (al[j] * ga[j - 1]) * qm2;
    rp[j] = qm1 * rcp(q);
    qm2 = qm1;
    qm1 = q;
    if ((j & 3) == 0) {
      const T sc = pow2_inv_exponent(q);
      qm1 *= sc;
      qm2 *= sc;
    }
  }
  // c' and the two right-hand-side recurrences with the pivots known
  de[1] *= rp[1];
  al[1] *= rp[1];
  ga[1] *= rp[1];
#pragma unroll
  for (int j = 2; j <= M - 2; ++j) {
    const T r = rp[j];
    de[j] = (de[j] - al[j] * de[j - 1]) * r;
    al[j] = -(al[j] * al[j - 1]) * r;
    ga[j] = ga[j] * r;
  }
  T D = de[M - 2], A = al[M - 2], C = ga[M - 2];
  L.a = -al[M - 1] * A;
  L.b = be[M - 1] - al[M - 1] * C;
  L.c = ga[M - 1];
  L.d = de[M - 1] - al[M - 1] * D;
#pragma unroll
  for (int j = M - 3; j >= 1; --j) {
    D = de[j] - ga[j] * D;
    A = al[j] - ga[j] * A;
    C = -ga[j] * C;
  }
  F.a = al[0];
  F.b = be[0] - ga[0] * A;
  F.c = -ga[0] * C;
  F.d = de[0] - ga[0] * D;
}

// chunk_reduce with the interior's reciprocal pivots given: no divisions,
// only multiply-add recurrences.
template <typename T, int M>
__device__ __forceinline__ void chunk_reduce_given(T (&al)[M], const T (&be)[M], T (&ga)[M],
                                                   T (&de)[M], Row<T> &F, Row<T> &L,
                                                   const T (&rp)[M]) {
  static_assert(M >= 4, "chunks of at least four rows");
  ga[1] *= rp[1];
  de[1] *= rp[1];
  al[1] *= rp[1];
#pragma unroll
  for (int j = 2; j <= M - 2; ++j) {
    const T r = rp[j];
    de[j] = (de[j] - al[j] * de[j - 1]) * r;
    al[j] = -(al[j] * al[j - 1]) * r;
    ga[j] = ga[j] * r;
  }
  T D = de[M - 2], A = al[M - 2], C = ga[M - 2];
  L.a = -al[M - 1] * A;
  L.b = be[M - 1] - al[M - 1] * C;
  L.c = ga[M - 1];
  L.d = de[M - 1] - al[M - 1] * D;
#pragma unroll
  for (int j = M - 3; j >= 1; --j) {
    D = de[j] - ga[j] * D;
    A = al[j] - ga[j] * A;
    C = -ga[j] * C;
  }
  F.a = al[0];
  F.b = be[0] - ga[0] * A;
  F.c = -ga[0] * C;
  F.d = de[0] - ga[0] * D;
}

// Interior unknowns; the solution overwrites de[0..M-1].
template <typename T, int M>
__device__ __forceinline__ void chunk_backsub(const T (&al)[M], const T (&ga)[M], T (&de)[M],
                                              T xF, T xL) {
  if constexpr (M > 2) {
    T x = xL;
#pragma unroll
    for (int j = M - 2; j >= 1; --j) {
      x = de[j] - al[j] * xF - ga[j] * x;
      de[j] = x;
    }
  }
  de[0] = xF;
  de[M - 1] = xL;
}

// Solve the 64-row interface system held two rows per lane (all 32 lanes of
// the warp must call this).  Lane 0's F row must not couple to the left
// (fa = 0) and lane 31's L row not to the right (lc = 0).
// span: a power of two >= the number of lanes holding non-identity rows
// (lanes at or past it hold identity rows); PCR stops after log2(span)
// steps, when every such row is decoupled.
template <typename T, int W = kWarp>
__device__ __forceinline__ void warp_interface_solve(const Row<T> &F, const Row<T> &L, T &xF,
                                                     T &xL, int lane, int span = W) {
  // W < 32: the warp holds 32/W independent systems of W lanes each (lane
  // groups of W; shuffles stay inside a group)
  static_assert(W == 8 || W == 16 || W == 32, "lane groups of 8, 16 or 32");
  constexpr unsigned kFull = 0xffffffffu;
  if constexpr (W == kWarp) {  // the whole warp: the plain shuffles
    const T ifb = rcp(F.b);
    T nfa = __shfl_down_sync(kFull, F.a, 1);
    T nfi = __shfl_down_sync(kFull, ifb, 1);
    T nfc = __shfl_down_sync(kFull, F.c, 1);
    T nfd = __shfl_down_sync(kFull, F.d, 1);
    if (lane == kWarp - 1) {
      nfa = T(0);
      nfi = T(1);
      nfc = T(0);
      nfd = T(0);
    }
    const T p = L.a * ifb;
    const T q = L.c * nfi;
    T ra = -p * F.a;
    T rb = L.b - p * F.c - q * nfa;
    T rc = -q * nfc;
    T rd = L.d - p * F.d - q * nfd;
#pragma unroll
    for (int s = 1; s < kWarp; s <<= 1) {
      if (s >= span) break;
      const T ib = rcp(rb);
      const T sa = ra * ib, sc = rc * ib, sd = rd * ib;
      const T ua = __shfl_up_sync(kFull, sa, s);
      const T uc = __shfl_up_sync(kFull, sc, s);
      const T ud = __shfl_up_sync(kFull, sd, s);
      const T da = __shfl_down_sync(kFull, sa, s);
      const T dc = __shfl_down_sync(kFull, sc, s);
      const T dd = __shfl_down_sync(kFull, sd, s);
      const T k1 = (lane >= s) ? ra : T(0);
      const T k2 = (lane + s < kWarp) ? rc : T(0);
      ra = -k1 * ua;
      rc = -k2 * dc;
      rb = rb - k1 * uc - k2 * da;
      rd = rd - k1 * ud - k2 * dd;
    }
    xL = rd * rcp(rb);
    const T lprev = __shfl_up_sync(kFull, xL, 1);
    xF = (F.d - (lane > 0 ? F.a * lprev : T(0)) - F.c * xL) * ifb;
    return;
  }
  const int ll = lane & (W - 1);  // lane within its group
  const T ifb = rcp(F.b);
  // F row of the next chunk (its pivot as a reciprocal)
  T nfa = __shfl_down_sync(kFull, F.a, 1, W);
  T nfi = __shfl_down_sync(kFull, ifb, 1, W);
  T nfc = __shfl_down_sync(kFull, F.c, 1, W);
  T nfd = __shfl_down_sync(kFull, F.d, 1, W);
  if (ll == W - 1) {
    nfa = T(0);
    nfi = T(1);
    nfc = T(0);
    nfd = T(0);
  }
  // eliminate F_t and F_{t+1} from the L row -> tridiagonal in L only
  const T p = L.a * ifb;
  const T q = L.c * nfi;
  T ra = -p * F.a;
  T rb = L.b - p * F.c - q * nfa;
  T rc = -q * nfc;
  T rd = L.d - p * F.d - q * nfd;
  // parallel cyclic reduction over the W lanes; each row sends its
  // coefficients pre-divided by its pivot, so a neighbour needs 3 values
#pragma unroll
  for (int s = 1; s < W; s <<= 1) {
    if (s >= span) break;
    const T ib = rcp(rb);
    const T sa = ra * ib, sc = rc * ib, sd = rd * ib;
    const T ua = __shfl_up_sync(kFull, sa, s, W);
    const T uc = __shfl_up_sync(kFull, sc, s, W);
    const T ud = __shfl_up_sync(kFull, sd, s, W);
    const T da = __shfl_down_sync(kFull, sa, s, W);
    const T dc = __shfl_down_sync(kFull, sc, s, W);
    const T dd = __shfl_down_sync(kFull, sd, s, W);
    const T k1 = (ll >= s) ? ra : T(0);
    const T k2 = (ll + s < W) ? rc : T(0);
    ra = -k1 * ua;
    rc = -k2 * dc;
    rb = rb - k1 * uc - k2 * da;
    rd = rd - k1 * ud - k2 * dd;
  }
  xL = rd * rcp(rb);
  const T lprev = __shfl_up_sync(kFull, xL, 1, W);
  xF = (F.d - (ll > 0 ? F.a * lprev : T(0)) - F.c * xL) * ifb;
}

// The interface system of one warp with several right-hand sides: NR
// independent RHS columns share the elimination (used to express a block's
// interior in terms of its two boundary unknowns).  Same recurrence as
// warp_interface_solve.
template <typename T, int NR>
struct RowN {
  T a, b, c, d[NR];
};

template <typename T, int NR>
__device__ __forceinline__ void warp_interface_solve_n(const RowN<T, NR> &F, const RowN<T, NR> &L,
                                                       T (&xF)[NR], T (&xL)[NR], int lane) {
  constexpr unsigned kFull = 0xffffffffu;
  const T ifb = rcp(F.b);
  T nfa = __shfl_down_sync(kFull, F.a, 1);
  T nfi = __shfl_down_sync(kFull, ifb, 1);
  T nfc = __shfl_down_sync(kFull, F.c, 1);
  T nfd[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) nfd[k] = __shfl_down_sync(kFull, F.d[k], 1);
  if (lane == kWarp - 1) {
    nfa = T(0);
    nfi = T(1);
    nfc = T(0);
#pragma unroll
    for (int k = 0; k < NR; ++k) nfd[k] = T(0);
  }
  const T p = L.a * ifb;
  const T q = L.c * nfi;
  T ra = -p * F.a;
  T rb = L.b - p * F.c - q * nfa;
  T rc = -q * nfc;
  T rd[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) rd[k] = L.d[k] - p * F.d[k] - q * nfd[k];
#pragma unroll
  for (int s = 1; s < kWarp; s <<= 1) {
    const T ib = rcp(rb);
    const T sa = ra * ib, sc = rc * ib;
    const T ua = __shfl_up_sync(kFull, sa, s);
    const T uc = __shfl_up_sync(kFull, sc, s);
    const T da = __shfl_down_sync(kFull, sa, s);
    const T dc = __shfl_down_sync(kFull, sc, s);
    const T k1 = (lane >= s) ? ra : T(0);
    const T k2 = (lane + s < kWarp) ? rc : T(0);
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const T sd = rd[k] * ib;
      const T ud = __shfl_up_sync(kFull, sd, s);
      const T dd = __shfl_down_sync(kFull, sd, s);
      rd[k] = rd[k] - k1 * ud - k2 * dd;
    }
    ra = -k1 * ua;
    rc = -k2 * dc;
    rb = rb - k1 * uc - k2 * da;
  }
  const T irb = rcp(rb);
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    xL[k] = rd[k] * irb;
    const T lprev = __shfl_up_sync(kFull, xL[k], 1);
    xF[k] = (F.d[k] - (lane > 0 ? F.a * lprev : T(0)) - F.c * xL[k]) * ifb;
  }
}

// Block reduction: the 32 chunks of a warp form a block of 32*M rows whose
// first unknown F^B (lane 0's F) and last unknown L^B (lane 31's L) are kept;
// the 62 interface unknowns in between are expressed as
//   x = P + F^B * UF + L^B * UL
// by one 3-RHS solve in which lane 0's F row and lane 31's L row are replaced
// by identity rows.  Returns, per lane, (P, UF, UL) for its F and L unknown.
template <typename T>
__device__ __forceinline__ void warp_block_basis(const Row<T> &F, const Row<T> &L, int lane,
                                                 T (&bF)[3], T (&bL)[3]) {
  RowN<T, 3> F3, L3;
  F3.a = F.a;
  F3.b = F.b;
  F3.c = F.c;
  F3.d[0] = F.d;
  F3.d[1] = T(0);
  F3.d[2] = T(0);
  L3.a = L.a;
  L3.b = L.b;
  L3.c = L.c;
  L3.d[0] = L.d;
  L3.d[1] = T(0);
  L3.d[2] = T(0);
  if (lane == 0) {  // F_0 = F^B
    F3.a = T(0);
    F3.b = T(1);
    F3.c = T(0);
    F3.d[0] = T(0);
    F3.d[1] = T(1);
  }
  if (lane == kWarp - 1) {  // L_31 = L^B
    L3.a = T(0);
    L3.b = T(1);
    L3.c = T(0);
    L3.d[0] = T(0);
    L3.d[2] = T(1);
  }
  warp_interface_solve_n<T, 3>(F3, L3, bF, bL, lane);
}

// A block's interface unknowns once its first unknown F^B = f (lane 0's F)
// and last unknown L^B = l (lane 31's L) are known: the interface system with
// those two rows replaced by identity rows, one right-hand side (a third of
// warp_block_basis's work; the same values up to rounding).
template <typename T>
__device__ __forceinline__ void warp_block_finish(const Row<T> &F, const Row<T> &L, T f, T l,
                                                  int lane, T &xF, T &xL) {
  Row<T> F1 = F, L1 = L;
  if (lane == 0) F1 = {T(0), T(1), T(0), f};
  if (lane == kWarp - 1) L1 = {T(0), T(1), T(0), l};
  warp_interface_solve(F1, L1, xF, xL, lane);
}

// The two rows of a block's reduced equations, from the original interface
// rows of lanes 0 and 31 and the basis of warp_block_basis:
//   FB row: fa*L^B_{k-1} + (fb + fc*UF(L_0))*F^B + fc*UL(L_0)*L^B = fd - fc*P(L_0)
//   LB row: la*UF(F_31)*F^B + (lb + la*UL(F_31))*L^B + lc*F^B_{k+1} = ld - la*P(F_31)
// (lane 0 fills FB, lane 31 fills LB).
template <typename T>
__device__ __forceinline__ void block_rows(const Row<T> &F, const Row<T> &L, const T (&bF)[3],
                                           const T (&bL)[3], int lane, Row<T> &FB, Row<T> &LB) {
  const T l0P = __shfl_sync(0xffffffffu, bL[0], 0);
  const T l0F = __shfl_sync(0xffffffffu, bL[1], 0);
  const T l0L = __shfl_sync(0xffffffffu, bL[2], 0);
  const T f31P = __shfl_sync(0xffffffffu, bF[0], kWarp - 1);
  const T f31F = __shfl_sync(0xffffffffu, bF[1], kWarp - 1);
  const T f31L = __shfl_sync(0xffffffffu, bF[2], kWarp - 1);
  const T fa = __shfl_sync(0xffffffffu, F.a, 0), fb = __shfl_sync(0xffffffffu, F.b, 0);
  const T fc = __shfl_sync(0xffffffffu, F.c, 0), fd = __shfl_sync(0xffffffffu, F.d, 0);
  const T la = __shfl_sync(0xffffffffu, L.a, kWarp - 1), lb = __shfl_sync(0xffffffffu, L.b, kWarp - 1);
  const T lc = __shfl_sync(0xffffffffu, L.c, kWarp - 1), ld = __shfl_sync(0xffffffffu, L.d, kWarp - 1);
  (void)lane;
  FB = {fa, fb + fc * l0F, fc * l0L, fd - fc * l0P};
  LB = {la * f31F, lb + la * f31L, lc, ld - la * f31P};
}

}  // namespace tridb200
