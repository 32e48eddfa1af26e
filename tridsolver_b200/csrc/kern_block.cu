// Block-tridiagonal batched solve and its adjoint (sm_100a).
//
// Systems (reference block/src/blktrid_gpu.cuh:265-431, CPU gold
// block/src/blktrid_cpu.cpp:388-495):
//     A_n x_{n-1} + B_n x_n + C_n x_{n+1} = d_n,   n = 0..N-1,
// with M x M row-major blocks in the GPU interleaved layout: block (n, p) at
// ((n*P + p)*M*M), vector (n, p) at ((n*P + p)*M).  A_0 and C_{N-1} are never
// read.  Block Thomas:
//     C'_0 = B_0^{-1} C_0, d'_0 = B_0^{-1} d_0,
//     X_n = B_n - A_n C'_{n-1}, C'_n = X_n^{-1} C_n, d'_n = X_n^{-1}(d_n - A_n d'_{n-1}),
//     x_{N-1} = d'_{N-1}, x_n = d'_n - C'_n x_{n+1}.
//
// Thread mapping: M lanes per system, lane i owns row i of every block (the
// reference's kernel owns columns).  Rows are contiguous, so the lanes of a
// warp read consecutive systems' blocks as one contiguous segment.  Products
// A_n C'_{n-1} broadcast rows of C' across the system's lanes by shuffles;
// X_n [C'_n | d'_n] = [C_n | d_n - A_n d'_{n-1}] is solved by Gauss-Jordan on
// the augmented rows (pivot row broadcast by shuffles, no pivoting: block
// diagonal dominance, as the reference GPU kernel assumes).  C'_n and d'_n go
// to the scratch arrays Cstar/dstar (the reference API's scratch) for the
// backward pass.
//
// Adjoint: the transposed block system has sub-diagonal C_{n-1}^T, diagonal
// B_n^T, super-diagonal A_{n+1}^T; lane i then owns column i of the original
// blocks.  With g the solution for the cotangent w and u the forward
// solution: dA_n = -g_n u_{n-1}^T, dB_n = -g_n u_n^T, dC_n = -g_n u_{n+1}^T,
// dd_n = g_n, formed in the backward sweep.
#include "trid_internal.cuh"

namespace tridb200 {

template <typename T>
struct BlkArgs {
  const T *A, *B, *C, *d;  // forward: rhs d; adjoint: rhs w
  const T *u;              // adjoint: forward solution
  T *x;                    // forward: solution; adjoint: unused
  T *dA, *dB, *dC, *dd;    // adjoint outputs (may be null)
  T *Cs, *ds;              // scratch C'/d' (N*P*M*M, N*P*M)
  int N, P;
};

template <typename T, int M, bool ADJ>
__global__ void __launch_bounds__(128) block_thomas_kernel(BlkArgs<T> a) {
  constexpr int SPW = kWarp / M;  // systems per warp
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & (kWarp - 1);
  const int sw = lane / M;        // system within warp
  const int i = lane % M;         // row owned
  const int base = sw * M;        // first lane of this system
  const int64_t p = ((int64_t)blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp) * SPW + sw;
  const bool valid = (sw < SPW) && (p < a.P);
  const int64_t P = a.P;
  const int N = a.N;
  const int src_base = (sw < SPW) ? base : 0;  // idle lanes shadow system 0
  auto bx = [&](int n) { return ((int64_t)n * P + p) * (M * M); };
  auto vx = [&](int n) { return ((int64_t)n * P + p) * M; };

  // row i of a block (forward) or column i (adjoint: row i of the transpose)
  auto load_row = [&](const T *Mat, int n, T (&r)[M]) {
#pragma unroll
    for (int j = 0; j < M; ++j)
      r[j] = valid ? (ADJ ? Mat[bx(n) + (int64_t)j * M + i] : Mat[bx(n) + (int64_t)i * M + j]) : T(0);
  };

  T Cp[M], dp = T(0);
#pragma unroll
  for (int j = 0; j < M; ++j) Cp[j] = T(0);

  for (int n = 0; n < N; ++n) {
    T X[M], R[M], Al[M];
    T rd;
    // diagonal block (transposed for the adjoint)
    load_row(a.B, n, X);
    if (!valid) X[i] = T(1);
    // sub-diagonal: A_n (forward) or C_{n-1}^T (adjoint); unused at n = 0
    if (n > 0) {
      if (ADJ)
        load_row(a.C, n - 1, Al);
      else
        load_row(a.A, n, Al);
    } else {
#pragma unroll
      for (int j = 0; j < M; ++j) Al[j] = T(0);
    }
    // super-diagonal: C_n (forward) or A_{n+1}^T (adjoint); unused at n = N-1
    if (n < N - 1) {
      if (ADJ)
        load_row(a.A, n + 1, R);
      else
        load_row(a.C, n, R);
    } else {
#pragma unroll
      for (int j = 0; j < M; ++j) R[j] = T(0);
    }
    rd = valid ? a.d[vx(n) + i] : T(0);
    // X = B - A C'_{n-1};  rd = d - A d'_{n-1}
#pragma unroll
    for (int k = 0; k < M; ++k) {
      const T ak = Al[k];
#pragma unroll
      for (int j = 0; j < M; ++j) X[j] -= ak * __shfl_sync(kFull, Cp[j], src_base + k);
      rd -= ak * __shfl_sync(kFull, dp, src_base + k);
    }
    // Gauss-Jordan on [X | R | rd]
#pragma unroll
    for (int q = 0; q < M; ++q) {
      T pX[M], pR[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        pX[j] = __shfl_sync(kFull, X[j], src_base + q);
        pR[j] = __shfl_sync(kFull, R[j], src_base + q);
      }
      const T pd = __shfl_sync(kFull, rd, src_base + q);
      const T inv = rcp(pX[q]);
      if (i == q) {
#pragma unroll
        for (int j = 0; j < M; ++j) {
          X[j] *= inv;
          R[j] *= inv;
        }
        rd *= inv;
      } else {
        const T f = X[q] * inv;
#pragma unroll
        for (int j = 0; j < M; ++j) {
          X[j] -= f * pX[j];
          R[j] -= f * pR[j];
        }
        rd -= f * pd;
      }
    }
    // C'_n row i, d'_n[i]
#pragma unroll
    for (int j = 0; j < M; ++j) Cp[j] = R[j];
    dp = rd;
    if (valid) {
#pragma unroll
      for (int j = 0; j < M; ++j) a.Cs[bx(n) + (int64_t)i * M + j] = R[j];
      a.ds[vx(n) + i] = rd;
    }
  }

  // backward sweep: x_{N-1} = d'_{N-1}; x_n = d'_n - C'_n x_{n+1}
  T xn = dp;        // x_{N-1}[i]
  T unext[M];       // adjoint: u_{n+1} (all components), zero past the end
  T ucur[M];        // adjoint: u_n
#pragma unroll
  for (int j = 0; j < M; ++j) {
    unext[j] = T(0);
    ucur[j] = (ADJ && valid) ? a.u[vx(N - 1) + j] : T(0);
  }
  for (int n = N - 1; n >= 0; --n) {
    if (n < N - 1) {
      T cr[M];
      if (valid) {
#pragma unroll
        for (int j = 0; j < M; ++j) cr[j] = a.Cs[bx(n) + (int64_t)i * M + j];
      } else {
#pragma unroll
        for (int j = 0; j < M; ++j) cr[j] = T(0);
      }
      const T dd = valid ? a.ds[vx(n) + i] : T(0);
      T acc = dd;
#pragma unroll
      for (int k = 0; k < M; ++k) acc -= cr[k] * __shfl_sync(kFull, xn, src_base + k);
      xn = acc;
    }
    if (!valid) continue;
    if (!ADJ) {
      a.x[vx(n) + i] = xn;
    } else {
      // gradients of block row n from g_n (= xn, lane i holds g_n[i])
      T uprev[M];
#pragma unroll
      for (int j = 0; j < M; ++j) uprev[j] = (n > 0) ? a.u[vx(n - 1) + j] : T(0);
      if (a.dd) a.dd[vx(n) + i] = xn;
#pragma unroll
      for (int j = 0; j < M; ++j) {
        if (a.dA) a.dA[bx(n) + (int64_t)i * M + j] = (n > 0) ? -xn * uprev[j] : T(0);
        if (a.dB) a.dB[bx(n) + (int64_t)i * M + j] = -xn * ucur[j];
        if (a.dC) a.dC[bx(n) + (int64_t)i * M + j] = (n < N - 1) ? -xn * unext[j] : T(0);
      }
#pragma unroll
      for (int j = 0; j < M; ++j) {
        unext[j] = ucur[j];
        ucur[j] = uprev[j];
      }
    }
  }
}

template <typename T, bool ADJ>
cudaError_t launch_block(const BlkArgs<T> &a, int M, cudaStream_t st) {
  auto go = [&](auto kern, int m) {
    const int spw = kWarp / m;
    const int64_t warps = (a.P + spw - 1) / spw;
    const int64_t blocks = (warps + 3) / 4;
    if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
    kern<<<dim3((unsigned)blocks), dim3(128), 0, st>>>(a);
    return cudaGetLastError();
  };
  switch (M) {
    case 1: return go(block_thomas_kernel<T, 1, ADJ>, 1);
    case 2: return go(block_thomas_kernel<T, 2, ADJ>, 2);
    case 3: return go(block_thomas_kernel<T, 3, ADJ>, 3);
    case 4: return go(block_thomas_kernel<T, 4, ADJ>, 4);
    case 5: return go(block_thomas_kernel<T, 5, ADJ>, 5);
    case 6: return go(block_thomas_kernel<T, 6, ADJ>, 6);
    case 7: return go(block_thomas_kernel<T, 7, ADJ>, 7);
    case 8: return go(block_thomas_kernel<T, 8, ADJ>, 8);
    case 9: return go(block_thomas_kernel<T, 9, ADJ>, 9);
    case 10: return go(block_thomas_kernel<T, 10, ADJ>, 10);
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------- host --
template <typename T>
static tridStatus_t blk_solve(const T *A, const T *B, const T *C, const T *d, T *x, int N, int P,
                              int M, T *Cs, T *ds) {
  if (N < 1 || P < 0 || M < 1 || M > 10 || !A || !B || !C || !d || !x)
    return TRID_STATUS_INVALID_VALUE;
  if (P == 0) return TRID_STATUS_SUCCESS;
  const size_t ne = (size_t)N * P * M * M, nv = (size_t)N * P * M;
  if (!Cs || !ds) {
    T *w = (T *)scratch((ne + nv) * sizeof(T), 0);
    if (!w) return TRID_STATUS_ALLOC_FAILED;
    Cs = w;
    ds = w + ne;
  }
  BlkArgs<T> a = {A, B, C, d, nullptr, x, nullptr, nullptr, nullptr, nullptr, Cs, ds, N, P};
  return launch_block<T, false>(a, M, current_stream()) == cudaSuccess ? TRID_STATUS_SUCCESS
                                                                      : TRID_STATUS_EXECUTION_FAILED;
}

template <typename T>
static tridStatus_t blk_adjoint(const T *A, const T *B, const T *C, const T *u, const T *w, T *dA,
                                T *dB, T *dC, T *dd, int N, int P, int M) {
  if (N < 1 || P < 0 || M < 1 || M > 10 || !A || !B || !C || !u || !w)
    return TRID_STATUS_INVALID_VALUE;
  if (P == 0) return TRID_STATUS_SUCCESS;
  const size_t ne = (size_t)N * P * M * M, nv = (size_t)N * P * M;
  T *s = (T *)scratch((ne + nv) * sizeof(T), 0);
  if (!s) return TRID_STATUS_ALLOC_FAILED;
  BlkArgs<T> a = {A, B, C, w, u, nullptr, dA, dB, dC, dd, s, s + ne, N, P};
  return launch_block<T, true>(a, M, current_stream()) == cudaSuccess ? TRID_STATUS_SUCCESS
                                                                     : TRID_STATUS_EXECUTION_FAILED;
}

}  // namespace tridb200

using namespace tridb200;

extern "C" tridStatus_t tridDbtsvBatch(const double *A, const double *B, const double *C,
                                       const double *d, double *x, int N, int P, int M,
                                       double *Cstar, double *dstar) {
  return blk_solve<double>(A, B, C, d, x, N, P, M, Cstar, dstar);
}
extern "C" tridStatus_t tridSbtsvBatch(const float *A, const float *B, const float *C,
                                       const float *d, float *x, int N, int P, int M,
                                       float *Cstar, float *dstar) {
  return blk_solve<float>(A, B, C, d, x, N, P, M, Cstar, dstar);
}
extern "C" tridStatus_t tridDbtsvBatchAdjoint(const double *A, const double *B, const double *C,
                                              const double *u, const double *w, double *dA,
                                              double *dB, double *dC, double *dd, int N, int P,
                                              int M) {
  return blk_adjoint<double>(A, B, C, u, w, dA, dB, dC, dd, N, P, M);
}
extern "C" tridStatus_t tridSbtsvBatchAdjoint(const float *A, const float *B, const float *C,
                                              const float *u, const float *w, float *dA,
                                              float *dB, float *dC, float *dd, int N, int P,
                                              int M) {
  return blk_adjoint<float>(A, B, C, u, w, dA, dB, dC, dd, N, P, M);
}

// The reference's block entry points, same C++ linkage and argument order
// (block/include/blktrid_gpu.h:38-40); the result lands in u.  Unlike the
// reference they neither print nor synchronise; errors are dropped as the
// void signature leaves no channel (use tridDbtsvBatch for a status).
void sbtsv_gpu(float *A, float *B, float *C, float *d, float *Cstar, float *dstar, float *u,
               const int N, const int P, const int blkdim) {
  (void)blk_solve<float>(A, B, C, d, u, N, P, blkdim, Cstar, dstar);
}
void dbtsv_gpu(double *A, double *B, double *C, double *d, double *Cstar, double *dstar, double *u,
               const int N, const int P, const int blkdim) {
  (void)blk_solve<double>(A, B, C, d, u, N, P, blkdim, Cstar, dstar);
}
