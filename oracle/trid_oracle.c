/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C, single-threaded restatement of the reference CPU algorithms for
 * the batched tridiagonal hot path.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load this library, and only as the checker.
 * Nothing in tridsolver_b200/ links, loads or calls it.
 *
 * Pinning: tests/test_oracle.py checks every function here against the
 * reference's golden fixtures (the .npz files in tests/golden, regenerated with the
 * reference's scalar/test/gen_testcases.py) and against the reference's own
 * CPU code compiled unmodified into oracle/_ref (scalar/src/cpu/trid_cpu.cpp,
 * block/src/blktrid_cpu.cpp, apps/adi/src/adi_orig.c).
 *
 * Compiled with -ffp-contract=off so every operation rounds exactly as
 * written, in the reference's operation order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_MAXDIM 8

/* ------------------------------------------------------------------------ */
/* Scalar Thomas on one system with per-array strides.                      */
/* Follows trid_cpu.cpp:360-401 (trid_scalar<INC>): bb = 1/b0, cc = bb*c0,   */
/* dd = bb*d0; for i>=1: bb = b-a*cc, dd = d-a*dd, bb = 1/bb, cc = bb*c,     */
/* dd = bb*dd; reverse dd = d2-c2*dd.  a[0] and c[n-1] are never read.       */
/* INC=1: u += x and d is left untouched; INC=0: x overwrites d.             */
/* ------------------------------------------------------------------------ */
#define DEFINE_THOMAS(T, SUF, ONE)                                                   \
  static void thomas_##SUF(const T *a, int64_t sa, const T *b, int64_t sb,         \
                           const T *c, int64_t sc, T *d, int64_t sd, T *u,         \
                           int64_t su, int64_t n, int inc, T *c2, T *d2) {         \
    T aa, bb, cc, dd;                                                               \
    int64_t i;                                                                      \
    if (n <= 0) return;                                                             \
    bb = ONE / b[0];                                                                \
    cc = bb * c[0];                                                                 \
    dd = bb * d[0];                                                                 \
    c2[0] = cc;                                                                     \
    d2[0] = dd;                                                                     \
    for (i = 1; i < n; i++) {                                                       \
      aa = a[i * sa];                                                               \
      bb = b[i * sb] - aa * cc;                                                     \
      dd = d[i * sd] - aa * dd;                                                     \
      bb = ONE / bb;                                                                \
      cc = bb * c[i * sc];                                                          \
      dd = bb * dd;                                                                 \
      c2[i] = cc;                                                                   \
      d2[i] = dd;                                                                   \
    }                                                                               \
    if (inc) u[(n - 1) * su] += dd; else d[(n - 1) * sd] = dd;                      \
    for (i = n - 2; i >= 0; i--) {                                                  \
      dd = d2[i] - c2[i] * dd;                                                      \
      if (inc) u[i * su] += dd; else d[i * sd] = dd;                                \
    }                                                                               \
  }

DEFINE_THOMAS(double, f64, 1.0)
DEFINE_THOMAS(float, f32, 1.0F)

/* trid_scalarD / trid_scalarS (trid_cpu.cpp:550-555, :597-602): one system,
 * one stride for every array. */
void oracle_trid_scalar_f64(const double *a, const double *b, const double *c,
                            double *d, double *u, int64_t n, int64_t stride, int inc) {
  double *w = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
  thomas_f64(a, stride, b, stride, c, stride, d, stride, u, stride, n, inc, w, w + n);
  free(w);
}
void oracle_trid_scalar_f32(const float *a, const float *b, const float *c,
                            float *d, float *u, int64_t n, int64_t stride, int inc) {
  float *w = (float *)malloc(sizeof(float) * 2 * (size_t)(n > 0 ? n : 1));
  thomas_f32(a, stride, b, stride, c, stride, d, stride, u, stride, n, inc, w, w + n);
  free(w);
}

/* ------------------------------------------------------------------------ */
/* N-D strided batch with per-array pads.                                   */
/* Layout: element (i0,i1,...) of array X at sum_k i_k * prod_{j<k} padsX[j]  */
/* (dims[0] fastest; trid_cpu.cpp:422,468,504 and the N-D decode of          */
/* trid_strided_multidim.hpp:125-147).  Systems run along `solvedim`; one    */
/* system per multi-index over the other axes.  Returns 0, or 3 (INVALID).   */
/* ------------------------------------------------------------------------ */
#define DEFINE_MTSV(T, SUF)                                                          \
  int oracle_mtsv_##SUF(const T *a, const int *ap, const T *b, const int *bp,        \
                        const T *c, const int *cp, T *d, const int *dp, T *u,        \
                        const int *up, int ndim, int solvedim, const int *dims,      \
                        int inc) {                                                   \
    int64_t cum[5][ORACLE_MAXDIM + 1];                                               \
    const int *pads[5] = {ap, bp, cp, dp, up};                                       \
    int64_t idx[ORACLE_MAXDIM];                                                      \
    int64_t nsys = 1, n, s, off[5], str[5];                                          \
    int k, q;                                                                        \
    T *w;                                                                            \
    if (ndim < 1 || ndim > ORACLE_MAXDIM || solvedim < 0 || solvedim >= ndim)        \
      return 3;                                                                      \
    for (q = 0; q < 5; q++) {                                                        \
      if (q == 4 && !inc) { for (k = 0; k <= ndim; k++) cum[4][k] = 0; continue; }   \
      cum[q][0] = 1;                                                                 \
      for (k = 0; k < ndim; k++) cum[q][k + 1] = cum[q][k] * pads[q][k];            \
    }                                                                                \
    for (k = 0; k < ndim; k++) {                                                     \
      if (dims[k] < 0) return 3;                                                     \
      if (k != solvedim) nsys *= dims[k];                                            \
    }                                                                                \
    n = dims[solvedim];                                                              \
    if (n == 0 || nsys == 0) return 0;                                               \
    w = (T *)malloc(sizeof(T) * 2 * (size_t)n);                                      \
    for (k = 0; k < ndim; k++) idx[k] = 0;                                           \
    for (q = 0; q < 5; q++) str[q] = cum[q][solvedim];                               \
    for (s = 0; s < nsys; s++) {                                                     \
      for (q = 0; q < 5; q++) {                                                      \
        off[q] = 0;                                                                  \
        for (k = 0; k < ndim; k++)                                                   \
          if (k != solvedim) off[q] += idx[k] * cum[q][k];                           \
      }                                                                              \
      thomas_##SUF(a + off[0], str[0], b + off[1], str[1], c + off[2], str[2],       \
                   d + off[3], str[3], inc ? u + off[4] : (T *)0, str[4], n, inc,    \
                   w, w + n);                                                        \
      for (k = 0; k < ndim; k++) { /* odometer over the non-solve axes */            \
        if (k == solvedim) continue;                                                 \
        if (++idx[k] < dims[k]) break;                                               \
        idx[k] = 0;                                                                  \
      }                                                                              \
    }                                                                                \
    free(w);                                                                         \
    return 0;                                                                        \
  }

DEFINE_MTSV(double, f64)
DEFINE_MTSV(float, f32)

/* Complex element types: the same Thomas and N-D batch in C99 complex
 * arithmetic (the reference declares tridC/ZmtsvStridedBatch over
 * tridMultiDimBatchSolve<complexf/complexd> and leaves them commented out,
 * scalar/src/cuda/trid_cuda.cu:546-600; its CPU Thomas, trid_cpu.cpp:360-401,
 * is written for any element type).  Pinned by tests/test_oracle.py against
 * the real functions above (zero imaginary parts) and against dense complex
 * LU. */
DEFINE_THOMAS(double _Complex, c128, 1.0)
DEFINE_THOMAS(float _Complex, c64, 1.0F)
DEFINE_MTSV(double _Complex, c128)
DEFINE_MTSV(float _Complex, c64)

/* ------------------------------------------------------------------------ */
/* Variable-length packed batch: system s occupies rows                      */
/* [offsets[s], offsets[s+1]) of every array, unit stride.  Each system is    */
/* trid_scalar (trid_cpu.cpp:360-401) with stride 1.                          */
/* ------------------------------------------------------------------------ */
void oracle_varlen_f64(const double *a, const double *b, const double *c, double *d,
                       double *u, const int64_t *offsets, int64_t nsys, int inc) {
  int64_t s, maxn = 1;
  double *w;
  for (s = 0; s < nsys; s++)
    if (offsets[s + 1] - offsets[s] > maxn) maxn = offsets[s + 1] - offsets[s];
  w = (double *)malloc(sizeof(double) * 2 * (size_t)maxn);
  for (s = 0; s < nsys; s++) {
    int64_t o = offsets[s];
    thomas_f64(a + o, 1, b + o, 1, c + o, 1, d + o, 1, inc ? u + o : (double *)0, 1,
               offsets[s + 1] - o, inc, w, w + maxn);
  }
  free(w);
}
void oracle_varlen_f32(const float *a, const float *b, const float *c, float *d,
                       float *u, const int64_t *offsets, int64_t nsys, int inc) {
  int64_t s, maxn = 1;
  float *w;
  for (s = 0; s < nsys; s++)
    if (offsets[s + 1] - offsets[s] > maxn) maxn = offsets[s + 1] - offsets[s];
  w = (float *)malloc(sizeof(float) * 2 * (size_t)maxn);
  for (s = 0; s < nsys; s++) {
    int64_t o = offsets[s];
    thomas_f32(a + o, 1, b + o, 1, c + o, 1, d + o, 1, inc ? u + o : (float *)0, 1,
               offsets[s + 1] - o, inc, w, w + maxn);
  }
  free(w);
}

/* ------------------------------------------------------------------------ */
/* Adjoint of a batch of contiguous systems (no reference counterpart).      */
/* For A u = d with loss L = <w,u>: g = A^-T w, dL/dd = g,                   */
/* dL/da_i = -g_i u_{i-1} (i>=1, 0 at i=0), dL/db_i = -g_i u_i,              */
/* dL/dc_i = -g_i u_{i+1} (i<=n-2, 0 at i=n-1).                              */
/* A^T has sub-diagonal c_{i-1}, diagonal b_i, super-diagonal a_{i+1}; it is  */
/* solved with the same Thomas recurrence as above.                          */
/* System s occupies [s*n, (s+1)*n).  Outputs may be NULL to skip them.      */
/* ------------------------------------------------------------------------ */
void oracle_adjoint_f64(const double *a, const double *b, const double *c,
                        const double *u, const double *w, double *g, double *ga,
                        double *gb, double *gc, int64_t n, int64_t nsys) {
  double *at = (double *)malloc(sizeof(double) * (size_t)n * 5);
  double *ct = at + n, *gg = at + 2 * n, *wk = at + 3 * n;
  int64_t s, i;
  for (s = 0; s < nsys; s++) {
    const double *as = a + s * n, *bs = b + s * n, *cs = c + s * n, *us = u + s * n;
    for (i = 0; i < n; i++) {
      at[i] = i > 0 ? cs[i - 1] : 0.0;
      ct[i] = i < n - 1 ? as[i + 1] : 0.0;
      gg[i] = w[s * n + i];
    }
    thomas_f64(at, 1, bs, 1, ct, 1, gg, 1, (double *)0, 1, n, 0, wk, wk + n);
    for (i = 0; i < n; i++) {
      if (g) g[s * n + i] = gg[i];
      if (ga) ga[s * n + i] = i > 0 ? -gg[i] * us[i - 1] : 0.0;
      if (gb) gb[s * n + i] = -gg[i] * us[i];
      if (gc) gc[s * n + i] = i < n - 1 ? -gg[i] * us[i + 1] : 0.0;
    }
  }
  free(at);
}

/* ------------------------------------------------------------------------ */
/* Block tridiagonal Thomas.                                                 */
/* Follows gold_blkThomas_solve (block/src/blktrid_cpu.cpp:388-495) with the  */
/* inversion of gold_invert (:83-205; closed forms for M=2 :45-56 and M=3     */
/* :58-78, Gauss-Jordan with partial pivoting otherwise) and the vector ops   */
/* gold_MVmultiply (:330-361), gold_matAdd (:208-236), gold_vecAdd (:238-242).*/
/* The matrix product is the CORRECT one, Mans[i][j] = sum_k M1[i][k]*M2[k][j]*/
/* accumulated in k order; the reference's gold_MMmultiply (:301-326) reads   */
/* M2[i][j] instead of M2[k][j].                                             */
/* Blocks are MxM row-major.  layout 0 = the GPU's interleaved layout         */
/* [n][p][M*M] / [n][p][M] (blktrid_gpu.cuh:279-280,348); layout 1 = the CPU's*/
/* system-major layout [p][n][M*M] / [p][n][M] (blktrid_cpu.cpp:410-435).    */
/* transpose=1 solves the transposed block system (adjoint): sub-diagonal     */
/* C_{n-1}^T, diagonal B_n^T, super-diagonal A_{n+1}^T.                       */
/* ------------------------------------------------------------------------ */
static void blk_invert(int M, const double *in, double *inv) {
  double a[100];
  int i, j, q, p;
  memcpy(a, in, sizeof(double) * (size_t)(M * M));
  if (M == 1) { inv[0] = 1.0 / a[0]; return; }
  if (M == 2) {
    double det = a[0] * a[3] - a[1] * a[2];
    inv[0] = a[3] / det;
    inv[1] = (-1) * a[1] / det;
    inv[2] = (-1) * a[2] / det;
    inv[3] = a[0] / det;
    return;
  }
  if (M == 3) {
    double A0 = a[4] * a[8] - a[5] * a[7], D0 = -(a[1] * a[8] - a[2] * a[7]),
           G0 = (a[1] * a[5] - a[2] * a[4]), B0 = -(a[3] * a[8] - a[5] * a[6]),
           E0 = (a[0] * a[8] - a[2] * a[6]), H0 = -(a[0] * a[5] - a[2] * a[3]),
           C0 = (a[3] * a[7] - a[4] * a[6]), F0 = -(a[0] * a[7] - a[1] * a[6]),
           I0 = (a[0] * a[4] - a[1] * a[3]);
    double det = a[0] * A0 + a[1] * B0 + a[2] * C0;
    inv[0] = A0 / det; inv[1] = D0 / det; inv[2] = G0 / det;
    inv[3] = B0 / det; inv[4] = E0 / det; inv[5] = H0 / det;
    inv[6] = C0 / det; inv[7] = F0 / det; inv[8] = I0 / det;
    return;
  }
  for (i = 0; i < M; i++) {
    for (j = 0; j < M; j++) inv[M * i + j] = 0.0;
    inv[M * i + i] = 1.0;
  }
  for (i = 0; i < M; i++) {
    double best = fabs(a[i + M * i]), piv, r;
    p = i;
    for (j = i + 1; j < M; j++)
      if (fabs(a[M * j + i]) > best) { p = j; best = fabs(a[M * j + i]); }
    for (j = 0; j < M; j++) {
      double t = a[M * i + j]; a[M * i + j] = a[M * p + j]; a[M * p + j] = t;
      t = inv[M * i + j]; inv[M * i + j] = inv[M * p + j]; inv[M * p + j] = t;
    }
    piv = a[M * i + i];
    r = 1.0 / piv;
    for (j = 0; j < M; j++) { a[M * i + j] = a[M * i + j] * r; inv[M * i + j] = inv[M * i + j] * r; }
    for (q = 0; q < M; q++) {
      double f;
      if (q == i) continue;
      f = a[M * q + i];
      for (j = 0; j < M; j++) {
        a[M * q + j] = a[M * q + j] - f * a[M * i + j];
        inv[M * q + j] = inv[M * q + j] - f * inv[M * i + j];
      }
    }
  }
}

static void blk_mm(int M, const double *m1, const double *m2, double *out) {
  int i, j, k;
  for (i = 0; i < M * M; i++) out[i] = 0.0;
  for (i = 0; i < M; i++)
    for (k = 0; k < M; k++) {
      double t = m1[i * M + k];
      for (j = 0; j < M; j++) out[i * M + j] += t * m2[k * M + j];
    }
}

static void blk_mv(int M, const double *m, const double *v, double *out) {
  int i, j;
  for (i = 0; i < M; i++) {
    double acc = 0.0;
    for (j = 0; j < M; j++) acc += m[i * M + j] * v[j];
    out[i] = acc;
  }
}

static void blk_load(int M, const double *src, int transpose, double *dst) {
  int i, j;
  for (i = 0; i < M; i++)
    for (j = 0; j < M; j++) dst[i * M + j] = transpose ? src[j * M + i] : src[i * M + j];
}

int oracle_btsv_f64(const double *A, const double *B, const double *C, const double *d,
                    double *u, int N, int P, int M, int layout, int transpose) {
  const int E = M * M;
  double *Cs, *ds;
  double Ab[100], Bb[100], Cb[100], X[100], Xi[100], T[100], v[10], t[10];
  int p, n, i;
  if (M < 1 || M > 10 || N < 1 || P < 0) return 3;
  Cs = (double *)malloc(sizeof(double) * (size_t)N * E);
  ds = (double *)malloc(sizeof(double) * (size_t)N * M);
#define MOFF(nn) (layout == 0 ? ((int64_t)(nn) * P + p) * E : ((int64_t)p * N + (nn)) * E)
#define VOFF(nn) (layout == 0 ? ((int64_t)(nn) * P + p) * M : ((int64_t)p * N + (nn)) * M)
  for (p = 0; p < P; p++) {
    /* row 0 */
    blk_load(M, B + MOFF(0), transpose, Bb);
    if (transpose) { if (N > 1) blk_load(M, A + MOFF(1), 1, Cb); else memset(Cb, 0, sizeof(Cb)); }
    else blk_load(M, C + MOFF(0), 0, Cb);
    blk_invert(M, Bb, Xi);
    blk_mm(M, Xi, Cb, Cs);
    blk_mv(M, Xi, d + VOFF(0), ds);
    for (n = 1; n < N; n++) {
      if (transpose) {
        blk_load(M, C + MOFF(n - 1), 1, Ab);
        if (n + 1 < N) blk_load(M, A + MOFF(n + 1), 1, Cb); else memset(Cb, 0, sizeof(Cb));
      } else {
        blk_load(M, A + MOFF(n), 0, Ab);
        blk_load(M, C + MOFF(n), 0, Cb);
      }
      blk_load(M, B + MOFF(n), transpose, Bb);
      blk_mm(M, Ab, Cs + (int64_t)(n - 1) * E, T);           /* A_n C'_{n-1}      */
      for (i = 0; i < E; i++) X[i] = 1.0 * Bb[i] + (-1.0) * T[i]; /* B_n - A_n C'   */
      blk_invert(M, X, Xi);
      blk_mm(M, Xi, Cb, Cs + (int64_t)n * E);                /* C'_n = X^-1 C_n   */
      blk_mv(M, Ab, ds + (int64_t)(n - 1) * M, v);            /* A_n d'_{n-1}      */
      for (i = 0; i < M; i++) v[i] = 1.0 * d[VOFF(n) + i] + (-1.0) * v[i];
      blk_mv(M, Xi, v, ds + (int64_t)n * M);                  /* d'_n              */
    }
    for (i = 0; i < M; i++) u[VOFF(N - 1) + i] = ds[(int64_t)(N - 1) * M + i];
    for (n = N - 2; n >= 0; n--) {
      blk_mv(M, Cs + (int64_t)n * E, u + VOFF(n + 1), t);
      for (i = 0; i < M; i++) u[VOFF(n) + i] = 1.0 * ds[(int64_t)n * M + i] + (-1.0) * t[i];
    }
  }
#undef MOFF
#undef VOFF
  free(Cs);
  free(ds);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* ADI heat-diffusion time steps on an nx*ny*nz grid (x fastest).            */
/* Follows adi_orig.c:147-240 / preproc.hpp:172-214: boundary points get     */
/* d=0 and the identity row (a=c=0, b=1); interior points get                 */
/* d = lambda*(u[i-1]+u[i+1]+u[j-1]+u[j+1]+u[k-1]+u[k+1] - 6u) and the        */
/* coefficients (a_int, b_int, c_int); then x, y and z Thomas solves on d and */
/* u += d.  The reference app uses (-lambda/2, 1+lambda, -lambda/2).         */
/* ------------------------------------------------------------------------ */
void oracle_adi_f64(double *u, int nx, int ny, int nz, int iters, double lambda,
                    double a_int, double b_int, double c_int) {
  int64_t N = (int64_t)nx * ny * nz, ind;
  double *du = (double *)malloc(sizeof(double) * (size_t)N);
  double *ca = (double *)malloc(sizeof(double) * (size_t)N);
  double *cb = (double *)malloc(sizeof(double) * (size_t)N);
  double *cc = (double *)malloc(sizeof(double) * (size_t)N);
  int nmax = nx > ny ? nx : ny;
  double *w;
  int it, i, j, k;
  nmax = nmax > nz ? nmax : nz;
  w = (double *)malloc(sizeof(double) * 2 * (size_t)nmax);
  for (it = 0; it < iters; it++) {
    for (k = 0; k < nz; k++)
      for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
          ind = (int64_t)k * nx * ny + (int64_t)j * nx + i;
          if (i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1) {
            du[ind] = 0.0; ca[ind] = 0.0; cb[ind] = 1.0; cc[ind] = 0.0;
          } else {
            du[ind] = lambda * (u[ind - 1] + u[ind + 1] + u[ind - nx] + u[ind + nx] +
                                u[ind - (int64_t)nx * ny] + u[ind + (int64_t)nx * ny] -
                                6.0 * u[ind]);
            ca[ind] = a_int; cb[ind] = b_int; cc[ind] = c_int;
          }
        }
    for (k = 0; k < nz; k++)
      for (j = 0; j < ny; j++) {
        ind = (int64_t)k * nx * ny + (int64_t)j * nx;
        thomas_f64(ca + ind, 1, cb + ind, 1, cc + ind, 1, du + ind, 1, (double *)0, 1, nx, 0, w, w + nmax);
      }
    for (k = 0; k < nz; k++)
      for (i = 0; i < nx; i++) {
        ind = (int64_t)k * nx * ny + i;
        thomas_f64(ca + ind, nx, cb + ind, nx, cc + ind, nx, du + ind, nx, (double *)0, nx, ny, 0, w, w + nmax);
      }
    for (j = 0; j < ny; j++)
      for (i = 0; i < nx; i++) {
        ind = (int64_t)j * nx + i;
        thomas_f64(ca + ind, (int64_t)nx * ny, cb + ind, (int64_t)nx * ny, cc + ind, (int64_t)nx * ny,
                   du + ind, (int64_t)nx * ny, u + ind, (int64_t)nx * ny, nz, 1, w, w + nmax);
      }
  }
  free(w);
  free(du);
  free(ca);
  free(cb);
  free(cc);
}
