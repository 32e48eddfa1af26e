/*
 * tridsolver_b200 -- block-tridiagonal batched solve (libtridb200.so and
 * libtridb200_cudacompat.so).
 *
 * Systems A_n x_{n-1} + B_n x_n + C_n x_{n+1} = d_n (n = 0..N-1) of P
 * independent problems with M x M blocks (M = 1..10), row-major, in the
 * reference GPU's interleaved layout: block (n, p) starts at (n*P + p)*M*M,
 * vector (n, p) at (n*P + p)*M.  A_0 and C_{N-1} are never read.  Device
 * pointers; work is enqueued on the calling thread's stream (tridSetStream).
 */
#ifndef BLKTRID_B200_H
#define BLKTRID_B200_H

#include "trid_b200.h"

/* Replaces block/include/blktrid_gpu.h:38-40 (dbtsv_gpu / sbtsv_gpu) with a
 * status return.  x receives the solution; Cstar (N*P*M*M) and dstar (N*P*M)
 * are scratch for the modified blocks, as in the reference; pass NULL for
 * both to use library scratch. */
TRID_EXTERN_C tridStatus_t tridDbtsvBatch(const double *A, const double *B, const double *C,
                                          const double *d, double *x, int N, int P, int M,
                                          double *Cstar, double *dstar);
TRID_EXTERN_C tridStatus_t tridSbtsvBatch(const float *A, const float *B, const float *C,
                                          const float *d, float *x, int N, int P, int M,
                                          float *Cstar, float *dstar);

/* Adjoint (no reference counterpart): for the forward solution u and the
 * cotangent w = dL/dx, solves the transposed block system (sub-diagonal
 * C_{n-1}^T, diagonal B_n^T, super-diagonal A_{n+1}^T) for g and writes
 * dA_n = -g_n u_{n-1}^T, dB_n = -g_n u_n^T, dC_n = -g_n u_{n+1}^T, dd_n = g_n
 * (dA_0 = dC_{N-1} = 0).  Any output may be NULL; outputs must not alias the
 * inputs. */
TRID_EXTERN_C tridStatus_t tridDbtsvBatchAdjoint(const double *A, const double *B,
                                                 const double *C, const double *u,
                                                 const double *w, double *dA, double *dB,
                                                 double *dC, double *dd, int N, int P, int M);
TRID_EXTERN_C tridStatus_t tridSbtsvBatchAdjoint(const float *A, const float *B, const float *C,
                                                 const float *u, const float *w, float *dA,
                                                 float *dB, float *dC, float *dd, int N, int P,
                                                 int M);

#ifdef __cplusplus
/* The reference's own entry points, same C++ linkage, argument order and
 * meaning (block/include/blktrid_gpu.h:38-40): the solution lands in u.  They
 * do not print or synchronise (the reference does both,
 * blktrid_gpu.cu:61,136-138); use the tridXbtsvBatch forms for a status. */
void sbtsv_gpu(float *A, float *B, float *C, float *d, float *Cstar, float *dstar, float *u,
               const int N, const int P, const int blkdim);
void dbtsv_gpu(double *A, double *B, double *C, double *d, double *Cstar, double *dstar, double *u,
               const int N, const int P, const int blkdim);
#endif

#endif /* BLKTRID_B200_H */
