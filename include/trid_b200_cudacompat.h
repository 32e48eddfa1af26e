/*
 * tridsolver_b200 -- 11-argument GPU form of the strided-batch API, exported by
 * libtridb200_cudacompat.so (built from the same sources as libtridb200.so).
 *
 * Replaces scalar/include/trid_cuda.h:44-80 symbol for symbol, so callers
 * written against the reference GPU library (apps/adi/src/adi_cuda.cu:297-326,
 * scalar/test/test_cuda.cu:40-56) link unchanged.  Pointers are device
 * pointers; dims, pads and opts are host arrays.
 *   opts[solvedim]: 0/5 automatic, 1/2 Thomas, 3/4 Thomas-PCR hybrid (a hint;
 *                   the reference picks kernels with it, trid_cuda.cu:98-168);
 *                   other values return TRID_STATUS_INVALID_VALUE.  opts may
 *                   be NULL.
 *   sync == 1:      the call waits for the solve to complete.
 * The Padded forms, initTridMultiDimBatchSolve and the extensions
 * (tridSetStream, ...) have the same signatures as in trid_b200.h and are
 * exported by this library too.
 */
#ifndef TRID_B200_CUDACOMPAT_H
#define TRID_B200_CUDACOMPAT_H

#define tridSmtsvStridedBatch tridSmtsvStridedBatch_9arg_unused
#define tridDmtsvStridedBatch tridDmtsvStridedBatch_9arg_unused
#define tridSmtsvStridedBatchInc tridSmtsvStridedBatchInc_9arg_unused
#define tridDmtsvStridedBatchInc tridDmtsvStridedBatchInc_9arg_unused
#include "trid_b200.h"
#undef tridSmtsvStridedBatch
#undef tridDmtsvStridedBatch
#undef tridSmtsvStridedBatchInc
#undef tridDmtsvStridedBatchInc

/* trid_cuda.h:57 */
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatch(const float *a, const float *b, const float *c,
                                                 float *d, float *u, int ndim, int solvedim,
                                                 int *dims, int *pads, int *opts, int sync);
/* trid_cuda.h:59 */
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatch(const double *a, const double *b,
                                                 const double *c, double *d, double *u, int ndim,
                                                 int solvedim, int *dims, int *pads, int *opts,
                                                 int sync);
/* trid_cuda.h:74 */
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchInc(const float *a, const float *b,
                                                    const float *c, float *d, float *u, int ndim,
                                                    int solvedim, int *dims, int *pads, int *opts,
                                                    int sync);
/* trid_cuda.h:76 */
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatchInc(const double *a, const double *b,
                                                    const double *c, double *d, double *u,
                                                    int ndim, int solvedim, int *dims, int *pads,
                                                    int *opts, int sync);

#endif /* TRID_B200_CUDACOMPAT_H */
