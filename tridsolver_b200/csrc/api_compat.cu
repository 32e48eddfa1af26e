// 11-argument GPU form of the strided-batch API (libtridb200_cudacompat.so).
//
// Same symbol names as scalar/include/trid_cuda.h:57-80, which take
// `int *opts, int sync` after pads; C cannot overload, so this form ships as a
// separate library built from the same sources (api_scalar.cu is compiled
// with TRID_CUDACOMPAT, dropping its 9-argument exports).  `opts[solvedim]`
// is an algorithm hint (0 automatic, 1/2 Thomas, 3/4 Thomas-PCR hybrid, 5
// automatic; anything else is INVALID_VALUE); `sync == 1` waits for the solve
// before returning (the reference forces this, trid_cuda.cu:519-520).
// The compat header must come first: it declares the 11-argument forms
// under the names the 9-argument header would otherwise claim.
#include "../../include/trid_b200_cudacompat.h"
#include "dispatch.cuh"

using namespace tridb200;

extern "C" tridStatus_t tridSmtsvStridedBatch(const float *a, const float *b, const float *c,
                                              float *d, float *u, int ndim, int solvedim,
                                              int *dims, int *pads, int *opts, int sync) {
  (void)u;
  const int *p[5] = {pads, pads, pads, pads, pads};
  return solve_strided_batch<float, 0>(a, b, c, d, nullptr, ndim, solvedim, dims, p, opts, sync);
}

extern "C" tridStatus_t tridDmtsvStridedBatch(const double *a, const double *b, const double *c,
                                              double *d, double *u, int ndim, int solvedim,
                                              int *dims, int *pads, int *opts, int sync) {
  (void)u;
  const int *p[5] = {pads, pads, pads, pads, pads};
  return solve_strided_batch<double, 0>(a, b, c, d, nullptr, ndim, solvedim, dims, p, opts, sync);
}

extern "C" tridStatus_t tridSmtsvStridedBatchInc(const float *a, const float *b, const float *c,
                                                 float *d, float *u, int ndim, int solvedim,
                                                 int *dims, int *pads, int *opts, int sync) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  return solve_strided_batch<float, 1>(a, b, c, d, u, ndim, solvedim, dims, p, opts, sync);
}

extern "C" tridStatus_t tridDmtsvStridedBatchInc(const double *a, const double *b,
                                                 const double *c, double *d, double *u, int ndim,
                                                 int solvedim, int *dims, int *pads, int *opts,
                                                 int sync) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  return solve_strided_batch<double, 1>(a, b, c, d, u, ndim, solvedim, dims, p, opts, sync);
}
