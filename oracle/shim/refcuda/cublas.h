/* Test infrastructure: stands in for the legacy cuBLAS header that the
 * reference's cutil_inline.h includes, so that its GPU library (which also
 * includes cublas_v2.h) compiles with CUDA 12: the v2 API plus the one
 * legacy type name the reference uses. */
#include <cublas_v2.h>
typedef cublasStatus_t cublasStatus;
