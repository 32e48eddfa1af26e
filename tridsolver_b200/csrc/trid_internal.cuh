// Internal declarations shared by the tridsolver_b200 CUDA sources.
//
// Everything here is sm_100a device code or C++ host code of the library;
// the public C ABI lives in include/trid_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/trid_b200.h"

namespace tridb200 {

constexpr int kMaxDim = 8;        // dims/pads entries accepted (the reference GPU path decodes up to 8)
constexpr int kWarp = 32;

// Geometry of one strided-batch call, flattened for the kernels.
//
// A "system" is one line along `solvedim`.  Systems are numbered s = 0..nsys-1
// with the non-solve axes in their original order, dims[0] fastest; so for a
// solve along axis >= 1 consecutive s are consecutive addresses (coalesced).
// For each of the five arrays (a,b,c,d,u) element (i_0, ..., i_{ndim-1}) sits
// at sum_k i_k * prod_{j<k} pads_X[j].
struct Geom {
  int64_t nsys;                  // number of systems
  int n;                         // system length (dims[solvedim])
  int nod;                       // number of non-solve axes (ndim - 1)
  int odims[kMaxDim];            // extents of the non-solve axes, fastest first
  int64_t ocum[5][kMaxDim];      // per array: element stride of each non-solve axis
  int64_t stride[5];             // per array: element stride along the solve axis
};

enum Arr { kA = 0, kB = 1, kC = 2, kD = 3, kU = 4 };

// Offsets of system s in each of the 5 arrays.
__host__ __device__ __forceinline__ void system_offsets(const Geom &g, int64_t s, int64_t off[5]) {
#pragma unroll
  for (int q = 0; q < 5; ++q) off[q] = 0;
  for (int k = 0; k < g.nod; ++k) {
    const int64_t e = g.odims[k];
    const int64_t i = s % e;
    s /= e;
#pragma unroll
    for (int q = 0; q < 5; ++q) off[q] += i * g.ocum[q][k];
  }
}

// Reciprocal, correctly rounded (IEEE round-to-nearest).
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }

// Per-thread library state (stream), defined in api_scalar.cu.
cudaStream_t current_stream();

// Device scratch owned by the library (grow-only, per device).  Returns
// nullptr on allocation failure.
void *scratch(size_t bytes);

// Kernel launchers (return cudaSuccess or the launch error).
template <typename T, int INC>
cudaError_t launch_xsolve(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u,
                          int chunk, cudaStream_t st);
template <typename T, int INC>
cudaError_t launch_strided(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u,
                           int chunk, int sys_per_cta, cudaStream_t st);
template <typename T, int INC>
cudaError_t launch_generic(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u,
                           T *work, int64_t work_systems, cudaStream_t st);

}  // namespace tridb200
