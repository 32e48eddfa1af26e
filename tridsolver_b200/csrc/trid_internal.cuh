// Internal declarations shared by the tridsolver_b200 CUDA sources.
//
// Everything here is sm_100a device code or C++ host code of the library;
// the public C ABI lives in include/trid_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

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
  // division by odims[k] as multiply-high + shifts (valid when nsys < 2^32),
  // see fastdiv below
  uint32_t dmul[kMaxDim];
  uint32_t dshift[kMaxDim];      // 0xffffffff marks a divisor of 1
  int fastdiv;
};

// Unsigned 32-bit division by an invariant divisor d >= 1 without a hardware
// divide (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, sec. 4): with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1,  q = (t + ((n - t) >> 1)) >> (l - 1),
// t = mulhi(m, n), exact for every 32-bit n.
inline void fastdiv_setup(uint32_t d, uint32_t &mul, uint32_t &shift) {
  if (d <= 1) {
    mul = 0;
    shift = 0xffffffffu;
    return;
  }
  uint32_t l = 0;
  while (((uint64_t)1 << l) < d) ++l;
  mul = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << l) - d)) / d + 1);
  shift = l;
}

__host__ __device__ __forceinline__ uint32_t fastdiv(uint32_t n, uint32_t mul, uint32_t shift) {
  if (shift == 0xffffffffu) return n;
#ifdef __CUDA_ARCH__
  const uint32_t t = __umulhi(mul, n);
#else
  const uint32_t t = (uint32_t)(((uint64_t)mul * n) >> 32);
#endif
  return (t + ((n - t) >> 1)) >> (shift - 1);
}

enum Arr { kA = 0, kB = 1, kC = 2, kD = 3, kU = 4 };

// Offsets of system s in each of the 5 arrays.
__host__ __device__ __forceinline__ void system_offsets(const Geom &g, int64_t s, int64_t off[5]) {
#pragma unroll
  for (int q = 0; q < 5; ++q) off[q] = 0;
  if (g.fastdiv) {
    uint32_t r = (uint32_t)s;
    for (int k = 0; k < g.nod; ++k) {
      const uint32_t qk = fastdiv(r, g.dmul[k], g.dshift[k]);
      const int64_t i = (int64_t)(r - qk * (uint32_t)g.odims[k]);
      r = qk;
#pragma unroll
      for (int q = 0; q < 5; ++q) off[q] += i * g.ocum[q][k];
    }
    return;
  }
  for (int k = 0; k < g.nod; ++k) {
    const int64_t e = g.odims[k];
    const int64_t i = s % e;
    s /= e;
#pragma unroll
    for (int q = 0; q < 5; ++q) off[q] += i * g.ocum[q][k];
  }
}

// Reciprocal: the hardware approximation (rcp.approx.ftz) refined by
// Newton-Raphson steps y <- y + y*(1 - x*y), each of which squares the
// relative error; two steps for FP64 and one for FP32 reach the last bit
// (within 1 ulp of the correctly rounded value).  Measured on B200 this is
// ~1.6x the throughput of the correctly rounded __drcp_rn, whose FP64
// special-function pipe is the scarce resource of these kernels.
__device__ __forceinline__ double rcp(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}
__device__ __forceinline__ float rcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  const float e = fmaf(-x, y, 1.0f);
  return fmaf(y, e, y);
}

// Per-thread library state (stream), defined in api_scalar.cu.
cudaStream_t current_stream();

// Device scratch held for the duration of one call on `stream` (the object
// lives in the scope that enqueues every launch using it).  Outside stream capture it is a
// grow-only buffer kept per (device, stream, nesting level): calls on one
// stream run in order and share it, calls on other streams get their own, and
// a long-system solve at level L solves its block system at level L+1, so
// levels never share a buffer.  While the stream is being
// captured into a CUDA graph it is a stream-ordered allocation freed when the
// object goes out of scope, so the graph carries its own allocate and free
// nodes and never refers to a buffer that a later call may replace.  get() is
// nullptr for 0 bytes and on allocation failure.
class Scratch {
 public:
  Scratch(size_t bytes, int level, cudaStream_t stream);
  ~Scratch();
  Scratch(const Scratch &) = delete;
  Scratch &operator=(const Scratch &) = delete;
  void *get() const { return ptr_; }

 private:
  void *ptr_ = nullptr;
  cudaStream_t stream_ = nullptr;
  bool stream_ordered_ = false;
};

// Per-device word of error bits set by kernels whose bounded waits gave up
// (read and cleared by tridGetDeviceErrors).  nullptr if it cannot be made.
unsigned *device_error_flags();
// The same word when it exists already on the current device (nullptr if no
// kernel has needed it yet); never allocates.
unsigned *device_error_flags_if_present();
// Length-bucket cut-offs of the variable-length batch (api_scalar.cu): rows
// per lane 2 up to m2max, 4 up to m4max, else 8; from the tuning table.
void varlen_buckets(int dtype_bytes, int &m2max, int &m4max);
// The allocation-free varlen solve's own error word on the current device
// (kern_varlen.cu), nullptr until that entry point has run there.
unsigned *noalloc_error_word();

// Kernel launchers (return cudaSuccess or the launch error).
template <typename T, int INC>
cudaError_t launch_xsolve(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u,
                          int chunk, cudaStream_t st);
template <typename T, int INC>
cudaError_t launch_strided(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u,
                           int chunk, int sys_per_cta, cudaStream_t st);
template <typename T, int INC>
cudaError_t launch_xsolve_tma(const Geom &g, const int *const pads[5], int ndim, const T *a,
                              const T *b, const T *c, T *d, T *u, int chunk, unsigned *err,
                              cudaStream_t st);
template <typename T, int INC>
cudaError_t launch_strided_part_tma(const Geom &g, const int *dims, const int *const pads[5],
                                    int ndim, int solvedim, const T *a, const T *b, const T *c,
                                    T *d, T *u, int chunk, int spc, bool prefetch,
                                    unsigned *err, cudaStream_t st);
// general partitioned kernels (kern_general.cu)
enum GenModeId { kGenFwd = 0, kGenFwdInc = 1, kGenAdj = 2 };
enum GenPhaseId { kGenSingle = 0, kGenReduce = 1, kGenFinish = 2 };
template <typename T>
struct GenArgs {
  const T *a, *b, *c;
  const T *rhs;    // d (forward) or w = dL/dx (adjoint)
  const T *usol;   // adjoint: the forward solution
  T *out;          // forward: d (non-Inc) or u (Inc)
  T *ga, *gb, *gc, *gd;  // adjoint outputs, each may be null
  T *red;          // reduce phase: block rows, 4 arrays of nsys*2*nblk (a, b, c, d)
  const T *bsol;   // finish phase: block unknowns, nsys*2*nblk
  int nblk;        // blocks per system
};
template <typename T, int MODE>
cudaError_t launch_general_phase(const Geom &g, const GenArgs<T> &A, int axis, int chunk, int spc,
                                 int phase, cudaStream_t st);

// one-CTA-per-system blocked partition on axis 0 (kern_xcta.cu)
enum XModeIdPub { kXcFwd = 0, kXcFwdInc = 1, kXcAdj = 2, kXcFused = 3 };
template <typename T>
struct XArgs {
  const T *a, *b, *c, *d;
  const T *w;
  const T *usol;
  T *x;
  T *ga, *gb, *gc, *gd;
};
template <typename T, int MODE>
cudaError_t launch_xcta(const Geom &g, const XArgs<T> &A, int chunk, cudaStream_t st);
// the variable-length batch's systems of kVarlenShort+1 .. 512*kVarlenCtaBuckets
// rows, one CTA of W = ceil(n/512) warps each: bucket W-1 lists its systems
// (lists + (W-1)*list_stride, counts[W-1] of them); solved in place in d.
// counts[kVarlenClaims + k] is list k's claim counter (zero before the
// launch): CTAs take the list's systems one at a time from it.
constexpr int kVarlenShort = 256;
constexpr int kVarlenCtaBuckets = 8;
constexpr int kVarlenClaims = 16;
template <typename T>
cudaError_t launch_xcta_varlen(const T *a, const T *b, const T *c, T *d, const int64_t *offsets,
                               const int *lists, int64_t list_stride, unsigned *counts,
                               cudaStream_t st);
template <typename T, int INC>
cudaError_t launch_generic(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u,
                           T *work, int64_t work_systems, cudaStream_t st);

// systems split along the solve axis across ranks (kern_split.cu): a slab's
// six boundary numbers [6][nsys] in FP64; the gathered slabs [nranks][6][nsys]
// turned into the slab's patched first and last d (old values to `saved`,
// [2][nsys], when not null); their restore
template <typename T>
cudaError_t launch_split_reduce(const Geom &g, const T *a, const T *b, const T *c, const T *d,
                                double *bnd, cudaStream_t st);
template <typename T>
cudaError_t launch_split_patch(const Geom &g, const T *a, const T *c, T *d, const double *bnd_all,
                               int nranks, int rank, T *saved, cudaStream_t st);
template <typename T>
cudaError_t launch_split_restore(const Geom &g, T *d, const T *saved, cudaStream_t st);

// Programmatic dependent launch.  A kernel launched by launch_pdl may be
// scheduled while the previous kernel on the stream finishes; it calls
// pdl_enter() before its first global access, which waits for that kernel
// to complete (its writes visible) and lets the next kernel be scheduled
// once every CTA of this grid has started, so a dependent grid only takes
// the slots this one has left.  Launched without the attribute, pdl_enter()
// does nothing.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*kern)(P...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, A &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

}  // namespace tridb200
