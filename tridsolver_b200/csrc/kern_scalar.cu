// Scalar batched tridiagonal kernels for sm_100a.
//
//  xsolve_kernel   solve axis 0 (unit stride inside a system): one warp per
//                  system, lane t owns rows [t*M, t*M+M) -> partitioned
//                  Thomas fully in registers (partition.cuh).  Replaces the
//                  reference's x-direction kernels (trid_linear*.hpp) and its
//                  cuBLAS-transpose x path (trid_cuda.cu:235-280).
//  strided_kernel  solve axis >= 1 (systems interleaved, consecutive systems
//                  adjacent in memory): a CTA owns SB adjacent systems; thread
//                  (system sl, chunk t) loads its M rows with warp-wide
//                  coalesced row segments, reduces its chunk, the SB warps
//                  solve one interface system each (lane = chunk), and every
//                  thread back-substitutes its chunk.  Replaces
//                  trid_strided_multidim.hpp:94-189 and the strided ThomasPCR
//                  (trid_thomaspcr.hpp:391-587).
//  generic_kernel  any length: one thread per system, Thomas in the
//                  reference's operation order (trid_cpu.cpp:360-401), c'/d' in
//                  library scratch laid out [row][system] so consecutive
//                  threads touch consecutive addresses.
#include "partition.cuh"

namespace tridb200 {

// ---------------------------------------------------------------------------
// solve axis 0
// ---------------------------------------------------------------------------
template <typename T, int M, int INC>
__global__ void __launch_bounds__(128) xsolve_kernel(Geom g, const T *__restrict__ a,
                                                     const T *__restrict__ b,
                                                     const T *__restrict__ c, T *__restrict__ d,
                                                     T *__restrict__ u) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t sys = (int64_t)blockIdx.x * (blockDim.x / kWarp) + (threadIdx.x / kWarp);
  if (sys >= g.nsys) return;  // uniform per warp
  int64_t off[5];
  system_offsets(g, sys, off);
  const int n = g.n;
  const int r0 = lane * M;

  T al[M], be[M], ga[M], de[M];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = r0 + j;
    if (r < n) {
      al[j] = (r == 0) ? T(0) : a[off[kA] + r];
      be[j] = b[off[kB] + r];
      ga[j] = (r == n - 1) ? T(0) : c[off[kC] + r];
      de[j] = d[off[kD] + r];
    } else {
      al[j] = T(0);
      be[j] = T(1);
      ga[j] = T(0);
      de[j] = T(0);
    }
  }
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  T xF, xL;
  warp_interface_solve(F, L, xF, xL, lane);
  chunk_backsub<T, M>(al, ga, de, xF, xL);
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = r0 + j;
    if (r < n) {
      if (INC)
        u[off[kU] + r] += de[j];
      else
        d[off[kD] + r] = de[j];
    }
  }
}

// ---------------------------------------------------------------------------
// solve axis >= 1
// ---------------------------------------------------------------------------
template <typename T, int M, int SB, int INC>
__global__ void __launch_bounds__(SB * kWarp) strided_kernel(Geom g, const T *__restrict__ a,
                                                             const T *__restrict__ b,
                                                             const T *__restrict__ c,
                                                             T *__restrict__ d,
                                                             T *__restrict__ u) {
  // interface rows, [component][chunk][system] (+1 pad against bank conflicts)
  __shared__ T red[8][kWarp][SB + 1];
  __shared__ T sol[2][kWarp][SB + 1];

  const int tid = threadIdx.x;
  const int sl = tid % SB;  // system within the tile (fastest: coalesced rows)
  const int t = tid / SB;   // chunk
  const int64_t sys = (int64_t)blockIdx.x * SB + sl;
  const bool valid = sys < g.nsys;
  int64_t off[5] = {0, 0, 0, 0, 0};
  if (valid) system_offsets(g, sys, off);
  const int n = g.n;
  const int r0 = t * M;
  const int64_t sa = g.stride[kA], sb = g.stride[kB], sc = g.stride[kC], sd = g.stride[kD];

  T al[M], be[M], ga[M], de[M];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = r0 + j;
    if (valid && r < n) {
      al[j] = (r == 0) ? T(0) : a[off[kA] + r * sa];
      be[j] = b[off[kB] + r * sb];
      ga[j] = (r == n - 1) ? T(0) : c[off[kC] + r * sc];
      de[j] = d[off[kD] + r * sd];
    } else {
      al[j] = T(0);
      be[j] = T(1);
      ga[j] = T(0);
      de[j] = T(0);
    }
  }
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  red[0][t][sl] = F.a;
  red[1][t][sl] = F.b;
  red[2][t][sl] = F.c;
  red[3][t][sl] = F.d;
  red[4][t][sl] = L.a;
  red[5][t][sl] = L.b;
  red[6][t][sl] = L.c;
  red[7][t][sl] = L.d;
  __syncthreads();
  {
    const int w = tid / kWarp;  // this warp solves the interface system of tile system w
    const int lane = tid & (kWarp - 1);
    const Row<T> F2{red[0][lane][w], red[1][lane][w], red[2][lane][w], red[3][lane][w]};
    const Row<T> L2{red[4][lane][w], red[5][lane][w], red[6][lane][w], red[7][lane][w]};
    T xF, xL;
    warp_interface_solve(F2, L2, xF, xL, lane);
    sol[0][lane][w] = xF;
    sol[1][lane][w] = xL;
  }
  __syncthreads();
  chunk_backsub<T, M>(al, ga, de, sol[0][t][sl], sol[1][t][sl]);
  if (!valid) return;
  const int64_t su = g.stride[kU];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = r0 + j;
    if (r < n) {
      if (INC)
        u[off[kU] + r * su] += de[j];
      else
        d[off[kD] + r * sd] = de[j];
    }
  }
}

// ---------------------------------------------------------------------------
// any length: Thomas, one thread per system
// ---------------------------------------------------------------------------
template <typename T, int INC>
__global__ void __launch_bounds__(128) generic_kernel(Geom g, const T *__restrict__ a,
                                                      const T *__restrict__ b,
                                                      const T *__restrict__ c,
                                                      T *__restrict__ d, T *__restrict__ u,
                                                      T *__restrict__ work, int64_t s0,
                                                      int64_t ns) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  int64_t off[5];
  system_offsets(g, s0 + k, off);
  const int64_t sa = g.stride[kA], sb = g.stride[kB], sc = g.stride[kC], sd = g.stride[kD],
                su = g.stride[kU];
  const int n = g.n;
  T *c2 = work + k;
  T *d2 = work + (int64_t)n * ns + k;
  const T *ap = a + off[kA];
  const T *bp = b + off[kB];
  const T *cp = c + off[kC];
  T *dp = d + off[kD];
  T *up = u + off[kU];

  T bb = T(1) / bp[0];
  T cc = (n > 1) ? bb * cp[0] : T(0);
  T dd = bb * dp[0];
  c2[0] = cc;
  d2[0] = dd;
  for (int i = 1; i < n; ++i) {
    const T aa = ap[i * sa];
    bb = bp[i * sb] - aa * cc;
    dd = dp[i * sd] - aa * dd;
    bb = T(1) / bb;
    cc = (i < n - 1) ? bb * cp[i * sc] : T(0);
    dd = bb * dd;
    c2[(int64_t)i * ns] = cc;
    d2[(int64_t)i * ns] = dd;
  }
  if (INC)
    up[(int64_t)(n - 1) * su] += dd;
  else
    dp[(int64_t)(n - 1) * sd] = dd;
  for (int i = n - 2; i >= 0; --i) {
    dd = d2[(int64_t)i * ns] - c2[(int64_t)i * ns] * dd;
    if (INC)
      up[i * su] += dd;
    else
      dp[i * sd] = dd;
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename T, int INC>
cudaError_t launch_xsolve(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u, int chunk,
                          cudaStream_t st) {
  constexpr int kWarpsPerCta = 4;
  const int64_t blocks = (g.nsys + kWarpsPerCta - 1) / kWarpsPerCta;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  const dim3 grid((unsigned)blocks), block(kWarpsPerCta * kWarp);
  switch (chunk) {
    case 2: xsolve_kernel<T, 2, INC><<<grid, block, 0, st>>>(g, a, b, c, d, u); break;
    case 4: xsolve_kernel<T, 4, INC><<<grid, block, 0, st>>>(g, a, b, c, d, u); break;
    case 8: xsolve_kernel<T, 8, INC><<<grid, block, 0, st>>>(g, a, b, c, d, u); break;
    case 16: xsolve_kernel<T, 16, INC><<<grid, block, 0, st>>>(g, a, b, c, d, u); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename T, int M, int INC>
static cudaError_t launch_strided_m(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u,
                                    int spc, cudaStream_t st) {
  auto go = [&](auto kern, int sb) {
    const int64_t blocks = (g.nsys + sb - 1) / sb;
    if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
    kern<<<dim3((unsigned)blocks), dim3(sb * kWarp), 0, st>>>(g, a, b, c, d, u);
    return cudaGetLastError();
  };
  switch (spc) {
    case 4: return go(strided_kernel<T, M, 4, INC>, 4);
    case 8: return go(strided_kernel<T, M, 8, INC>, 8);
    case 16: return go(strided_kernel<T, M, 16, INC>, 16);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T, int INC>
cudaError_t launch_strided(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u,
                           int chunk, int spc, cudaStream_t st) {
  switch (chunk) {
    case 2: return launch_strided_m<T, 2, INC>(g, a, b, c, d, u, spc, st);
    case 4: return launch_strided_m<T, 4, INC>(g, a, b, c, d, u, spc, st);
    case 8: return launch_strided_m<T, 8, INC>(g, a, b, c, d, u, spc, st);
    case 16: return launch_strided_m<T, 16, INC>(g, a, b, c, d, u, spc, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T, int INC>
cudaError_t launch_generic(const Geom &g, const T *a, const T *b, const T *c, T *d, T *u, T *work,
                           int64_t work_systems, cudaStream_t st) {
  for (int64_t s0 = 0; s0 < g.nsys; s0 += work_systems) {
    const int64_t ns = (g.nsys - s0 < work_systems) ? (g.nsys - s0) : work_systems;
    const int64_t blocks = (ns + 127) / 128;
    generic_kernel<T, INC><<<dim3((unsigned)blocks), dim3(128), 0, st>>>(g, a, b, c, d, u, work,
                                                                         s0, ns);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

#define TRID_INSTANTIATE(T, INC)                                                               \
  template cudaError_t launch_xsolve<T, INC>(const Geom &, const T *, const T *, const T *, T *, \
                                             T *, int, cudaStream_t);                          \
  template cudaError_t launch_strided<T, INC>(const Geom &, const T *, const T *, const T *,    \
                                              T *, T *, int, int, cudaStream_t);               \
  template cudaError_t launch_generic<T, INC>(const Geom &, const T *, const T *, const T *,    \
                                              T *, T *, T *, int64_t, cudaStream_t);

TRID_INSTANTIATE(float, 0)
TRID_INSTANTIATE(float, 1)
TRID_INSTANTIATE(double, 0)
TRID_INSTANTIATE(double, 1)

}  // namespace tridb200
