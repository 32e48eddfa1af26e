// Strided-batch solves over element types beyond FP32/FP64 (sm_100a).
//
//  * complex<float>, complex<double>: interleaved (re, im) pairs, the layout
//    of cuComplex / cuDoubleComplex, std::complex and C99 _Complex.  The
//    reference declares these forms and leaves them commented out
//    (scalar/include/trid_cuda.h:39-52, scalar/src/cuda/trid_cuda.cu:468-600,
//    tridMultiDimBatchSolve<complexf/complexd>); the algorithm is the real
//    one in complex arithmetic, without pivoting.
//  * FP32 storage with FP64 arithmetic ("mixed"): every load widens to
//    double, the whole solve runs in double and each result is rounded to
//    float once (Inc: u = float(double(u) + x)).
//
// S is the storage type, T the arithmetic type.  The solvers are the
// partitioned Thomas building blocks of partition.cuh instantiated for T:
//
//  ext_x_kernel       axis 0 (unit stride), n <= 32*M: one warp per system,
//                     lane t owns rows [t*M, t*M+M).
//  ext_stream_kernel  axes >= 1, n <= 256 (tile within 200 KB of shared
//                     memory): persistent, one CTA per SM; tiles of SB
//                     systems x n rows stream through shared memory by
//                     cp.async while the previous tile is solved.
//  ext_strided_kernel the other axes >= 1 cases up to 512 rows: a CTA owns
//                     SB adjacent systems x 32 chunks; the interface rows go
//                     through shared memory to one warp per system.
//  ext_thomas_kernel  longer systems: one thread per system, Thomas with
//                     c'/d' in library scratch laid out [row][system] (in T).
// The longest chunk is 16 rows for 8-byte T and 8 for complex<double>.
#include <string.h>

#include <type_traits>

#include "partition.cuh"
#include "tma.cuh"
#include "trid_b200.h"

namespace tridb200 {

// ------------------------------------------------------------ complex T --
template <typename R>
struct Cx {
  R x, y;
  Cx() = default;
  __host__ __device__ constexpr Cx(R re) : x(re), y(R(0)) {}
  __host__ __device__ constexpr Cx(R re, R im) : x(re), y(im) {}
};

template <typename R>
__device__ __forceinline__ Cx<R> operator+(const Cx<R> &p, const Cx<R> &q) {
  return {p.x + q.x, p.y + q.y};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator-(const Cx<R> &p, const Cx<R> &q) {
  return {p.x - q.x, p.y - q.y};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator-(const Cx<R> &p) {
  return {-p.x, -p.y};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator*(const Cx<R> &p, const Cx<R> &q) {
  return {p.x * q.x - p.y * q.y, p.x * q.y + p.y * q.x};
}
template <typename R>
__device__ __forceinline__ Cx<R> &operator*=(Cx<R> &p, const Cx<R> &q) {
  p = p * q;
  return p;
}

// 1/z by Smith's scaling (R. L. Smith, "Algorithm 116: Complex division",
// CACM 5(8), 1962): divide through by the larger component so that no
// intermediate squares the magnitude.
template <typename R>
__device__ __forceinline__ Cx<R> rcp(const Cx<R> &z) {
  if (fabs(z.x) >= fabs(z.y)) {
    const R r = z.y * rcp(z.x);
    const R t = rcp(z.x + z.y * r);
    return {t, -r * t};
  }
  const R r = z.x * rcp(z.y);
  const R t = rcp(z.x * r + z.y);
  return {r * t, -t};
}

// warp shuffles of a complex value (found by argument-dependent lookup from
// the partition.cuh templates)
template <typename R>
__device__ __forceinline__ Cx<R> __shfl_down_sync(unsigned m, const Cx<R> &v, unsigned s,
                                                  int w = 32) {
  return {::__shfl_down_sync(m, v.x, s, w), ::__shfl_down_sync(m, v.y, s, w)};
}
template <typename R>
__device__ __forceinline__ Cx<R> __shfl_up_sync(unsigned m, const Cx<R> &v, unsigned s,
                                                int w = 32) {
  return {::__shfl_up_sync(m, v.x, s, w), ::__shfl_up_sync(m, v.y, s, w)};
}

// ------------------------------------------------- storage <-> arithmetic --
template <typename S, typename T>
struct Elem;
template <>
struct Elem<float, double> {
  static __device__ __forceinline__ double ld(const float *p) { return (double)__ldg(p); }
  static __device__ __forceinline__ double ldw(const float *p) { return (double)*p; }
  static __device__ __forceinline__ void st(float *p, double v) { *p = (float)v; }
  static __device__ __forceinline__ double cv(float v) { return (double)v; }
};
template <>
struct Elem<float2, Cx<float>> {
  static __device__ __forceinline__ Cx<float> ld(const float2 *p) {
    const float2 v = __ldg(p);
    return {v.x, v.y};
  }
  static __device__ __forceinline__ Cx<float> ldw(const float2 *p) {
    const float2 v = *p;
    return {v.x, v.y};
  }
  static __device__ __forceinline__ void st(float2 *p, Cx<float> v) { *p = make_float2(v.x, v.y); }
  static __device__ __forceinline__ Cx<float> cv(float2 v) { return {v.x, v.y}; }
};
template <>
struct Elem<double2, Cx<double>> {
  static __device__ __forceinline__ Cx<double> ld(const double2 *p) {
    const double2 v = __ldg(p);
    return {v.x, v.y};
  }
  static __device__ __forceinline__ Cx<double> ldw(const double2 *p) {
    const double2 v = *p;
    return {v.x, v.y};
  }
  static __device__ __forceinline__ void st(double2 *p, Cx<double> v) {
    *p = make_double2(v.x, v.y);
  }
  static __device__ __forceinline__ Cx<double> cv(double2 v) { return {v.x, v.y}; }
};

// x -> d (INC = 0) or u += x (INC = 1)
template <typename S, typename T, int INC>
__device__ __forceinline__ void ext_out(S *d, S *u, T x) {
  using E = Elem<S, T>;
  if (INC)
    E::st(u, E::ldw(u) + x);
  else
    E::st(d, x);
}

// Element-wise asynchronous global -> shared copies of 4, 8 or 16 bytes
// (cp.async; 16-byte copies bypass L1)
template <int B>
__device__ __forceinline__ void cp_async_elem(void *dst, const void *src) {
  if constexpr (B == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src),
                 "n"(B)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ------------------------------------------------------------- kernels --
// M consecutive elements as 16-byte accesses (M * sizeof(S) a multiple of 16,
// p 16-byte aligned)
template <typename S, int M, bool NC>
__device__ __forceinline__ void load16(const S *p, S (&v)[M]) {
  constexpr int K = M * (int)sizeof(S) / 16;
  static_assert(K * 16 == M * (int)sizeof(S), "whole 16-byte words");
  const uint4 *q = reinterpret_cast<const uint4 *>(p);
  uint4 w[K];
#pragma unroll
  for (int k = 0; k < K; ++k) w[k] = NC ? __ldg(q + k) : q[k];
  memcpy(v, w, sizeof(w));
}
template <typename S, int M>
__device__ __forceinline__ void store16(S *p, const S (&v)[M]) {
  constexpr int K = M * (int)sizeof(S) / 16;
  uint4 w[K];
  memcpy(w, v, sizeof(w));
  uint4 *q = reinterpret_cast<uint4 *>(p);
#pragma unroll
  for (int k = 0; k < K; ++k) q[k] = w[k];
}

// Axis 0: one warp per system, lane = chunk of M rows.  VEC: n == 32*M and
// every array's rows 16-byte aligned, so a lane reads and writes its chunk
// as 16-byte words instead of one element at a time.
template <typename S, typename T, int M, int INC, bool VEC>
__global__ void __launch_bounds__(128) ext_x_kernel(Geom g, const S *__restrict__ a,
                                                    const S *__restrict__ b,
                                                    const S *__restrict__ c, S *__restrict__ d,
                                                    S *__restrict__ u) {
  using E = Elem<S, T>;
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t sys = (int64_t)blockIdx.x * (blockDim.x / kWarp) + (threadIdx.x / kWarp);
  if (sys >= g.nsys) return;  // uniform per warp
  int64_t off[5];
  system_offsets(g, sys, off);
  const int n = VEC ? kWarp * M : g.n;
  const int r0 = lane * M;
  T al[M], be[M], ga[M], de[M];
  if constexpr (VEC) {
    S va[M], vb[M], vc[M], vd[M];
    load16<S, M, true>(a + off[kA] + r0, va);
    load16<S, M, true>(b + off[kB] + r0, vb);
    load16<S, M, true>(c + off[kC] + r0, vc);
    load16<S, M, false>(d + off[kD] + r0, vd);
#pragma unroll
    for (int j = 0; j < M; ++j) {
      al[j] = (j == 0 && lane == 0) ? T(0) : E::cv(va[j]);
      be[j] = E::cv(vb[j]);
      ga[j] = (j == M - 1 && lane == kWarp - 1) ? T(0) : E::cv(vc[j]);
      de[j] = E::cv(vd[j]);
    }
  } else {
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int r = r0 + j;
      if (r < n) {
        al[j] = (r == 0) ? T(0) : E::ld(a + off[kA] + r);
        be[j] = E::ld(b + off[kB] + r);
        ga[j] = (r == n - 1) ? T(0) : E::ld(c + off[kC] + r);
        de[j] = E::ldw(d + off[kD] + r);
      } else {
        al[j] = T(0);
        be[j] = T(1);
        ga[j] = T(0);
        de[j] = T(0);
      }
    }
  }
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  T xF, xL;
  warp_interface_solve(F, L, xF, xL, lane);
  chunk_backsub<T, M>(al, ga, de, xF, xL);
  if constexpr (VEC) {
    S vx[M];
    if constexpr (INC) load16<S, M, false>(u + off[kU] + r0, vx);
#pragma unroll
    for (int j = 0; j < M; ++j) E::st(vx + j, INC ? E::cv(vx[j]) + de[j] : de[j]);
    store16<S, M>((INC ? u + off[kU] : d + off[kD]) + r0, vx);
  } else {
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int r = r0 + j;
      if (r < n) ext_out<S, T, INC>(d + off[kD] + r, INC ? u + off[kU] + r : nullptr, de[j]);
    }
  }
}

// Axis 0, whole systems (n == 32*M): one warp per system; the system's rows
// of every array arrive by coalesced cp.async copies (32 consecutive
// elements per warp copy) in shared memory, row i of an array at slot
// i + i/M (one pad slot per chunk, so lane l's chunk starts at l*(M+1) and
// the lanes' reads of a row fall in distinct banks); each lane takes its
// chunk from there, and the solution leaves the same way (written into the
// right-hand-side slots, then stored by coalesced warp stores).  Used for
// elements of 16 bytes, which leave no room for wider per-lane words.
template <typename S, typename T, int M, int INC>
__global__ void __launch_bounds__(128) ext_x_staged_kernel(Geom g, const S *__restrict__ a,
                                                           const S *__restrict__ b,
                                                           const S *__restrict__ c,
                                                           S *__restrict__ d, S *__restrict__ u) {
  using E = Elem<S, T>;
  constexpr int NA = INC ? 5 : 4;
  constexpr int SL = kWarp * (M + 1);  // slots per array
  extern __shared__ __align__(16) unsigned char xs_smem[];
  const int lane = threadIdx.x & (kWarp - 1);
  const int w = threadIdx.x / kWarp;
  const int64_t sys = (int64_t)blockIdx.x * (blockDim.x / kWarp) + w;
  if (sys >= g.nsys) return;  // uniform per warp
  int64_t off[5];
  system_offsets(g, sys, off);
  S *sm = reinterpret_cast<S *>(xs_smem) + (size_t)w * NA * SL;
  const S *src[5] = {a + off[kA], b + off[kB], c + off[kC], d + off[kD],
                     INC ? u + off[kU] : nullptr};
#pragma unroll
  for (int q = 0; q < NA; ++q)
#pragma unroll
    for (int k = 0; k < M; ++k) {
      const int i = k * kWarp + lane;
      cp_async_elem<(int)sizeof(S)>(sm + q * SL + i + i / M, src[q] + i);
    }
  cp_async_commit();
  cp_async_wait_all();
  __syncwarp();
  T al[M], be[M], ga[M], de[M], uo[INC ? M : 1];
  const int s0 = lane * (M + 1);
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const T va = E::cv(sm[s0 + j]), vc = E::cv(sm[2 * SL + s0 + j]);
    al[j] = (j == 0 && lane == 0) ? T(0) : va;
    be[j] = E::cv(sm[SL + s0 + j]);
    ga[j] = (j == M - 1 && lane == kWarp - 1) ? T(0) : vc;
    de[j] = E::cv(sm[3 * SL + s0 + j]);
    if constexpr (INC) uo[j] = E::cv(sm[4 * SL + s0 + j]);
  }
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  T xF, xL;
  warp_interface_solve(F, L, xF, xL, lane);
  chunk_backsub<T, M>(al, ga, de, xF, xL);
  // each lane overwrites only the slots it read itself
#pragma unroll
  for (int j = 0; j < M; ++j) E::st(sm + 3 * SL + s0 + j, INC ? uo[INC ? j : 0] + de[j] : de[j]);
  __syncwarp();
  S *dst = INC ? u + off[kU] : d + off[kD];
#pragma unroll
  for (int k = 0; k < M; ++k) {
    const int i = k * kWarp + lane;
    dst[i] = sm[3 * SL + i + i / M];
  }
}

template <typename S, typename T, int M, int SB, int INC>
__global__ void __launch_bounds__(SB * kWarp) ext_strided_kernel(Geom g, const S *__restrict__ a,
                                                                 const S *__restrict__ b,
                                                                 const S *__restrict__ c,
                                                                 S *__restrict__ d,
                                                                 S *__restrict__ u) {
  using E = Elem<S, T>;
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
      al[j] = (r == 0) ? T(0) : E::ld(a + off[kA] + r * sa);
      be[j] = E::ld(b + off[kB] + r * sb);
      ga[j] = (r == n - 1) ? T(0) : E::ld(c + off[kC] + r * sc);
      de[j] = E::ldw(d + off[kD] + r * sd);
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
    if (r < n)
      ext_out<S, T, INC>(d + off[kD] + r * sd, INC ? u + off[kU] + r * su : nullptr, de[j]);
  }
}

// Strided axes, persistent (one CTA per SM): tiles of SB adjacent systems x n
// rows of every array stream into shared memory by per-element cp.async
// (consecutive threads take consecutive systems of a row: coalesced), each
// thread copies its chunk rows into registers, the buffer is released and
// a later tile's copies are issued into it before the current tile is
// solved, so the copies overlap the arithmetic.  NBUF tile buffers: with
// two, two tiles' copies are in flight while one is solved (FP32 storage
// tiles are small, and one tile in flight per SM keeps too few bytes moving).
// CP >= 1: every tile is SB consecutive systems of one axis-0 row with
// 16-byte aligned rows (dims[0] a multiple of SB, row strides multiples of
// 16 bytes), so the copies move 16 bytes (16/sizeof(S) systems) each;
// CP == 2 adds n == 32*M (whole chunks): no row or system guards, and the
// copy loops have fixed trip counts.
template <typename S, typename T, int M, int SB, int INC, int CP, int NBUF>
__global__ void __launch_bounds__(SB * kWarp, 1) ext_stream_kernel(Geom g, const S *__restrict__ a,
                                                                   const S *__restrict__ b,
                                                                   const S *__restrict__ c,
                                                                   S *__restrict__ d,
                                                                   S *__restrict__ u,
                                                                   int64_t ntiles) {
  using E = Elem<S, T>;
  constexpr int NA = INC ? 5 : 4;
  constexpr bool VEC = CP >= 1;
  constexpr bool FULL = CP == 2;
  constexpr int NSET = NBUF + 1;  // offset sets: the tiles in flight and the one being solved
  extern __shared__ __align__(16) unsigned char ext_smem[];
  // per array, a tile's system offsets (-1: past the last system)
  __shared__ int64_t soff[NSET][NA][SB];
  const int n = FULL ? kWarp * M : g.n;
  const size_t tsz = (size_t)n * SB;  // [row][system] per array
  S *const tiles = reinterpret_cast<S *>(ext_smem);  // [NBUF][NA][tsz]
  T *red = reinterpret_cast<T *>(tiles + NBUF * NA * tsz);  // [8][32][SB+1]
  T *sol = red + 8 * kWarp * (SB + 1);                      // [2][32][SB+1]
  const S *src[5] = {a, b, c, d, u};
  const int tid = threadIdx.x;
  const int sl = tid % SB;
  const int t = tid / SB;
  auto offsets = [&](int64_t blk, int set) {
    if (tid < SB) {
      const int64_t s = blk * SB + tid;
      int64_t off[5] = {-1, -1, -1, -1, -1};
      if (s < g.nsys) system_offsets(g, s, off);
#pragma unroll
      for (int q = 0; q < NA; ++q) soff[set][q][tid] = s < g.nsys ? off[q] : -1;
    }
  };
  // copies of the tile whose offsets are in `set` into buffer `tb`; always
  // closes a commit group (possibly empty) so that the group count per loop
  // iteration stays fixed
  auto issue = [&](int tb, int set, bool any) {
    S *tile = tiles + (size_t)tb * NA * tsz;
    if (any) {
      if constexpr (VEC) {
        constexpr int V = 16 / (int)sizeof(S);  // systems per copy
        constexpr int PR = SB / V;              // copies per row
#pragma unroll
        for (int q = 0; q < NA; ++q) {
          const int64_t base = soff[set][q][0];
          const int64_t str = g.stride[q];
          for (int i = tid; i < n * PR; i += SB * kWarp) {
            const int r = i / PR, v = i % PR;
            cp_async_elem<16>(tile + q * tsz + (size_t)r * SB + v * V,
                              src[q] + base + r * str + v * V);
          }
        }
      } else {
#pragma unroll
        for (int q = 0; q < NA; ++q) {
          const int64_t base = soff[set][q][sl];
          if (base < 0) continue;
          const int64_t str = g.stride[q];
          for (int r = t; r < n; r += kWarp)
            cp_async_elem<(int)sizeof(S)>(tile + q * tsz + (size_t)r * SB + sl,
                                          src[q] + base + r * str);
        }
      }
    }
    cp_async_commit();
  };
  auto R = [&](int comp, int chunk, int s) -> T & {
    return red[((size_t)comp * kWarp + chunk) * (SB + 1) + s];
  };

  int64_t blk = blockIdx.x;
  if (blk >= ntiles) return;
  const int64_t G = gridDim.x;
#pragma unroll
  for (int k = 0; k < NBUF; ++k)
    if (blk + k * G < ntiles) offsets(blk + k * G, k);
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NBUF; ++k) issue(k, k, blk + k * G < ntiles);
  int tb = 0, set = 0;
  const int r0 = t * M;
  const int64_t so = INC ? g.stride[kU] : g.stride[kD];
  S *const out = INC ? u : d;
  for (; blk < ntiles; blk += G) {
    // the tile NBUF steps ahead takes this tile's buffer once it is read
    const int64_t ahead = blk + NBUF * G;
    const int aset = (set + NBUF) % NSET;
    if (ahead < ntiles) offsets(ahead, aset);
    // this tile's group is the oldest of the NBUF outstanding ones
    if constexpr (NBUF == 2)
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    else
      cp_async_wait_all();
    __syncthreads();  // every thread's copies of this tile have landed
    const S *tile = tiles + (size_t)tb * NA * tsz;
    const int64_t obase = soff[set][INC ? kU : kD][sl];
    const bool valid = FULL || obase >= 0;
    T al[M], be[M], ga[M], de[M], uo[INC ? M : 1];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int r = r0 + j;
      if constexpr (FULL) {
        const size_t o = (size_t)r * SB + sl;
        const T va = E::cv(tile[o]), vc = E::cv(tile[2 * tsz + o]);
        al[j] = (j == 0 && t == 0) ? T(0) : va;
        be[j] = E::cv(tile[tsz + o]);
        ga[j] = (j == M - 1 && t == kWarp - 1) ? T(0) : vc;
        de[j] = E::cv(tile[3 * tsz + o]);
        if constexpr (INC) uo[j] = E::cv(tile[4 * tsz + o]);
      } else {
        const bool in = valid && r < n;
        const size_t o = (size_t)(r < n ? r : n - 1) * SB + sl;
        al[j] = (in && r != 0) ? E::cv(tile[o]) : T(0);
        be[j] = in ? E::cv(tile[tsz + o]) : T(1);
        ga[j] = (in && r != n - 1) ? E::cv(tile[2 * tsz + o]) : T(0);
        de[j] = in ? E::cv(tile[3 * tsz + o]) : T(0);
        if constexpr (INC) uo[j] = in ? E::cv(tile[4 * tsz + o]) : T(0);
      }
    }
    __syncthreads();  // the buffer is free: a later tile streams into it meanwhile
    issue(tb, aset, ahead < ntiles);

    Row<T> F, L;
    chunk_reduce<T, M>(al, be, ga, de, F, L);
    R(0, t, sl) = F.a;
    R(1, t, sl) = F.b;
    R(2, t, sl) = F.c;
    R(3, t, sl) = F.d;
    R(4, t, sl) = L.a;
    R(5, t, sl) = L.b;
    R(6, t, sl) = L.c;
    R(7, t, sl) = L.d;
    __syncthreads();
    {
      const int w = tid / kWarp;
      const int lane = tid & (kWarp - 1);
      const Row<T> F2{R(0, lane, w), R(1, lane, w), R(2, lane, w), R(3, lane, w)};
      const Row<T> L2{R(4, lane, w), R(5, lane, w), R(6, lane, w), R(7, lane, w)};
      T xF, xL;
      warp_interface_solve(F2, L2, xF, xL, lane);
      sol[(0 * kWarp + lane) * (SB + 1) + w] = xF;
      sol[(1 * kWarp + lane) * (SB + 1) + w] = xL;
    }
    __syncthreads();
    chunk_backsub<T, M>(al, ga, de, sol[(0 * kWarp + t) * (SB + 1) + sl],
                        sol[(1 * kWarp + t) * (SB + 1) + sl]);
    if (valid) {
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const int r = r0 + j;
        if (FULL || r < n) E::st(out + obase + r * so, INC ? uo[INC ? j : 0] + de[j] : de[j]);
      }
    }
    tb = (tb + 1) % NBUF;
    set = (set + 1) % NSET;
  }
  cp_async_wait_all();  // empty groups only; nothing may be left in flight at exit
}

// Thomas in the reference's operation order (scalar/src/cpu/trid_cpu.cpp:
// 360-401); a[0] and c[n-1] are never read
template <typename S, typename T, int INC>
__global__ void __launch_bounds__(128) ext_thomas_kernel(Geom g, const S *__restrict__ a,
                                                         const S *__restrict__ b,
                                                         const S *__restrict__ c,
                                                         S *__restrict__ d, S *__restrict__ u,
                                                         T *__restrict__ work, int64_t s0,
                                                         int64_t ns) {
  using E = Elem<S, T>;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  int64_t off[5];
  system_offsets(g, s0 + k, off);
  const int64_t sa = g.stride[kA], sb = g.stride[kB], sc = g.stride[kC], sd = g.stride[kD],
                su = g.stride[kU];
  const int n = g.n;
  T *c2 = work + k;
  T *d2 = work + (int64_t)n * ns + k;
  const S *ap = a + off[kA];
  const S *bp = b + off[kB];
  const S *cp = c + off[kC];
  S *dp = d + off[kD];
  S *up = INC ? u + off[kU] : nullptr;

  T bb = rcp(E::ld(bp));
  T cc = (n > 1) ? bb * E::ld(cp) : T(0);
  T dd = bb * E::ldw(dp);
  c2[0] = cc;
  d2[0] = dd;
  for (int i = 1; i < n; ++i) {
    const T aa = E::ld(ap + i * sa);
    bb = E::ld(bp + i * sb) - aa * cc;
    dd = E::ldw(dp + i * sd) - aa * dd;
    bb = rcp(bb);
    cc = (i < n - 1) ? bb * E::ld(cp + i * sc) : T(0);
    dd = bb * dd;
    c2[(int64_t)i * ns] = cc;
    d2[(int64_t)i * ns] = dd;
  }
  ext_out<S, T, INC>(dp + (int64_t)(n - 1) * sd, INC ? up + (int64_t)(n - 1) * su : nullptr, dd);
  for (int i = n - 2; i >= 0; --i) {
    dd = d2[(int64_t)i * ns] - c2[(int64_t)i * ns] * dd;
    ext_out<S, T, INC>(dp + (int64_t)i * sd, INC ? up + (int64_t)i * su : nullptr, dd);
  }
}

// ------------------------------------------------------------ launchers --
// Largest chunk (rows per lane) of the partitioned kernels: 16 for 8-byte
// arithmetic, 8 for complex<double> (16 rows of 16 bytes per array exceed the
// register file at one CTA per SM).
// dynamic shared memory of the streamed kernel: tiles plus interface rows
constexpr size_t kExtStreamSmem = 220 * 1024;

template <typename T>
constexpr int ext_max_chunk() {
  return sizeof(T) >= 16 ? 8 : 16;
}

template <typename S, typename T, int INC>
cudaError_t launch_ext(const Geom &g, int solvedim, const S *a, const S *b, const S *c, S *d,
                       S *u, cudaStream_t st) {
  int M = 2;
  while (32 * M < g.n && M < ext_max_chunk<T>()) M *= 2;
  if (32 * M >= g.n) {
    if (solvedim == 0) {
      const int64_t blocks = (g.nsys + 3) / 4;
      if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
      const dim3 grid((unsigned)blocks), block(128);
      // 16-byte words per lane: whole systems, rows of every array used
      // 16-byte aligned in every system (bases and outer strides), elements
      // of at most 8 bytes
      bool vec = sizeof(S) <= 8 && g.n == kWarp * M && (M * sizeof(S)) % 16 == 0;
      const void *ptrs[5] = {a, b, c, d, u};
      for (int q = 0; q < (INC ? 5 : 4) && vec; ++q) {
        vec = ((uintptr_t)ptrs[q] & 15) == 0;
        for (int k = 0; k < g.nod && vec; ++k) vec = (g.ocum[q][k] * (int64_t)sizeof(S)) % 16 == 0;
      }
      auto go = [&](auto kern) {
        kern<<<grid, block, 0, st>>>(g, a, b, c, d, u);
        return cudaGetLastError();
      };
      // whole systems of 16-byte elements: staged through shared memory
      // (for narrower elements the 16-byte words per lane measured faster:
      // 256^3 axis 0, FP32 storage 4.81 against 4.41 TB/s, complex<float>
      // 5.65 against 4.19)
      if constexpr (sizeof(S) == 16) {
        auto go_staged = [&](auto kern) {
          const size_t smem = (size_t)4 * (INC ? 5 : 4) * kWarp * (M + 1) * sizeof(S);
          cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
          if (e != cudaSuccess) return e;
          kern<<<grid, block, smem, st>>>(g, a, b, c, d, u);
          return cudaGetLastError();
        };
        if (g.n == kWarp * M) {
          switch (M) {
            case 2: return go_staged(ext_x_staged_kernel<S, T, 2, INC>);
            case 4: return go_staged(ext_x_staged_kernel<S, T, 4, INC>);
            default: return go_staged(ext_x_staged_kernel<S, T, 8, INC>);
          }
        }
      }
      switch (M) {
        case 2:
          if constexpr (sizeof(S) == 8) if (vec) return go(ext_x_kernel<S, T, 2, INC, true>);
          return go(ext_x_kernel<S, T, 2, INC, false>);
        case 4:
          if constexpr (sizeof(S) <= 8) if (vec) return go(ext_x_kernel<S, T, 4, INC, true>);
          return go(ext_x_kernel<S, T, 4, INC, false>);
        case 8:
          if constexpr (sizeof(S) <= 8) if (vec) return go(ext_x_kernel<S, T, 8, INC, true>);
          return go(ext_x_kernel<S, T, 8, INC, false>);
        default:
          if constexpr (ext_max_chunk<T>() >= 16) {
            if constexpr (sizeof(S) <= 8) if (vec) return go(ext_x_kernel<S, T, 16, INC, true>);
            return go(ext_x_kernel<S, T, 16, INC, false>);
          }
          return cudaErrorInvalidValue;
      }
    }
    // SB systems per CTA: 8 for 16-byte T and for 16-row chunks (whose 64
    // register-resident values per thread need 256-thread CTAs), else 16
    constexpr int SB = sizeof(T) >= 16 ? 8 : 16;
    if (M <= 8) {
      // streamed tiles, one CTA per SM; two tile buffers when they fit
      constexpr int NA = INC ? 5 : 4;
      const size_t tile_bytes = (size_t)NA * g.n * SB * sizeof(S);
      const size_t red_bytes = (size_t)10 * kWarp * (SB + 1) * sizeof(T);
      const bool two = 2 * tile_bytes + red_bytes <= kExtStreamSmem;
      const size_t smem = (two ? 2 : 1) * tile_bytes + red_bytes;
      int dev = 0, sms = 0;
      if (smem <= kExtStreamSmem && cudaGetDevice(&dev) == cudaSuccess &&
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess) {
        const int64_t ntiles = (g.nsys + SB - 1) / SB;
        const unsigned grid = (unsigned)(ntiles < sms ? ntiles : sms);
        auto go = [&](auto kern) {
          cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
          if (e != cudaSuccess) return e;
          kern<<<dim3(grid), dim3(SB * kWarp), smem, st>>>(g, a, b, c, d, u, ntiles);
          return cudaGetLastError();
        };
        // 16-byte copies: whole tiles in one row, 16-byte aligned bases and
        // row strides (always so for 16-byte elements, whose copies are one
        // element either way; the mode also admits the guard-free variant)
        bool vec = g.odims[0] % SB == 0;
        const void *ptrs[5] = {a, b, c, d, u};
        constexpr int64_t kV = 16 / (int64_t)sizeof(S);
        for (int q = 0; q < NA && vec; ++q) {
          vec = ((uintptr_t)ptrs[q] & 15) == 0 && g.stride[q] % kV == 0;
          for (int k = 1; k < g.nod && vec; ++k) vec = g.ocum[q][k] % kV == 0;
        }
        auto pick = [&](auto cp_tag, auto nbuf_tag) {
          constexpr int CP = decltype(cp_tag)::value;
          constexpr int NB = decltype(nbuf_tag)::value;
          switch (M) {
            case 2: return go(ext_stream_kernel<S, T, 2, SB, INC, CP, NB>);
            case 4: return go(ext_stream_kernel<S, T, 4, SB, INC, CP, NB>);
            default: return go(ext_stream_kernel<S, T, 8, SB, INC, CP, NB>);
          }
        };
        using C2 = std::integral_constant<int, 2>;
        using C1 = std::integral_constant<int, 1>;
        using C0 = std::integral_constant<int, 0>;
        using B2 = std::integral_constant<int, 2>;
        using B1 = std::integral_constant<int, 1>;
        if (vec && g.n == kWarp * M) return two ? pick(C2{}, B2{}) : pick(C2{}, B1{});
        if (vec) return two ? pick(C1{}, B2{}) : pick(C1{}, B1{});
        return two ? pick(C0{}, B2{}) : pick(C0{}, B1{});
      }
    }
    auto go = [&](auto kern, int sb) {
      const int64_t blocks = (g.nsys + sb - 1) / sb;
      if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
      kern<<<dim3((unsigned)blocks), dim3(sb * kWarp), 0, st>>>(g, a, b, c, d, u);
      return cudaGetLastError();
    };
    switch (M) {
      case 2: return go(ext_strided_kernel<S, T, 2, SB, INC>, SB);
      case 4: return go(ext_strided_kernel<S, T, 4, SB, INC>, SB);
      case 8: return go(ext_strided_kernel<S, T, 8, SB, INC>, SB);
      default:
        if constexpr (ext_max_chunk<T>() >= 16) return go(ext_strided_kernel<S, T, 16, 8, INC>, 8);
        return cudaErrorInvalidValue;
    }
  }
  // Thomas with c'/d' in scratch, in batches of systems bounded to ~1 GiB
  const size_t per_sys = (size_t)2 * g.n * sizeof(T);
  int64_t ws = (int64_t)(((size_t)1 << 30) / per_sys);
  ws = ws < 1 ? 1 : (ws > g.nsys ? g.nsys : ws);
  const Scratch sc(per_sys * (size_t)ws, 0, st);
  T *work = (T *)sc.get();
  if (!work) return cudaErrorMemoryAllocation;
  for (int64_t s0 = 0; s0 < g.nsys; s0 += ws) {
    const int64_t ns = (g.nsys - s0 < ws) ? (g.nsys - s0) : ws;
    ext_thomas_kernel<S, T, INC><<<dim3((unsigned)((ns + 127) / 128)), dim3(128), 0, st>>>(
        g, a, b, c, d, u, work, s0, ns);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

tridStatus_t make_geom(int ndim, int solvedim, const int *dims, const int *const pads[5],
                       bool inc, Geom &g);

template <typename S, typename T, int INC>
static tridStatus_t solve_ext(const void *a, const void *b, const void *c, void *d, void *u,
                              int ndim, int solvedim, const int *dims, const int *pads) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  Geom g;
  const tridStatus_t st = make_geom(ndim, solvedim, dims, p, INC != 0, g);
  if (st != TRID_STATUS_SUCCESS) return st;
  auto ok = [](const void *q) { return q != nullptr && ((uintptr_t)q % sizeof(S)) == 0; };
  if (!ok(a) || !ok(b) || !ok(c) || !ok(d) || (INC && !ok(u))) return TRID_STATUS_INVALID_VALUE;
  if (g.n == 0 || g.nsys == 0) return TRID_STATUS_SUCCESS;
  const cudaError_t e = launch_ext<S, T, INC>(g, solvedim, (const S *)a, (const S *)b,
                                             (const S *)c, (S *)d, INC ? (S *)u : nullptr,
                                             current_stream());
  if (e == cudaErrorMemoryAllocation) return TRID_STATUS_ALLOC_FAILED;
  return e == cudaSuccess ? TRID_STATUS_SUCCESS : TRID_STATUS_EXECUTION_FAILED;
}

}  // namespace tridb200

using namespace tridb200;

#define TRID_EXT_ABI(NAME, ST, S, T, INC)                                                    \
  extern "C" tridStatus_t NAME(const ST *a, const ST *b, const ST *c, ST *d, ST *u, int ndim, \
                               int solvedim, int *dims, int *pads) {                          \
    return solve_ext<S, T, INC>(a, b, c, d, u, ndim, solvedim, dims, pads);                   \
  }
TRID_EXT_ABI(tridCmtsvStridedBatch, tridComplexF, float2, Cx<float>, 0)
TRID_EXT_ABI(tridCmtsvStridedBatchInc, tridComplexF, float2, Cx<float>, 1)
TRID_EXT_ABI(tridZmtsvStridedBatch, tridComplexD, double2, Cx<double>, 0)
TRID_EXT_ABI(tridZmtsvStridedBatchInc, tridComplexD, double2, Cx<double>, 1)
TRID_EXT_ABI(tridSmtsvStridedBatchMixed, float, float, double, 0)
TRID_EXT_ABI(tridSmtsvStridedBatchMixedInc, float, float, double, 1)
