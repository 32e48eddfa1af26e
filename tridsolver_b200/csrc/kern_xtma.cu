// Axis-0 solve with TMA-staged tiles (sm_100a).
//
// One warp per system, as xsolve_kernel, but the system's a, b, c, d (and u)
// arrive in shared memory by one bulk tensor copy each (cp.async.bulk.tensor,
// 128-byte swizzle, completion on an mbarrier) instead of 32 strided loads per
// lane.  The array is viewed as a 2-D tensor of 128-byte rows; with the
// 128-byte swizzle the 16-byte unit u of row r sits at unit u ^ (r % 8), so
// lane l reading its M consecutive elements hits 8 distinct bank groups per
// quarter-warp: conflict-free.  When the system length is a multiple of the
// row length the solution goes back the same way (bulk tensor store from the
// swizzled tile), otherwise with plain stores.
//
// Preconditions (checked by launch_xsolve_tma, which returns
// cudaErrorNotSupported otherwise): pads[0] of every array a multiple of the
// row length (16 doubles / 32 floats), 16-byte aligned base pointers,
// n <= 32*M.
#include "partition.cuh"
#include "tma.cuh"

namespace tridb200 {

template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
};
template <>
struct Vec16<float> {
  using type = float4;
};

template <typename T>
__device__ __forceinline__ int swz(int byte) {
  const int row = byte >> 7;
  return (row << 7) | ((((byte >> 4) & 7) ^ (row & 7)) << 4) | (byte & 15);
}

// load M consecutive elements starting at element e0 of a swizzled tile
template <typename T, int M>
__device__ __forceinline__ void tile_read(const unsigned char *tile, int e0, T (&v)[M]) {
  constexpr int kPer16 = 16 / (int)sizeof(T);
  if constexpr (M % kPer16 == 0) {
    using V = typename Vec16<T>::type;
#pragma unroll
    for (int j = 0; j < M; j += kPer16) {
      const V w = *reinterpret_cast<const V *>(tile + swz<T>((e0 + j) * (int)sizeof(T)));
      if constexpr (sizeof(T) == 8) {
        v[j] = w.x;
        v[j + 1] = w.y;
      } else {
        v[j] = w.x;
        v[j + 1] = w.y;
        v[j + 2] = w.z;
        v[j + 3] = w.w;
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < M; ++j)
      v[j] = *reinterpret_cast<const T *>(tile + swz<T>((e0 + j) * (int)sizeof(T)));
  }
}

template <typename T, int M>
__device__ __forceinline__ void tile_write(unsigned char *tile, int e0, const T (&v)[M]) {
#pragma unroll
  for (int j = 0; j < M; ++j) *reinterpret_cast<T *>(tile + swz<T>((e0 + j) * (int)sizeof(T))) = v[j];
}

constexpr int kXWarps = 4;  // systems (warps) per CTA

template <typename T, int M>
struct XTile {
  static constexpr int kRowElems = 128 / (int)sizeof(T);
  static constexpr int kRows = (32 * M + kRowElems - 1) / kRowElems;
  static constexpr int kBytes = ((kRows * 128 + 1023) / 1024) * 1024;  // swizzle atom: 1 KB
};

template <typename T, int M, int INC, bool TSTORE>
__global__ void __launch_bounds__(kXWarps * kWarp) xsolve_tma_kernel(
    const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb,
    const __grid_constant__ CUtensorMap mc, const __grid_constant__ CUtensorMap md,
    const __grid_constant__ CUtensorMap mu, Geom g, int rows, T *__restrict__ d,
    T *__restrict__ u, unsigned *err) {
  pdl_enter();
  using Tile = XTile<T, M>;
  constexpr int NA = INC ? 5 : 4;
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t bars[kXWarps];
  // the 128-byte swizzle repeats every 1 KB: align the tiles to 1 KB
  unsigned char *smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);

  const int w = threadIdx.x / kWarp;
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t sys = (int64_t)blockIdx.x * kXWarps + w;
  if (sys >= g.nsys) return;  // whole warp
  if (!tma_smem_aligned(smem)) {
    if (lane == 0) atomicOr(err, kErrMisaligned);
    return;
  }
  int64_t off[5];
  system_offsets(g, sys, off);
  unsigned char *tile = smem + (size_t)w * NA * Tile::kBytes;
  uint64_t *bar = &bars[w];
  constexpr int RE = Tile::kRowElems;

  if (lane == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncwarp();
  if (lane == 0) {
    mbar_arrive_expect_tx(bar, (uint32_t)(NA * rows * 128));
    tma_load_2d(tile + 0 * Tile::kBytes, &ma, bar, 0, (int)(off[kA] / RE));
    tma_load_2d(tile + 1 * Tile::kBytes, &mb, bar, 0, (int)(off[kB] / RE));
    tma_load_2d(tile + 2 * Tile::kBytes, &mc, bar, 0, (int)(off[kC] / RE));
    tma_load_2d(tile + 3 * Tile::kBytes, &md, bar, 0, (int)(off[kD] / RE));
    if (INC) tma_load_2d(tile + 4 * Tile::kBytes, &mu, bar, 0, (int)(off[kU] / RE));
  }
  if (!mbar_wait(bar, 0, err)) {
    mbar_wait(bar, 0, nullptr);  // give copies in flight a second bounded chance
    return;
  }

  const int n = g.n;
  const int r0 = lane * M;
  T al[M], be[M], ga[M], de[M];
  tile_read<T, M>(tile + 0 * Tile::kBytes, r0, al);
  tile_read<T, M>(tile + 1 * Tile::kBytes, r0, be);
  tile_read<T, M>(tile + 2 * Tile::kBytes, r0, ga);
  tile_read<T, M>(tile + 3 * Tile::kBytes, r0, de);
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = r0 + j;
    if (r == 0) al[j] = T(0);
    if (r >= n - 1) ga[j] = T(0);
    if (r >= n) {
      al[j] = T(0);
      be[j] = T(1);
      de[j] = T(0);
    }
  }
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  T xF, xL;
  warp_interface_solve(F, L, xF, xL, lane);
  chunk_backsub<T, M>(al, ga, de, xF, xL);

  if constexpr (TSTORE) {
    // n is a whole number of rows: write the tile back with one bulk store
    unsigned char *out = tile + (INC ? 4 : 3) * Tile::kBytes;
    if (INC) {
      T uu[M];
      tile_read<T, M>(out, r0, uu);
#pragma unroll
      for (int j = 0; j < M; ++j) de[j] += uu[j];
    }
    if (r0 < n) tile_write<T, M>(out, r0, de);
    fence_proxy_async();
    __syncwarp();
    if (lane == 0) {
      tma_store_2d(INC ? &mu : &md, out, 0, (int)(off[INC ? kU : kD] / RE));
      tma_store_commit();
      tma_store_wait_read();
    }
    __syncwarp();
  } else {
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
}

template <typename T, int M, int INC>
static cudaError_t launch_xtma_m(const CUtensorMap *maps, const Geom &g, int rows, bool tstore,
                                 T *d, T *u, unsigned *err, cudaStream_t st) {
  using Tile = XTile<T, M>;
  const int NA = INC ? 5 : 4;
  const size_t smem = (size_t)kXWarps * NA * Tile::kBytes + 1024;
  const int64_t blocks = (g.nsys + kXWarps - 1) / kXWarps;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  auto go = [&](auto kern) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    return launch_pdl(kern, dim3((unsigned)blocks), dim3(kXWarps * kWarp), smem, st, maps[0],
                      maps[1], maps[2], maps[3], maps[4], g, rows, d, u, err);
  };
  if (tstore) return go(xsolve_tma_kernel<T, M, INC, true>);
  return go(xsolve_tma_kernel<T, M, INC, false>);
}

template <typename T, int INC>
cudaError_t launch_xsolve_tma(const Geom &g, const int *const pads[5], int ndim, const T *a,
                              const T *b, const T *c, T *d, T *u, int chunk, unsigned *err,
                              cudaStream_t st) {
  constexpr int RE = 128 / (int)sizeof(T);
  const void *ptrs[5] = {a, b, c, d, u};
  const int na = INC ? 5 : 4;
  const int rows = (g.n + RE - 1) / RE;
  if (rows > 256 || g.n > 32 * chunk) return cudaErrorNotSupported;
  CUtensorMap maps[5];
  for (int q = 0; q < 5; ++q) {
    const int qq = q < na ? q : 3;  // unused u map: any valid map
    if (((uintptr_t)ptrs[qq] & 15) != 0 || pads[qq][0] % RE != 0) return cudaErrorNotSupported;
    uint64_t total = 1;
    for (int k = 0; k < ndim; ++k) total *= (uint64_t)pads[qq][k];
    const uint64_t dims[2] = {(uint64_t)RE, total / RE};
    const uint64_t strides[1] = {128};
    const uint32_t box[2] = {(uint32_t)RE, (uint32_t)rows};
    if (dims[1] == 0 || dims[1] > 0xffffffffull) return cudaErrorNotSupported;
    if (!encode_tensor_map(&maps[q], ptrs[qq], (int)sizeof(T), 2, dims, strides, box, true))
      return cudaErrorNotSupported;
  }
  const bool tstore = (g.n % RE) == 0;
  switch (chunk) {
    case 2: return launch_xtma_m<T, 2, INC>(maps, g, rows, tstore, d, u, err, st);
    case 4: return launch_xtma_m<T, 4, INC>(maps, g, rows, tstore, d, u, err, st);
    case 8: return launch_xtma_m<T, 8, INC>(maps, g, rows, tstore, d, u, err, st);
    case 16: return launch_xtma_m<T, 16, INC>(maps, g, rows, tstore, d, u, err, st);
    default: return cudaErrorNotSupported;
  }
}

#define TRID_XTMA_INSTANTIATE(T, INC)                                                         \
  template cudaError_t launch_xsolve_tma<T, INC>(const Geom &, const int *const[5], int,        \
                                                 const T *, const T *, const T *, T *, T *, int, \
                                                 unsigned *, cudaStream_t);
TRID_XTMA_INSTANTIATE(float, 0)
TRID_XTMA_INSTANTIATE(float, 1)
TRID_XTMA_INSTANTIATE(double, 0)
TRID_XTMA_INSTANTIATE(double, 1)

}  // namespace tridb200
