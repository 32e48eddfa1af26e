// Strided-axis partitioned Thomas with TMA-staged tiles (sm_100a).
//
// Same algorithm and thread mapping as strided_kernel (kern_scalar.cu): a CTA
// owns SB adjacent systems, thread (system sl, chunk t) reduces rows
// [t*M, t*M+M) of system sl, SB warps solve the interface systems (lane =
// chunk), every thread back-substitutes its chunk.  The difference is data
// movement: the CTA's whole tile (SB systems x n rows of a, b, c, d and, for
// Inc, u) arrives by bulk tensor copies into shared memory (one or two boxes
// per array, completion on one mbarrier) and the solution leaves by bulk
// tensor stores, so every byte of the tile is in flight at once without
// occupying registers, and the loads of one CTA overlap the arithmetic of
// the others on the SM.  The tensor maps use the logical extents, so rows
// past n and systems past dims[0] are never written.
//
// Preconditions (launch_strided_part_tma returns cudaErrorNotSupported
// otherwise): solvedim >= 1, ndim <= 5, 16-byte aligned base pointers,
// pads[0]*sizeof(T) a multiple of 16 for every array, dims[0] >= SB,
// n <= 32*M and the tile fitting in shared memory.
#include <algorithm>

#include "partition.cuh"
#include "tma.cuh"

namespace tridb200 {

// Rows [r0, r0+M) of tile system sl from the staged tile ([array][row][SB]).
// Every shared-memory read is unconditional (row index clamped into the
// tile), and rows past n or systems past the axis become identity rows by
// selects afterwards, so the M*4 reads issue back to back instead of one
// guarded read at a time.
template <typename T, int M, int SB, int INC>
__device__ __forceinline__ void load_rows(const T *tile, size_t tsz, int r0, int sl, int n,
                                          int rows_cap, bool valid, T (&al)[M], T (&be)[M],
                                          T (&ga)[M], T (&de)[M], T (&uo)[INC ? M : 1]) {
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = r0 + j;
    const size_t o = (size_t)(r < rows_cap ? r : rows_cap - 1) * SB + sl;
    const T va = tile[o], vb = tile[tsz + o], vc = tile[2 * tsz + o], vd = tile[3 * tsz + o];
    const bool in = valid && r < n;
    al[j] = (in && r != 0) ? va : T(0);
    be[j] = in ? vb : T(1);
    ga[j] = (in && r != n - 1) ? vc : T(0);
    de[j] = in ? vd : T(0);
    if constexpr (INC) uo[j] = in ? tile[4 * tsz + o] : T(0);
  }
}

template <typename T, int M, int SB, int INC>
__global__ void __launch_bounds__(SB * kWarp) strided_part_tma_kernel(
    const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb,
    const __grid_constant__ CUtensorMap mc, const __grid_constant__ CUtensorMap md,
    const __grid_constant__ CUtensorMap mu, Geom g, int solvedim, int box_rows, int nbox,
    int red_off, int prefetch_dist, unsigned *err) {
  pdl_enter();
  constexpr int NA = INC ? 5 : 4;
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t bar;
  const int rows_cap = box_rows * nbox;                       // tile rows in smem
  // [NA][tsz]: each array tile starts on a 128-byte boundary
  T *tile = reinterpret_cast<T *>(smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127));
  constexpr int kAlignElems = 128 / (int)sizeof(T);
  const size_t tsz = (((size_t)rows_cap * SB + kAlignElems - 1) / kAlignElems) * kAlignElems;
  // interface rows / solutions alias the a, b, c tiles once they are consumed
  // (red_off = 0), or follow the tiles when those are too small
  T *red = tile + red_off;                                    // [8][32][SB+1]
  T *sol = red + 8 * kWarp * (SB + 1);                        // [2][32][SB+1]

  const int tid = threadIdx.x;
  const int sl = tid % SB;
  const int t = tid / SB;
  const int n = g.n;

  // tile -> coordinates (x0 on axis 0, the other non-solve axes)
  auto tile_coords = [&](uint32_t blk, int (&cc)[5]) {
    const int ntx = (g.odims[0] + SB - 1) / SB;
    cc[0] = (int)(blk % ntx) * SB;
    cc[1] = cc[2] = cc[3] = cc[4] = 0;
    uint32_t rest = blk / ntx;
    int o = 1;
    for (int k = 1; k < 5; ++k) {
      if (k == solvedim || o >= g.nod) continue;
      const uint32_t e = (uint32_t)g.odims[o++];
      cc[k] = (int)(rest % e);
      rest /= e;
    }
  };
  int coord[5];
  tile_coords(blockIdx.x, coord);
  const CUtensorMap *maps[5] = {&ma, &mb, &mc, &md, &mu};
  // every copy destination (tile starts, second boxes) must be 128-byte aligned
  if (!tma_smem_aligned(tile) || (nbox > 1 && ((size_t)box_rows * SB * sizeof(T)) % 128 != 0)) {
    if (tid == 0) atomicOr(err, kErrMisaligned);
    return;
  }

  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (tid == 0) {
    mbar_arrive_expect_tx(&bar, (uint32_t)(NA * nbox * box_rows * SB * sizeof(T)));
    for (int q = 0; q < NA; ++q)
      for (int bx = 0; bx < nbox; ++bx) {
        int c[5] = {coord[0], coord[1], coord[2], coord[3], coord[4]};
        c[solvedim] = bx * box_rows;
        tma_load_5d(tile + q * tsz + (size_t)bx * box_rows * SB, maps[q], &bar, c[0], c[1], c[2],
                    c[3], c[4]);
      }
    // warm L2 with the tile this CTA's successor on the SM will load: keeps
    // more bytes in flight than the resident tiles alone
    const uint32_t nb = blockIdx.x + (uint32_t)prefetch_dist;
    if (prefetch_dist > 0 && nb < gridDim.x) {
      int pc[5];
      tile_coords(nb, pc);
      for (int q = 0; q < NA; ++q)
        for (int bx = 0; bx < nbox; ++bx) {
          int c[5] = {pc[0], pc[1], pc[2], pc[3], pc[4]};
          c[solvedim] = bx * box_rows;
          tma_prefetch_5d(maps[q], c[0], c[1], c[2], c[3], c[4]);
        }
    }
  }
  if (!mbar_wait(&bar, 0, err)) {
    mbar_wait(&bar, 0, nullptr);
    return;
  }

  const int r0 = t * M;
  const bool valid = coord[0] + sl < g.odims[0];
  T al[M], be[M], ga[M], de[M];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = r0 + j;
    if (valid && r < n) {
      const size_t o = (size_t)r * SB + sl;
      al[j] = (r == 0) ? T(0) : tile[0 * tsz + o];
      be[j] = tile[1 * tsz + o];
      ga[j] = (r == n - 1) ? T(0) : tile[2 * tsz + o];
      de[j] = tile[3 * tsz + o];
    } else {
      al[j] = T(0);
      be[j] = T(1);
      ga[j] = T(0);
      de[j] = T(0);
    }
  }
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  __syncthreads();  // every thread holds its rows: the a/b/c tiles become scratch
  auto R = [&](int comp, int chunk, int s) -> T & {
    return red[((size_t)comp * kWarp + chunk) * (SB + 1) + s];
  };
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

  // solution into the d (or u) tile, then bulk tensor stores
  T *out = tile + (INC ? 4 : 3) * tsz;
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int r = r0 + j;
    if (r < rows_cap) {
      const size_t o = (size_t)r * SB + sl;
      if (INC)
        out[o] += de[j];
      else
        out[o] = de[j];
    }
  }
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    for (int bx = 0; bx < nbox; ++bx) {
      int c[5] = {coord[0], coord[1], coord[2], coord[3], coord[4]};
      c[solvedim] = bx * box_rows;
      const T *src = out + (size_t)bx * box_rows * SB;
      asm volatile(
          "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5, %6}],"
          " [%1];" ::"l"(maps[INC ? 4 : 3]),
          "r"(smem_u32(src)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4])
          : "memory");
    }
    tma_store_commit();
    tma_store_wait_read();
  }
}

// Persistent form for wide tiles (SB * sizeof(T) >= 128: one 128-byte line
// per row and array).  On large row strides (planes of 64 KiB and more) DRAM
// serves 64-byte row segments at about 60% of the rate of 128-byte ones, so
// the tile must be a full line wide; such a tile (128 KB for FP64 at n = 256)
// leaves room for one CTA per SM, and without overlap the SM's loads would
// stop while it computes.  So the CTA loops over tiles with one buffer: it
// copies the tile from shared memory into registers, releases the buffer,
// issues the next tile's bulk tensor loads, and solves and stores (plain
// coalesced stores of full lines) while those loads are in flight.
template <typename T, int M, int SB, int NCH, int INC, bool FULL>
__global__ void __launch_bounds__(SB * NCH, 1) strided_stream_kernel(
    const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb,
    const __grid_constant__ CUtensorMap mc, const __grid_constant__ CUtensorMap md,
    const __grid_constant__ CUtensorMap mu, Geom g, int solvedim, int box_rows, int nbox,
    uint32_t ntiles, uint32_t ntx_mul, uint32_t ntx_shift, T *__restrict__ d,
    T *__restrict__ u, unsigned *err) {
  pdl_enter();
  // NCH chunks of M rows per system (32, or 16 for short systems: a warp
  // then solves the interface systems of two tile systems side by side);
  // FULL: n == NCH*M and dims[0] a multiple of SB (no row or system guards)
  constexpr int NA = INC ? 5 : 4;
  constexpr int kSysPerWarp = kWarp / NCH;
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t bar;
  T *tile = reinterpret_cast<T *>(smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127));
  constexpr int kAlignElems = 128 / (int)sizeof(T);
  const size_t tsz = FULL ? (size_t)NCH * M * SB
                          : (((size_t)box_rows * nbox * SB + kAlignElems - 1) / kAlignElems) *
                                kAlignElems;
  T *red = tile + NA * tsz;                                   // [8][NCH][SB+1]
  T *sol = red + 8 * NCH * (SB + 1);                          // [2][NCH][SB+1]
  const int rows_cap = FULL ? NCH * M : box_rows * nbox;

  const int tid = threadIdx.x;
  const int sl = tid % SB;
  const int t = tid / SB;
  const int n = FULL ? NCH * M : g.n;
  const uint32_t ntx = (uint32_t)(g.odims[0] + SB - 1) / SB;
  // tile -> coordinates (x0 on axis 0, then the other non-solve axes) and the
  // tile's index along the flattened outer axes; multiply-high divisions
  auto tile_coords = [&](uint32_t blk, int (&cc)[5]) -> uint32_t {
    const uint32_t outer = fastdiv(blk, ntx_mul, ntx_shift);
    cc[0] = (int)(blk - outer * ntx) * SB;
    cc[1] = cc[2] = cc[3] = cc[4] = 0;
    uint32_t rest = outer;
    int o = 1;
    for (int k = 1; k < 5; ++k) {
      if (k == solvedim || o >= g.nod) continue;
      const uint32_t q = fastdiv(rest, g.dmul[o], g.dshift[o]);
      cc[k] = (int)(rest - q * (uint32_t)g.odims[o]);
      rest = q;
      ++o;
    }
    return outer;
  };
  const CUtensorMap *maps[5] = {&ma, &mb, &mc, &md, &mu};
  if (!tma_smem_aligned(tile) || (nbox > 1 && ((size_t)box_rows * SB * sizeof(T)) % 128 != 0)) {
    if (tid == 0) atomicOr(err, kErrMisaligned);
    return;
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const uint32_t tx_bytes = (uint32_t)(NA * nbox * box_rows * SB * sizeof(T));
  auto issue = [&](const int (&cc)[5]) {
    mbar_arrive_expect_tx(&bar, tx_bytes);
    for (int q = 0; q < NA; ++q)
      for (int bx = 0; bx < nbox; ++bx) {
        int c[5] = {cc[0], cc[1], cc[2], cc[3], cc[4]};
        c[solvedim] = bx * box_rows;
        tma_load_5d(tile + q * tsz + (size_t)bx * box_rows * SB, maps[q], &bar, c[0], c[1], c[2],
                    c[3], c[4]);
      }
  };
  uint32_t blk = blockIdx.x;
  if (tid == 0 && blk < ntiles) {
    int cc[5];
    tile_coords(blk, cc);
    issue(cc);
  }
  uint32_t parity = 0;
  const int r0 = t * M;
  const int64_t so = INC ? g.stride[kU] : g.stride[kD];
  T *const out = INC ? u : d;
  auto R = [&](int comp, int chunk, int s) -> T & {
    return red[((size_t)comp * NCH + chunk) * (SB + 1) + s];
  };
  for (; blk < ntiles; blk += gridDim.x) {
    // index work that does not need the tile, done while its copy lands: this
    // system's output offset and, for the issuing thread, the next tile
    int cc[5];
    const uint32_t outer = tile_coords(blk, cc);
    const bool valid = FULL || cc[0] + sl < g.odims[0];
    int64_t obase = 0;
    if (valid) {
      int64_t off[5];
      system_offsets(g, (int64_t)cc[0] + sl + (int64_t)g.odims[0] * outer, off);
      obase = off[INC ? kU : kD];
    }
    const bool more = blk + gridDim.x < ntiles;
    int cn[5];
    if (tid == 0 && more) tile_coords(blk + gridDim.x, cn);

    const bool got = mbar_wait(&bar, parity, err);
    T al[M], be[M], ga[M], de[M], uo[INC ? M : 1];
    load_rows<T, M, SB, INC>(tile, tsz, r0, sl, n, rows_cap, valid, al, be, ga, de, uo);
    // this thread's reads of the buffer come before the next tile's copies
    fence_proxy_async();
    if (!__syncthreads_and(got)) {
      // a copy that never completed: let it land (bounded) before leaving
      if (tid == 0) mbar_wait(&bar, parity, nullptr);
      return;
    }
    parity ^= 1;
    if (tid == 0 && more) issue(cn);

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
      const int lane = tid & (kWarp - 1);
      // this lane's system and chunk
      const int sw = (NCH == kWarp) ? tid / kWarp : (tid / kWarp) * kSysPerWarp + lane / NCH;
      const int ch = (NCH == kWarp) ? lane : lane & (NCH - 1);
      const Row<T> F2{R(0, ch, sw), R(1, ch, sw), R(2, ch, sw), R(3, ch, sw)};
      const Row<T> L2{R(4, ch, sw), R(5, ch, sw), R(6, ch, sw), R(7, ch, sw)};
      T xF, xL;
      warp_interface_solve<T, NCH>(F2, L2, xF, xL, lane);
      sol[(0 * NCH + ch) * (SB + 1) + sw] = xF;
      sol[(1 * NCH + ch) * (SB + 1) + sw] = xL;
    }
    __syncthreads();
    chunk_backsub<T, M>(al, ga, de, sol[(0 * NCH + t) * (SB + 1) + sl],
                        sol[(1 * NCH + t) * (SB + 1) + sl]);
    if (valid) {
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const int r = r0 + j;
        if (FULL || r < n) out[obase + r * so] = INC ? uo[INC ? j : 0] + de[j] : de[j];
      }
    }
  }
}

template <typename T, int M, int SB, int NCH, int INC>
static cudaError_t launch_stream(const CUtensorMap *maps, const Geom &g, int solvedim,
                                 int box_rows, int nbox, int64_t blocks, T *d, T *u,
                                 unsigned *err, cudaStream_t st, int optin) {
  constexpr int NA = INC ? 5 : 4;
  constexpr int kAlignElems = 128 / (int)sizeof(T);
  const size_t tsz = (((size_t)box_rows * nbox * SB + kAlignElems - 1) / kAlignElems) * kAlignElems;
  const size_t smem = (size_t)NA * tsz * sizeof(T) + (size_t)10 * NCH * (SB + 1) * sizeof(T) + 128;
  if (smem + 64 > (size_t)optin || !g.fastdiv || g.n > NCH * M) return cudaErrorNotSupported;
  const bool full = g.n == NCH * M && g.odims[0] % SB == 0;
  auto kern = full ? strided_stream_kernel<T, M, SB, NCH, INC, true>
                   : strided_stream_kernel<T, M, SB, NCH, INC, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0, dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SB * NCH, smem) != cudaSuccess ||
      per_sm < 1)
    return cudaErrorNotSupported;
  const int64_t grid = std::min<int64_t>(blocks, (int64_t)per_sm * sms);
  uint32_t ntx_mul = 0, ntx_shift = 0;
  fastdiv_setup((uint32_t)((g.odims[0] + SB - 1) / SB), ntx_mul, ntx_shift);
  return launch_pdl(kern, dim3((unsigned)grid), dim3(SB * NCH), smem, st, maps[0], maps[1],
                    maps[2], maps[3], maps[4], g, solvedim, box_rows, nbox, (uint32_t)blocks,
                    ntx_mul, ntx_shift, d, u, err);
}

template <typename T, int M, int SB, int INC>
static cudaError_t launch_sptma(const CUtensorMap *maps, const Geom &g, int solvedim,
                                int box_rows, int nbox, int64_t blocks, unsigned *err,
                                cudaStream_t st, int optin, bool prefetch_tiles) {
  constexpr int NA = INC ? 5 : 4;
  constexpr int kAlignElems = 128 / (int)sizeof(T);
  const size_t tsz = (((size_t)box_rows * nbox * SB + kAlignElems - 1) / kAlignElems) * kAlignElems;
  const size_t tile = (size_t)NA * tsz * sizeof(T);
  const size_t scratch = (size_t)10 * kWarp * (SB + 1) * sizeof(T);   // red + sol
  const bool alias = scratch <= (size_t)3 * tsz * sizeof(T);
  const int red_off = alias ? 0 : (int)(NA * tsz);
  const size_t smem = (alias ? tile : tile + scratch) + 128;          // + base alignment
  if (smem + 64 > (size_t)optin) return cudaErrorNotSupported;
  auto kern = strided_part_tma_kernel<T, M, SB, INC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // prefetch distance = CTAs resident on the whole GPU at once
  int per_sm = 0, dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SB * kWarp, smem) != cudaSuccess)
    per_sm = 0;
  const int dist = prefetch_tiles ? per_sm * sms : 0;
  return launch_pdl(kern, dim3((unsigned)blocks), dim3(SB * kWarp), smem, st, maps[0], maps[1],
                    maps[2], maps[3], maps[4], g, solvedim, box_rows, nbox, red_off, dist, err);
}

template <typename T, int M, int INC>
static cudaError_t launch_sptma_sb(const CUtensorMap *maps, const Geom &g, int solvedim,
                                   int box_rows, int nbox, int spc, int nch, int64_t ntiles_rest,
                                   T *d, T *u, unsigned *err, cudaStream_t st, int optin,
                                   bool prefetch) {
  const int64_t blocks = ((g.odims[0] + spc - 1) / spc) * ntiles_rest;
  if (blocks > 0x7fffffff || blocks == 0) return cudaErrorNotSupported;
  // full-line tiles (16 FP64 / 32 FP32 systems) stream through one persistent CTA per SM
  // (at most 8 rows per thread: 16 would spill at one CTA per SM)
  if (spc * (int)sizeof(T) >= 128) {
    if constexpr (sizeof(T) == 8) {
      if constexpr (M <= 8) {
        if (spc == 16) return launch_stream<T, M, 16, 32, INC>(maps, g, solvedim, box_rows, nbox, blocks, d, u, err, st, optin);
        // short FP64 systems (16 chunks of M rows): 32 systems, 256-byte rows
        if (spc == 32 && nch == 16) return launch_stream<T, M, 32, 16, INC>(maps, g, solvedim, box_rows, nbox, blocks, d, u, err, st, optin);
        if (spc == 64 && nch == 8) return launch_stream<T, M, 64, 8, INC>(maps, g, solvedim, box_rows, nbox, blocks, d, u, err, st, optin);
      }
    } else {
      if (spc == 32 && nch == 16) return launch_stream<T, M, 32, 16, INC>(maps, g, solvedim, box_rows, nbox, blocks, d, u, err, st, optin);
      if (spc == 64 && nch == 8) return launch_stream<T, M, 64, 8, INC>(maps, g, solvedim, box_rows, nbox, blocks, d, u, err, st, optin);
      if constexpr (M <= 8) {
        if (spc == 32) return launch_stream<T, M, 32, 32, INC>(maps, g, solvedim, box_rows, nbox, blocks, d, u, err, st, optin);
      }
    }
    return cudaErrorNotSupported;
  }
  switch (spc) {
    case 4: return launch_sptma<T, M, 4, INC>(maps, g, solvedim, box_rows, nbox, blocks, err, st, optin, prefetch);
    case 8: return launch_sptma<T, M, 8, INC>(maps, g, solvedim, box_rows, nbox, blocks, err, st, optin, prefetch);
    case 16: return launch_sptma<T, M, 16, INC>(maps, g, solvedim, box_rows, nbox, blocks, err, st, optin, prefetch);
    default: return cudaErrorNotSupported;
  }
}

template <typename T, int INC>
cudaError_t launch_strided_part_tma(const Geom &g, const int *dims, const int *const pads[5],
                                    int ndim, int solvedim, const T *a, const T *b, const T *c,
                                    T *d, T *u, int chunk, int spc, bool prefetch,
                                    unsigned *err, cudaStream_t st) {
  // Full-line tiles with 16 chunks per system (a warp solves two interface
  // systems): FP64 systems of at most 128 rows as 32 systems x 16 chunks (as
  // many bytes in flight per SM as 256-row tiles), FP32 systems of at most
  // 256 rows as 32 systems x 16 chunks (512 threads instead of 1024)
  int nch = 32;
  const bool wide = (sizeof(T) == 8 && spc == 16) || (sizeof(T) == 4 && spc == 32);
  if (wide && dims[0] >= 64 && g.n <= (sizeof(T) == 8 ? 64 : 128)) {
    // shorter still (FP64 up to 64 rows, FP32 up to 128): 64 systems x 8
    // chunks, four interface systems per warp -- 128 KB tiles again
    spc = 64;
    nch = 8;
    chunk = g.n <= 16 ? 2 : (g.n <= 32 ? 4 : (g.n <= 64 ? 8 : 16));
  } else if (dims[0] >= 32 && ((sizeof(T) == 8 && spc == 16 && g.n <= 128) ||
                               (sizeof(T) == 4 && spc == 32 && g.n <= 256))) {
    spc = 32;
    nch = 16;
    chunk = g.n <= 32 ? 2 : (g.n <= 64 ? 4 : (g.n <= 128 ? 8 : 16));
  }
  if (solvedim < 1 || ndim > 5 || g.n > 32 * chunk || dims[0] < spc) return cudaErrorNotSupported;
  const int box_rows = g.n < 256 ? g.n : 256;
  const int nbox = (g.n + box_rows - 1) / box_rows;
  const int na = INC ? 5 : 4;
  const void *ptrs[5] = {a, b, c, d, u};
  CUtensorMap maps[5];
  for (int q = 0; q < 5; ++q) {
    const int qq = q < na ? q : 3;
    if (((uintptr_t)ptrs[qq] & 15) != 0 || (pads[qq][0] * sizeof(T)) % 16 != 0)
      return cudaErrorNotSupported;
    uint64_t gd[5] = {1, 1, 1, 1, 1}, gs[4];
    uint32_t box[5] = {1, 1, 1, 1, 1};
    uint64_t cum = sizeof(T);
    for (int k = 0; k < 5; ++k) {
      if (k < ndim) gd[k] = (uint64_t)dims[k];
      if (k > 0) gs[k - 1] = cum;
      cum *= (k < ndim) ? (uint64_t)pads[qq][k] : 1;
    }
    box[0] = (uint32_t)spc;
    box[solvedim] = (uint32_t)box_rows;
    if (!encode_tensor_map(&maps[q], ptrs[qq], (int)sizeof(T), 5, gd, gs, box, false))
      return cudaErrorNotSupported;
  }
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int64_t rest = g.nsys / dims[0];
  switch (chunk) {
    case 2: return launch_sptma_sb<T, 2, INC>(maps, g, solvedim, box_rows, nbox, spc, nch, rest, d, u, err, st, optin, prefetch);
    case 4: return launch_sptma_sb<T, 4, INC>(maps, g, solvedim, box_rows, nbox, spc, nch, rest, d, u, err, st, optin, prefetch);
    case 8: return launch_sptma_sb<T, 8, INC>(maps, g, solvedim, box_rows, nbox, spc, nch, rest, d, u, err, st, optin, prefetch);
    case 16: return launch_sptma_sb<T, 16, INC>(maps, g, solvedim, box_rows, nbox, spc, nch, rest, d, u, err, st, optin, prefetch);
    default: return cudaErrorNotSupported;
  }
}

#define TRID_SPTMA_INSTANTIATE(T, INC)                                                         \
  template cudaError_t launch_strided_part_tma<T, INC>(                                        \
      const Geom &, const int *, const int *const[5], int, int, const T *, const T *, const T *, \
      T *, T *, int, int, bool, unsigned *, cudaStream_t);
TRID_SPTMA_INSTANTIATE(float, 0)
TRID_SPTMA_INSTANTIATE(float, 1)
TRID_SPTMA_INSTANTIATE(double, 0)
TRID_SPTMA_INSTANTIATE(double, 1)

}  // namespace tridb200
