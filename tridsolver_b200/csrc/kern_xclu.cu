// Long axis-0 systems solved by a thread-block cluster each (sm_100a): the
// partition of kern_xcta.cu carried one level further, so that systems of
// 4097 .. 65,536 rows are read once and written once (40 B per FP64 unknown)
// instead of twice as by the blocked partition of kern_general.cu (72 B).
//
// Cluster = one system, C = ceil(n / 4096) CTAs (at most 16); CTA r owns rows
// [4096 r, 4096 (r+1)), 8 warps of 32 lanes of 16 rows.  The rows go straight
// from global memory into registers (16-byte loads where the rows are
// aligned; no shared-memory staging, so that two CTAs fit on an SM) and stay
// there until the solution leaves:
//   1. every lane reduces its 16 rows (chunk_reduce_cont), every warp its 32
//      chunks to a block basis and two block rows (warp_block_basis,
//      block_rows);
//   2. warp 0 of each CTA does the same over the CTA's 8 warp blocks (their
//      block rows are an interface system of 8 lanes): a CTA basis and two
//      CTA rows, which it writes into the shared memory of the cluster's rank
//      0 (distributed shared memory);
//   3. cluster barrier; warp 0 of rank 0 solves the cluster system (2C rows,
//      one warp interface solve) and writes every CTA's two boundary unknowns
//      into that CTA's shared memory; cluster barrier;
//   4. each CTA expands them through its CTA basis into its warps' block
//      boundary unknowns, each warp through its block basis into its chunks'
//      interface unknowns, each lane back-substitutes its 16 rows and stores
//      them (16-byte stores where aligned).
// Rows past n (the last CTA's tail) are identity rows, decoupled because
// c[n-1] is never read.  Forward modes (x into d, or added into u).
#include <cooperative_groups.h>

#include "partition.cuh"

namespace tridb200 {

namespace cg = cooperative_groups;

constexpr int kCluWarps = 8;
constexpr int kCluM = 16;                          // rows per lane
constexpr int kCluRows = kCluWarps * 32 * kCluM;   // rows per CTA
constexpr int kCluMax = 16;                        // CTAs per cluster at most

// 16 consecutive values of p into v (16-byte loads when p is 16-byte aligned
// and all 16 rows exist; else element by element, rows >= cnt read as `fill`)
template <typename T>
__device__ __forceinline__ void clu_load16(const T *p, int cnt, T fill, T (&v)[kCluM]) {
  constexpr int V = 16 / (int)sizeof(T);
  if (cnt >= kCluM && ((uintptr_t)p & 15) == 0) {
#pragma unroll
    for (int j = 0; j < kCluM; j += V) {
      if constexpr (sizeof(T) == 8) {
        const double2 u = __ldcs(reinterpret_cast<const double2 *>(p + j));
        v[j] = u.x;
        v[j + 1] = u.y;
      } else {
        const float4 u = __ldcs(reinterpret_cast<const float4 *>(p + j));
        v[j] = u.x;
        v[j + 1] = u.y;
        v[j + 2] = u.z;
        v[j + 3] = u.w;
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < kCluM; ++j) v[j] = j < cnt ? __ldcs(p + j) : fill;
  }
}

template <typename T, bool ADD>
__device__ __forceinline__ void clu_store16(T *p, int cnt, const T (&v)[kCluM]) {
  constexpr int V = 16 / (int)sizeof(T);
  if (cnt >= kCluM && ((uintptr_t)p & 15) == 0) {
#pragma unroll
    for (int j = 0; j < kCluM; j += V) {
      if constexpr (sizeof(T) == 8) {
        double2 u = make_double2(v[j], v[j + 1]);
        if (ADD) {
          const double2 o = *reinterpret_cast<const double2 *>(p + j);
          u.x += o.x;
          u.y += o.y;
        }
        __stcs(reinterpret_cast<double2 *>(p + j), u);
      } else {
        float4 u = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        if (ADD) {
          const float4 o = *reinterpret_cast<const float4 *>(p + j);
          u.x += o.x;
          u.y += o.y;
          u.z += o.z;
          u.w += o.w;
        }
        __stcs(reinterpret_cast<float4 *>(p + j), u);
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < kCluM; ++j)
      if (j < cnt) p[j] = ADD ? p[j] + v[j] : v[j];
  }
}

template <typename T, int INC>
__global__ void __launch_bounds__(kCluWarps * 32, 2) xclu_kernel(Geom g, XArgs<T> A) {
  // shared: [0, 64) the warps' block rows (8 per warp), [64, 80) the warps'
  // block boundary unknowns, [80, 80 + 8*kCluMax) the CTA rows of the whole
  // cluster (rank 0 only), [208, 210) this CTA's boundary unknowns
  __shared__ T sm[210];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int C = (int)cluster.num_blocks();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t sys = blockIdx.x / C;
  int64_t off[5];
  system_offsets(g, sys, off);
  const int n = g.n;
  const int r0 = rank * kCluRows + w * 32 * kCluM + lane * kCluM;  // this lane's first row
  const int cnt = n - r0;  // rows of this lane that exist (may be <= 0 or > 16)

  // ---- 1. rows into registers, chunk reduction, warp block basis ----
  T al[kCluM], be[kCluM], ga[kCluM], de[kCluM], rp[kCluM];
  clu_load16(A.a + off[kA] + r0, cnt, T(0), al);
  clu_load16(A.b + off[kB] + r0, cnt, T(1), be);
  clu_load16(A.c + off[kC] + r0, cnt, T(0), ga);
  clu_load16(A.d + off[kD] + r0, cnt, T(0), de);
  if (r0 == 0) al[0] = T(0);                           // a[0] is never read
  if (cnt > 0 && cnt <= kCluM) ga[cnt - 1] = T(0);     // nor c[n-1]
  Row<T> F, L;
  chunk_reduce_cont<T, kCluM>(al, be, ga, de, F, L, rp);
  T bF[3], bL[3];
  warp_block_basis(F, L, lane, bF, bL);
  {
    Row<T> FB, LB;
    block_rows(F, L, bF, bL, lane, FB, LB);
    if (lane == 0) {
      T *q = sm + 8 * w;
      q[0] = FB.a; q[1] = FB.b; q[2] = FB.c; q[3] = FB.d;
      q[4] = LB.a; q[5] = LB.b; q[6] = LB.c; q[7] = LB.d;
    }
  }
  __syncthreads();

  // ---- 2. warp 0: CTA basis over the 8 warp blocks, CTA rows to rank 0 ----
  T cF[3] = {T(0), T(0), T(0)}, cL[3] = {T(0), T(0), T(0)};
  if (w == 0) {
    Row<T> RF{T(0), T(1), T(0), T(0)}, RL{T(0), T(1), T(0), T(0)};
    if (lane < kCluWarps) {
      const T *q = sm + 8 * lane;
      RF = {q[0], q[1], q[2], q[3]};
      RL = {q[4], q[5], q[6], q[7]};
    }
    warp_block_basis(RF, RL, lane, cF, cL, kCluWarps - 1);
    Row<T> FC, LC;
    block_rows(RF, RL, cF, cL, lane, FC, LC, kCluWarps - 1);
    if (lane == 0) {
      T *q = cluster.map_shared_rank(sm + 80, 0) + 8 * rank;
      q[0] = FC.a; q[1] = FC.b; q[2] = FC.c; q[3] = FC.d;
      q[4] = LC.a; q[5] = LC.b; q[6] = LC.c; q[7] = LC.d;
    }
  }
  cluster.sync();

  // ---- 3. rank 0, warp 0: the cluster system; boundary unknowns back ----
  if (rank == 0 && w == 0) {
    Row<T> RF{T(0), T(1), T(0), T(0)}, RL{T(0), T(1), T(0), T(0)};
    if (lane < C) {
      const T *q = sm + 80 + 8 * lane;
      RF = {q[0], q[1], q[2], q[3]};
      RL = {q[4], q[5], q[6], q[7]};
    }
    T f, l;
    int span = 1;
    while (span < C) span <<= 1;
    warp_interface_solve(RF, RL, f, l, lane, span);
    if (lane < C) {
      T *q = cluster.map_shared_rank(sm + 208, lane);
      q[0] = f;
      q[1] = l;
    }
  }
  cluster.sync();  // no distributed shared memory access after this point

  // ---- 4. expand: CTA -> warp blocks -> chunks; back-substitute; store ----
  if (w == 0) {
    const T fC = sm[208], lC = sm[209];
    if (lane < kCluWarps) {
      sm[64 + 2 * lane] = cF[0] + fC * cF[1] + lC * cF[2];
      sm[64 + 2 * lane + 1] = cL[0] + fC * cL[1] + lC * cL[2];
    }
  }
  __syncthreads();
  const T f = sm[64 + 2 * w], l = sm[64 + 2 * w + 1];
  const T xF = bF[0] + f * bF[1] + l * bF[2];
  const T xL = bL[0] + f * bL[1] + l * bL[2];
  chunk_backsub<T, kCluM>(al, ga, de, xF, xL);
  if (cnt > 0) {
    if (INC)
      clu_store16<T, true>(A.x + off[kU] + r0, cnt, de);
    else
      clu_store16<T, false>(A.x + off[kD] + r0, cnt, de);
  }
}

// cudaErrorNotSupported when the cluster form does not apply (n outside
// 4097 .. 16 * 4096, or clusters of that size do not fit); the caller then
// takes the blocked partition.
template <typename T, int INC>
cudaError_t launch_xclu(const Geom &g, const XArgs<T> &A, cudaStream_t st) {
  const int n = g.n;
  if (n <= 4096 || n > kCluMax * kCluRows || g.nsys <= 0) return cudaErrorNotSupported;
  const int C = (n + kCluRows - 1) / kCluRows;
  if ((int64_t)g.nsys * C > 0x7fffffff) return cudaErrorNotSupported;
  auto kern = xclu_kernel<T, INC>;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorNotSupported;
  static bool attr_set[64] = {};
  if (!attr_set[dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return cudaErrorNotSupported;
    }
    attr_set[dev] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(g.nsys * C));
  cfg.blockDim = dim3(kCluWarps * 32);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) {
    cudaGetLastError();
    return cudaErrorNotSupported;
  }
  e = cudaLaunchKernelEx(&cfg, kern, g, A);
  return e;
}

template cudaError_t launch_xclu<float, 0>(const Geom &, const XArgs<float> &, cudaStream_t);
template cudaError_t launch_xclu<float, 1>(const Geom &, const XArgs<float> &, cudaStream_t);
template cudaError_t launch_xclu<double, 0>(const Geom &, const XArgs<double> &, cudaStream_t);
template cudaError_t launch_xclu<double, 1>(const Geom &, const XArgs<double> &, cudaStream_t);

}  // namespace tridb200
