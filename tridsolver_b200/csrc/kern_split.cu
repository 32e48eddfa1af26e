// Systems split along the solve axis across ranks (sm_100a kernels).
//
// Every rank holds one slab -- rows [s, s+m) -- of every system.  Follows
// the reference's distributed Thomas (scalar/src/cuda/trid_cuda_mpi.cu:
// 473-583, trid_mpi_cpu.hpp:96-192): reduce each slab to two boundary
// equations, gather them over the ranks of the solve dimension, solve the
// reduced system of 2 rows per rank, then finish each slab from its
// neighbours' boundary unknowns.  The representation differs: a slab is kept
// as its two end unknowns in affine form of the unknowns just outside it,
//     x_first = y0 + p0 * l + q0 * r,   x_last = y1 + p1 * l + q1 * r
// (l = the left neighbour's last unknown, r = the right neighbour's first),
// six numbers per system and rank.  One row i is such a segment
// (y = d/b, p = -a/b, q = -c/b); two adjacent segments merge into one by
// eliminating the two unknowns between them (denominator 1 - q1*P0, whose
// factors are below 1 in magnitude for diagonally dominant rows), so a slab
// of any length >= 1 reduces by a left-to-right sweep.  The finish needs no
// kernel of its own: the slab's rows with the couplings a_first * l and
// c_last * r moved to the right-hand side are an ordinary batch (the solvers
// ignore a_first and c_last), solved by the fastest kernel for the layout.
//
// split_reduce_kernel : a thread per system and quarter of the slab sweeps
//                       its rows (consecutive lanes take adjacent systems:
//                       coalesced rows on strided axes), the quarters merge
//                       in shared memory; the six numbers go out as
//                       [6][nsys] in FP64 for both precisions.
// split_patch_kernel  : one thread per system combines the gathered slabs
//                       into the values just outside its own (FP64),
//                       subtracts the couplings from the slab's first and
//                       last d and keeps their old values (restored after an
//                       Inc solve).
#include "trid_internal.cuh"

namespace tridb200 {

struct Seg {
  double y0, p0, q0, y1, p1, q1;
};

// S (left) and T (right) adjacent: eliminate S's last and T's first unknown
__device__ __forceinline__ Seg seg_merge(const Seg &S, const Seg &T) {
  const double inv = rcp(1.0 - S.q1 * T.p0);
  const double vy = (S.y1 + S.q1 * T.y0) * inv, vp = S.p1 * inv, vq = S.q1 * T.q0 * inv;
  const double uy = T.y0 + T.p0 * vy, up = T.p0 * vp, uq = T.p0 * vq + T.q0;
  return {S.y0 + S.q0 * uy, S.p0 + S.q0 * up, S.q0 * uq,
          T.y1 + T.p1 * vy, T.p1 * vp, T.p1 * vq + T.q1};
}

// CTA = 32 adjacent systems (lane = system: coalesced rows on strided axes)
// x kSplitParts warps, warp w sweeping the w-th part of the slab's rows; the
// parts' segments merge in shared memory (warp 0, in row order)
constexpr int kSplitParts = 4;

template <typename T>
__global__ void __launch_bounds__(kSplitParts * 32) split_reduce_kernel(
    Geom g, const T *__restrict__ a, const T *__restrict__ b, const T *__restrict__ c,
    const T *__restrict__ d, double *__restrict__ bnd) {
  __shared__ double part[kSplitParts][6][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t sys = (int64_t)blockIdx.x * 32 + lane;
  const bool valid = sys < g.nsys;
  const int n = g.n;
  const int r0 = (int)((int64_t)n * w / kSplitParts), r1 = (int)((int64_t)n * (w + 1) / kSplitParts);
  Seg S{0, 0, 0, 0, 0, 0};
  if (valid && r1 > r0) {
    int64_t off[5];
    system_offsets(g, sys, off);
    const int64_t sa = g.stride[kA], sb = g.stride[kB], sc = g.stride[kC], sd = g.stride[kD];
    auto row = [&](int i) -> Seg {
      const double ib = rcp((double)b[off[kB] + i * sb]);
      const double y = (double)d[off[kD] + i * sd] * ib;
      const double p = -(double)a[off[kA] + i * sa] * ib;
      const double q = -(double)c[off[kC] + i * sc] * ib;
      return {y, p, q, y, p, q};
    };
    S = row(r0);
#pragma unroll 2
    for (int i = r0 + 1; i < r1; ++i) S = seg_merge(S, row(i));
  }
  part[w][0][lane] = S.y0;
  part[w][1][lane] = S.p0;
  part[w][2][lane] = S.q0;
  part[w][3][lane] = S.y1;
  part[w][4][lane] = S.p1;
  part[w][5][lane] = S.q1;
  __syncthreads();
  if (w != 0 || !valid) return;
  bool have = false;
  for (int k = 0; k < kSplitParts; ++k) {
    const int k0 = (int)((int64_t)n * k / kSplitParts), k1 = (int)((int64_t)n * (k + 1) / kSplitParts);
    if (k1 <= k0) continue;  // an empty part (fewer rows than parts)
    const Seg P{part[k][0][lane], part[k][1][lane], part[k][2][lane],
                part[k][3][lane], part[k][4][lane], part[k][5][lane]};
    S = have ? seg_merge(S, P) : P;
    have = true;
  }
  const int64_t ns = g.nsys;
  bnd[0 * ns + sys] = S.y0;
  bnd[1 * ns + sys] = S.p0;
  bnd[2 * ns + sys] = S.q0;
  bnd[3 * ns + sys] = S.y1;
  bnd[4 * ns + sys] = S.p1;
  bnd[5 * ns + sys] = S.q1;
}

// Gathered slabs of one system -> the unknowns just outside this rank's slab.
// The slabs left of it merge into one segment whose last unknown (the left
// neighbour l) is affine in this slab's first unknown f (its own left end
// is the boundary: 0); the slabs right of it likewise give r affine in this
// slab's last unknown e.  With this slab's own pair that is a 2x2 system in
// (f, e); l and r follow.
template <typename T>
__global__ void __launch_bounds__(128) split_patch_kernel(Geom g, const T *__restrict__ a,
                                                          const T *__restrict__ c,
                                                          T *__restrict__ d,
                                                          const double *__restrict__ bnd_all,
                                                          int nranks, int rank,
                                                          T *__restrict__ saved) {
  const int64_t sys = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (sys >= g.nsys) return;
  const int64_t ns = g.nsys;
  auto seg = [&](int k) -> Seg {
    const double *q = bnd_all + (int64_t)k * 6 * ns + sys;
    return {q[0], q[ns], q[2 * ns], q[3 * ns], q[4 * ns], q[5 * ns]};
  };
  // l = ly + lq * f   (0 without slabs to the left)
  double ly = 0.0, lq = 0.0;
  if (rank > 0) {
    Seg Lft = seg(0);
    for (int k = 1; k < rank; ++k) Lft = seg_merge(Lft, seg(k));
    ly = Lft.y1;
    lq = Lft.q1;
  }
  // r = ry + rp * e   (0 without slabs to the right)
  double ry = 0.0, rp = 0.0;
  if (rank < nranks - 1) {
    Seg Rgt = seg(rank + 1);
    for (int k = rank + 2; k < nranks; ++k) Rgt = seg_merge(Rgt, seg(k));
    ry = Rgt.y0;
    rp = Rgt.p0;
  }
  const Seg S = seg(rank);
  // (1 - p0 lq) f - q0 rp e = y0 + p0 ly + q0 ry
  // -p1 lq f + (1 - q1 rp) e = y1 + p1 ly + q1 ry
  const double m00 = 1.0 - S.p0 * lq, m01 = -S.q0 * rp;
  const double m10 = -S.p1 * lq, m11 = 1.0 - S.q1 * rp;
  const double r0 = S.y0 + S.p0 * ly + S.q0 * ry, r1 = S.y1 + S.p1 * ly + S.q1 * ry;
  const double det = m00 * m11 - m01 * m10;
  const double f = (r0 * m11 - m01 * r1) / det, e = (m00 * r1 - m10 * r0) / det;
  const double left = ly + lq * f, right = ry + rp * e;

  int64_t off[5];
  system_offsets(g, sys, off);
  const int64_t i0 = off[kD], i1 = off[kD] + (int64_t)(g.n - 1) * g.stride[kD];
  const T d0 = d[i0], d1 = d[i1];
  if (saved) {
    saved[sys] = d0;
    saved[ns + sys] = d1;
  }
  const double a0 = (double)a[off[kA]];
  const double c1 = (double)c[off[kC] + (int64_t)(g.n - 1) * g.stride[kC]];
  d[i0] = (T)((double)d0 - a0 * left);
  d[i1] = (T)((double)d1 - c1 * right);
}

template <typename T>
__global__ void __launch_bounds__(128) split_restore_kernel(Geom g, T *__restrict__ d,
                                                            const T *__restrict__ saved) {
  const int64_t sys = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (sys >= g.nsys) return;
  int64_t off[5];
  system_offsets(g, sys, off);
  d[off[kD]] = saved[sys];
  d[off[kD] + (int64_t)(g.n - 1) * g.stride[kD]] = saved[g.nsys + sys];
}

static dim3 split_grid(const Geom &g) { return dim3((unsigned)((g.nsys + 127) / 128)); }

template <typename T>
cudaError_t launch_split_reduce(const Geom &g, const T *a, const T *b, const T *c, const T *d,
                                double *bnd, cudaStream_t st) {
  const int64_t blocks = (g.nsys + 31) / 32;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  split_reduce_kernel<T><<<dim3((unsigned)blocks), kSplitParts * 32, 0, st>>>(g, a, b, c, d, bnd);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_split_patch(const Geom &g, const T *a, const T *c, T *d, const double *bnd_all,
                               int nranks, int rank, T *saved, cudaStream_t st) {
  if ((g.nsys + 127) / 128 > 0x7fffffff || nranks < 1 || rank < 0 || rank >= nranks)
    return cudaErrorInvalidConfiguration;
  split_patch_kernel<T><<<split_grid(g), 128, 0, st>>>(g, a, c, d, bnd_all, nranks, rank, saved);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_split_restore(const Geom &g, T *d, const T *saved, cudaStream_t st) {
  split_restore_kernel<T><<<split_grid(g), 128, 0, st>>>(g, d, saved);
  return cudaGetLastError();
}

#define TRID_SPLIT_INSTANTIATE(T)                                                              \
  template cudaError_t launch_split_reduce<T>(const Geom &, const T *, const T *, const T *,  \
                                              const T *, double *, cudaStream_t);             \
  template cudaError_t launch_split_patch<T>(const Geom &, const T *, const T *, T *,         \
                                             const double *, int, int, T *, cudaStream_t);    \
  template cudaError_t launch_split_restore<T>(const Geom &, T *, const T *, cudaStream_t);
TRID_SPLIT_INSTANTIATE(float)
TRID_SPLIT_INSTANTIATE(double)

}  // namespace tridb200
