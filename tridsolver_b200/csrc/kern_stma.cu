// Strided-axis solve (solvedim >= 1): TMA-staged two-sided Thomas (sm_100a).
//
// A CTA is one warp and owns 16 adjacent systems (16 consecutive x at a fixed
// position on the other non-solve axes; 128 contiguous bytes per row in FP64).
// Lanes 0-15 eliminate their system from the top (rows 0..h-1, the forward
// Thomas sweep of trid_cpu.cpp:360-401), lanes 16-31 eliminate the same
// system from the bottom (rows n-1..h, eliminating super-diagonals), in
// lockstep: both halves execute the same instruction stream on different
// rows, so nothing diverges.  The two halves meet at rows h-1 / h (a 2x2
// solve through one shuffle), then back-substitute outwards.  This
// "twisted" factorisation halves the dependent chain of reciprocals
// (the latency that bounds a one-thread-per-system Thomas).
//
// Rows arrive through a ring of TMA stages (cp.async.bulk.tensor, rank-5
// view of the N-D array, box = 16 x R rows, completion on mbarriers); the
// modified coefficients c'/d' (top) and a''/d'' (bottom) stay in shared
// memory, so global memory sees each input element read once and each
// output element written once.
//
// Preconditions (launch_strided_tma returns cudaErrorNotSupported otherwise):
// ndim <= 5, 16-byte aligned base pointers, pads[0]*sizeof(T) a multiple of
// 16 for every array, and 2*n*16*sizeof(T) bytes of c'/d' storage that fit
// in shared memory next to the stage ring.
#include "tma.cuh"
#include "trid_internal.cuh"

namespace tridb200 {

constexpr int kSW = 16;      // systems per CTA
constexpr int kSRows = 8;    // rows per stage per direction
constexpr int kSStages = 4;  // ring depth

template <typename T, int INC>
__global__ void __launch_bounds__(kWarp) strided_tma_kernel(
    const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb,
    const __grid_constant__ CUtensorMap mc, const __grid_constant__ CUtensorMap md, Geom g,
    int solvedim, T *__restrict__ d, T *__restrict__ u, unsigned *err) {
  constexpr int kBox = kSRows * kSW;            // elements per box
  constexpr int kStage = 4 * 2 * kBox;          // elements per stage (4 arrays, 2 boxes)
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t full[kSStages];
  // stage boxes are 1 KB (FP64) / 512 B (FP32) apart: align the ring to 128 B
  T *ring = reinterpret_cast<T *>(smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127));
  T *cq = ring + kSStages * kStage;             // c' (top rows) / a'' (bottom rows)
  T *cd = cq + (size_t)g.n * kSW;               // d' / d''

  const int lane = threadIdx.x;
  const int sl = lane & (kSW - 1);
  const bool top = lane < kSW;
  const int n = g.n;
  const int h = (n + 1) / 2;                    // top rows [0,h), bottom rows [h,n)
  const int nsteps = h;
  const int K = (h + kSRows - 1) / kSRows;      // stages

  // tile -> x0 and the coordinates of the other non-solve axes
  const int ntx = (g.odims[0] + kSW - 1) / kSW;
  const int x0 = (int)(blockIdx.x % ntx) * kSW;
  uint32_t rest = blockIdx.x / ntx;
  int coord[5] = {x0, 0, 0, 0, 0};
  int64_t roff[5] = {0, 0, 0, 0, 0};
  {
    int o = 1;
    for (int k = 1; k < 5; ++k) {
      if (k == solvedim) continue;
      if (o < g.nod) {
        const uint32_t e = (uint32_t)g.odims[o];
        const uint32_t i = rest % e;
        rest /= e;
        coord[k] = (int)i;
#pragma unroll
        for (int q = 0; q < 5; ++q) roff[q] += (int64_t)i * g.ocum[q][o];
        ++o;
      }
    }
  }
  const int x = x0 + sl;
  const bool valid = x < g.odims[0];

  auto issue = [&](int k) {
    const int slot = k % kSStages;
    T *st = ring + slot * kStage;
    uint32_t bytes = 4u * 2u * kBox * (uint32_t)sizeof(T);
    mbar_arrive_expect_tx(&full[slot], bytes);
    const CUtensorMap *maps[4] = {&ma, &mb, &mc, &md};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int c[5] = {coord[0], coord[1], coord[2], coord[3], coord[4]};
      c[solvedim] = k * kSRows;                       // top box
      tma_load_5d(st + (2 * q) * kBox, maps[q], &full[slot], c[0], c[1], c[2], c[3], c[4]);
      c[solvedim] = n - (k + 1) * kSRows;             // bottom box (may start below row 0)
      tma_load_5d(st + (2 * q + 1) * kBox, maps[q], &full[slot], c[0], c[1], c[2], c[3], c[4]);
    }
  };

  static_assert((kSRows * kSW * 4) % 128 == 0, "stage boxes must stay 128-byte aligned");
  if (!tma_smem_aligned(ring)) {
    if (lane == 0) atomicOr(err, kErrMisaligned);
    return;
  }
  if (lane == 0) {
    for (int s = 0; s < kSStages; ++s) mbar_init(&full[s], 1);
    fence_barrier_init();
  }
  __syncwarp();
  if (lane == 0)
    for (int k = 0; k < K && k < kSStages; ++k) issue(k);

  // ---------------------------------------------------------- elimination --
  T qprev = T(0), dprev = T(0);
  bool ok = true;
  for (int k = 0; k < K; ++k) {
    const int slot = k % kSStages;
    if (!mbar_wait(&full[slot], (uint32_t)((k / kSStages) & 1), err)) {
      ok = false;
      break;
    }
    const T *st = ring + slot * kStage;
#pragma unroll
    for (int j = 0; j < kSRows; ++j) {
      const int step = k * kSRows + j;
      const int i = top ? step : n - 1 - step;            // row of this lane
      const bool act = step < nsteps && (top || i >= h);
      const int lr = top ? j : kSRows - 1 - j;             // row inside the box
      const int box = top ? 0 : 1;
      const T av = st[(0 + box) * kBox + lr * kSW + sl];
      const T bv = st[(2 + box) * kBox + lr * kSW + sl];
      const T cv = st[(4 + box) * kBox + lr * kSW + sl];
      const T dv = st[(6 + box) * kBox + lr * kSW + sl];
      // p couples to the row already eliminated, q to the next one
      T p = top ? av : cv;
      T q = top ? cv : av;
      if (step == 0) p = T(0);                             // a[0] / c[n-1] never read
      if (top ? (i == n - 1) : (i == 0)) q = T(0);
      if (act) {
        const T r = rcp(bv - p * qprev);
        qprev = q * r;
        dprev = (dv - p * dprev) * r;
        cq[i * kSW + sl] = qprev;
        cd[i * kSW + sl] = dprev;
      }
    }
    fence_proxy_async();  // this slot's reads come before its next TMA write
    __syncwarp();
    if (lane == 0 && k + kSStages < K) issue(k + kSStages);
  }
  if (!ok) {
    for (int s = 0; s < kSStages; ++s) mbar_wait(&full[s], 0, nullptr);
    return;
  }

  // ------------------------------------------------- meet in the middle --
  // top: x_{h-1} + c' x_h = d' ; bottom: x_h + a'' x_{h-1} = d''
  const bool has_bottom = n - h > 0;
  T oq = __shfl_xor_sync(0xffffffffu, qprev, kSW);
  T od = __shfl_xor_sync(0xffffffffu, dprev, kSW);
  T tq = top ? qprev : oq, td = top ? dprev : od;       // top's c', d' at h-1
  T bq = top ? oq : qprev, bd = top ? od : dprev;       // bottom's a'', d'' at h
  if (!has_bottom) {
    bq = T(0);
    bd = T(0);
  }
  const T xm = (td - tq * bd) * rcp(T(1) - tq * bq);    // x_{h-1}
  const T xp = bd - bq * xm;                            // x_h
  T xcur = top ? xm : xp;

  // ------------------------------------------------------ back-substitution --
  const int64_t sd = g.stride[kD], su = g.stride[kU];
  const int64_t baseD = roff[kD] + x, baseU = roff[kU] + x;
  auto put = [&](int i, T v) {
    if (INC)
      u[baseU + (int64_t)i * su] += v;
    else
      d[baseD + (int64_t)i * sd] = v;
  };
  if (valid) {
    if (top) put(h - 1, xcur);
    else if (has_bottom) put(h, xcur);
  }
  for (int step = 1; step < nsteps; ++step) {
    const int i = top ? h - 1 - step : h + step;
    const bool act = top ? true : (i < n);
    if (act) {
      xcur = cd[i * kSW + sl] - cq[i * kSW + sl] * xcur;
      if (valid) put(i, xcur);
    }
  }
}

template <typename T, int INC>
cudaError_t launch_strided_tma(const Geom &g, const int *dims, const int *const pads[5],
                               int ndim, int solvedim, const T *a, const T *b, const T *c, T *d,
                               T *u, unsigned *err, cudaStream_t st) {
  if (solvedim < 1 || ndim > 5 || g.n < kSRows || dims[0] < kSW) return cudaErrorNotSupported;
  const size_t ring = (size_t)kSStages * 4 * 2 * kSRows * kSW * sizeof(T);
  const size_t store = (size_t)2 * g.n * kSW * sizeof(T);
  const size_t smem = ring + store + 128;  // + base alignment
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem + 64 > (size_t)optin) return cudaErrorNotSupported;

  const void *ptrs[4] = {a, b, c, d};
  CUtensorMap maps[4];
  for (int q = 0; q < 4; ++q) {
    if (((uintptr_t)ptrs[q] & 15) != 0 || (pads[q][0] * sizeof(T)) % 16 != 0)
      return cudaErrorNotSupported;
    uint64_t gd[5] = {1, 1, 1, 1, 1}, gs[4];
    uint32_t box[5] = {1, 1, 1, 1, 1};
    uint64_t cum = sizeof(T);
    for (int k = 0; k < 5; ++k) {
      if (k < ndim) gd[k] = (uint64_t)dims[k];
      if (k > 0) gs[k - 1] = cum;
      cum *= (k < ndim) ? (uint64_t)pads[q][k] : 1;
    }
    box[0] = kSW;
    box[solvedim] = kSRows;
    if (!encode_tensor_map(&maps[q], ptrs[q], (int)sizeof(T), 5, gd, gs, box, false))
      return cudaErrorNotSupported;
  }
  const int64_t ntx = (dims[0] + kSW - 1) / kSW;
  const int64_t blocks = ntx * (g.nsys / dims[0]);
  if (blocks > 0x7fffffff || blocks == 0) return cudaErrorNotSupported;
  auto kern = strided_tma_kernel<T, INC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<dim3((unsigned)blocks), dim3(kWarp), smem, st>>>(maps[0], maps[1], maps[2], maps[3], g,
                                                          solvedim, d, u, err);
  return cudaGetLastError();
}

#define TRID_STMA_INSTANTIATE(T, INC)                                                            \
  template cudaError_t launch_strided_tma<T, INC>(const Geom &, const int *, const int *const[5], \
                                                  int, int, const T *, const T *, const T *, T *, \
                                                  T *, unsigned *, cudaStream_t);
TRID_STMA_INSTANTIATE(float, 0)
TRID_STMA_INSTANTIATE(float, 1)
TRID_STMA_INSTANTIATE(double, 0)
TRID_STMA_INSTANTIATE(double, 1)

}  // namespace tridb200
