// ADI heat-diffusion kernels (sm_100a): the reference app's step
// (apps/adi/src/adi_orig.c:147-240, preproc.hpp:172-214, adi_cuda.cu:285-329)
// with the tridiagonal coefficients generated from the grid position instead
// of stored (the reference writes 9 coefficient arrays per step).
//
// Grid nx*ny*nz, x fastest.  A point is interior when no index is on a face.
// Interior rows: (a, b, c) = (ca, cb, cc); face rows: identity (0, 1, 0); the
// RHS of a step is r = lambda*(sum of the 6 neighbours - 6u) on interior
// points and 0 on faces.  One step:
//     du1 = X^{-1} r     (adi_x_kernel: stencil fused into the x solve)
//     du2 = Y^{-1} du1   (adi_s_kernel, axis 1)
//     u  += Z^{-1} du2   (adi_s_kernel, axis 2, Inc)
// Moved per step (FP64): 8 B read + 8 B write (x), 16 B (y), 24 B (z) per
// point = 56 B, against 80 B of coefficient writes alone in the reference.
//
// TRANS = true solves the transposed systems (sub-diagonal c_{i-1},
// super-diagonal a_{i+1}) for the adjoint of a step.
#include "partition.cuh"

namespace tridb200 {

template <typename T>
struct AdiArgs {
  int nx, ny, nz;
  T lam, ca, cb, cc;
  const T *rhs;   // x pass with stencil: u; otherwise the right-hand side
  T *out;         // solution (or += for Inc)
};

template <typename T>
__device__ __forceinline__ bool adi_inside(const AdiArgs<T> &g, int i, int j, int k) {
  return i > 0 && i < g.nx - 1 && j > 0 && j < g.ny - 1 && k > 0 && k < g.nz - 1;
}

// coefficients of row r of the line through (i,j,k) along `axis`
template <typename T, bool TRANS>
__device__ __forceinline__ void adi_row(const AdiArgs<T> &g, int axis, int i, int j, int k, T &al,
                                        T &be, T &ga) {
  auto at = [&](int d) {  // neighbour along the axis, inside?
    int ii = i, jj = j, kk = k;
    if (axis == 0) ii += d; else if (axis == 1) jj += d; else kk += d;
    return adi_inside(g, ii, jj, kk);
  };
  const bool in = adi_inside(g, i, j, k);
  be = in ? g.cb : T(1);
  if (!TRANS) {
    al = in ? g.ca : T(0);
    ga = in ? g.cc : T(0);
  } else {
    al = at(-1) ? g.cc : T(0);  // c of the row above
    ga = at(+1) ? g.ca : T(0);  // a of the row below
  }
}

// ------------------------------------------------------------- x lines --
// x lines, one warp per line (4 per CTA), every load coalesced: lane l
// holds the points i = q*32 + l (q < M) of the right-hand side -- with
// STENCIL formed there from the five lines the 7-point stencil reads (the
// line, j-1, j+1, k-1, k+1; the x neighbours i-1, i+1 by shuffles) -- which
// passes through the warp's shared-memory slot into the lane-per-chunk layout
// of the solve (lane l: points l*M .. l*M+M-1; point i at i + i/M,
// conflict-free both ways); the solution leaves the same way.  (Reading the
// stencil lane by lane -- 4 consecutive points per lane, 7 loads each,
// strided across the warp -- took 49-51 us per 128^3 step against 45.)
// The x, y and z kernels run under programmatic dependent launch
// (launch_pdl / pdl_enter): each may be scheduled while its predecessor
// finishes and waits for it before its first global access.
template <typename T, int M, bool STENCIL, bool TRANS>
__global__ void __launch_bounds__(128) adi_x_kernel(AdiArgs<T> g) {
  pdl_enter();
  __shared__ T sbuf[4][32 * (M + 1)];
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & (kWarp - 1);
  const int wi = threadIdx.x / kWarp;
  const int64_t line = (int64_t)blockIdx.x * 4 + wi;
  if (line >= (int64_t)g.ny * g.nz) return;  // whole warp
  const int j = (int)(line % g.ny), k = (int)(line / g.ny);
  const int64_t sxy = (int64_t)g.nx * g.ny;
  const int64_t base = (int64_t)k * sxy + (int64_t)j * g.nx;
  const T *u = g.rhs + base;
  T *sb = sbuf[wi];
  if (!STENCIL) {
#pragma unroll
    for (int q = 0; q < M; ++q) {
      const int i = q * kWarp + lane;
      sb[i + i / M] = i < g.nx ? u[i] : T(0);
    }
  }
  // interior line (its points off the x faces are interior points)
  const bool line_in = STENCIL && j > 0 && j < g.ny - 1 && k > 0 && k < g.nz - 1;
  T c[M];
#pragma unroll
  for (int q = 0; q < M; ++q) {
    const int i = q * kWarp + lane;
    c[q] = (line_in && i < g.nx) ? u[i] : T(0);
  }
#pragma unroll
  for (int q = 0; STENCIL && q < M; ++q) {
    const int i = q * kWarp + lane;
    T left = __shfl_up_sync(kFull, c[q], 1);
    const T lq = __shfl_sync(kFull, c[q > 0 ? q - 1 : 0], kWarp - 1);
    if (lane == 0) left = lq;
    T right = __shfl_down_sync(kFull, c[q], 1);
    const T rq = __shfl_sync(kFull, c[q + 1 < M ? q + 1 : q], 0);
    if (lane == kWarp - 1) right = rq;
    T r = T(0);
    if (line_in && i > 0 && i < g.nx - 1)
      r = g.lam * (left + right + u[i - g.nx] + u[i + g.nx] + u[i - sxy] + u[i + sxy] -
                   T(6) * c[q]);
    sb[i + i / M] = r;
  }
  __syncwarp();
  T al[M], be[M], ga[M], de[M];
#pragma unroll
  for (int q = 0; q < M; ++q) {
    const int i = lane * M + q;
    if (i < g.nx) {
      adi_row<T, TRANS>(g, 0, i, j, k, al[q], be[q], ga[q]);
      de[q] = sb[lane * (M + 1) + q];
    } else {
      al[q] = T(0);
      be[q] = T(1);
      ga[q] = T(0);
      de[q] = T(0);
    }
  }
  Row<T> F, L;
  chunk_reduce<T, M>(al, be, ga, de, F, L);
  T xF, xL;
  warp_interface_solve(F, L, xF, xL, lane);
  chunk_backsub<T, M>(al, ga, de, xF, xL);
  __syncwarp();  // every lane has read its r slots
#pragma unroll
  for (int q = 0; q < M; ++q) sb[lane * (M + 1) + q] = de[q];
  __syncwarp();
#pragma unroll
  for (int q = 0; q < M; ++q) {
    const int i = q * kWarp + lane;
    if (i < g.nx) g.out[base + i] = sb[i + i / M];
  }
}

// ------------------------------------------------------- y and z lines --
// CTA = SB adjacent lines x NCH chunks of M rows (NCH = 32, or 16 for lines
// of at most 128 rows: a warp then solves two lines' interface systems side
// by side in lane groups of 16)
template <typename T, int M, int SB, int NCH, int AXIS, bool TRANS, bool INC>
__global__ void __launch_bounds__(SB * NCH) adi_s_kernel(AdiArgs<T> g) {
  pdl_enter();
  __shared__ T red[8][NCH][SB + 1];
  __shared__ T sol[2][NCH][SB + 1];
  const int tid = threadIdx.x;
  const int sl = tid % SB, t = tid / SB;
  const int ntx = (g.nx + SB - 1) / SB;
  const int other = (AXIS == 1) ? g.nz : g.ny;
  const int64_t blk = blockIdx.x;
  const int i = (int)(blk % ntx) * SB + sl;
  const int o = (int)(blk / ntx);  // k for axis 1, j for axis 2
  const bool valid = i < g.nx && o < other;
  const int n = (AXIS == 1) ? g.ny : g.nz;
  const int64_t sxy = (int64_t)g.nx * g.ny;
  const int64_t stride = (AXIS == 1) ? g.nx : sxy;
  const int64_t base = (AXIS == 1) ? (int64_t)o * sxy + i : (int64_t)o * g.nx + i;
  T al[M], be[M], ga[M], de[M];
#pragma unroll
  for (int q = 0; q < M; ++q) {
    const int r = t * M + q;
    if (valid && r < n) {
      const int jj = (AXIS == 1) ? r : o, kk = (AXIS == 1) ? o : r;
      adi_row<T, TRANS>(g, AXIS, i, jj, kk, al[q], be[q], ga[q]);
      de[q] = g.rhs[base + (int64_t)r * stride];
    } else {
      al[q] = T(0);
      be[q] = T(1);
      ga[q] = T(0);
      de[q] = T(0);
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
    const int lane = tid & (kWarp - 1);
    const int w = (NCH == kWarp) ? tid / kWarp : (tid / kWarp) * (kWarp / NCH) + lane / NCH;
    const int ch = (NCH == kWarp) ? lane : lane & (NCH - 1);
    const Row<T> F2{red[0][ch][w], red[1][ch][w], red[2][ch][w], red[3][ch][w]};
    const Row<T> L2{red[4][ch][w], red[5][ch][w], red[6][ch][w], red[7][ch][w]};
    T xF, xL;
    warp_interface_solve<T, NCH>(F2, L2, xF, xL, lane);
    sol[0][ch][w] = xF;
    sol[1][ch][w] = xL;
  }
  __syncthreads();
  chunk_backsub<T, M>(al, ga, de, sol[0][t][sl], sol[1][t][sl]);
  if (!valid) return;
#pragma unroll
  for (int q = 0; q < M; ++q) {
    const int r = t * M + q;
    if (r < n) {
      const int64_t p = base + (int64_t)r * stride;
      if (INC)
        g.out[p] += de[q];
      else
        g.out[p] = de[q];
    }
  }
}

// L^T applied to g, scaled and added: out += lam * L^T g, where L is the
// interior-masked 7-point Laplacian (L u)_p = sum_nbr u - 6 u_p on interior
// p, 0 on faces.  (L^T g)_q = sum over interior neighbours p of q of g_p,
// minus 6 g_q if q is interior.
template <typename T>
__global__ void adi_lt_kernel(AdiArgs<T> g, const T *__restrict__ gin) {
  const int64_t total = (int64_t)g.nx * g.ny * g.nz;
  const int64_t sxy = (int64_t)g.nx * g.ny;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / sxy);
    T acc = adi_inside(g, i, j, k) ? T(-6) * gin[p] : T(0);
    if (i > 0 && adi_inside(g, i - 1, j, k)) acc += gin[p - 1];
    if (i < g.nx - 1 && adi_inside(g, i + 1, j, k)) acc += gin[p + 1];
    if (j > 0 && adi_inside(g, i, j - 1, k)) acc += gin[p - g.nx];
    if (j < g.ny - 1 && adi_inside(g, i, j + 1, k)) acc += gin[p + g.nx];
    if (k > 0 && adi_inside(g, i, j, k - 1)) acc += gin[p - sxy];
    if (k < g.nz - 1 && adi_inside(g, i, j, k + 1)) acc += gin[p + sxy];
    g.out[p] += g.lam * acc;
  }
}

// Cotangent of one step's lambda and the u-cotangent's Laplacian term, in one
// pass.  With du1 = X^{-1} r, du2 = Y^{-1} du1, du3 = Z^{-1} du2 (r = lam L u)
// and g3 = Z^{-T} ubar, g2 = Y^{-T} g3, g1 = X^{-T} g2:
//     ubar_prev = ubar + lam L^T g1
//     dL/dlam  += <g1, L u> - <g1, X' du1> - <g2, Y' du2> - <g3, Z' du3>
// with X' = dX/dlam the interior rows (da, db, dc) along x (Y', Z' along y,
// z; face rows are identity and do not depend on lam).  Each CTA writes its
// partial sum of the lam term; adi_vjp_sum_kernel adds the partials in a
// fixed order (the result does not depend on scheduling).
template <typename T>
struct AdiVjpArgs {
  int nx, ny, nz;
  T lam, da, db, dc;
  const T *u, *du1, *du2, *du3, *g1, *g2, *g3;
  T *ubar;      // in: cotangent of the step's output; out: of its input
  T *partial;   // one per CTA
};

template <typename T>
__global__ void __launch_bounds__(256) adi_vjp_kernel(AdiVjpArgs<T> v) {
  __shared__ T red[8];
  const int64_t total = (int64_t)v.nx * v.ny * v.nz;
  const int64_t sx = 1, sy = v.nx, sz = (int64_t)v.nx * v.ny;
  AdiArgs<T> g = {v.nx, v.ny, v.nz, v.lam, T(0), T(1), T(0), nullptr, nullptr};
  T acc = T(0);
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(p % v.nx), j = (int)((p / v.nx) % v.ny), k = (int)(p / sz);
    const bool in = adi_inside(g, i, j, k);
    const T g1 = v.g1[p];
    // (L^T g1)_p
    T lt = in ? T(-6) * g1 : T(0);
    if (i > 0 && adi_inside(g, i - 1, j, k)) lt += v.g1[p - sx];
    if (i < v.nx - 1 && adi_inside(g, i + 1, j, k)) lt += v.g1[p + sx];
    if (j > 0 && adi_inside(g, i, j - 1, k)) lt += v.g1[p - sy];
    if (j < v.ny - 1 && adi_inside(g, i, j + 1, k)) lt += v.g1[p + sy];
    if (k > 0 && adi_inside(g, i, j, k - 1)) lt += v.g1[p - sz];
    if (k < v.nz - 1 && adi_inside(g, i, j, k + 1)) lt += v.g1[p + sz];
    v.ubar[p] += v.lam * lt;
    if (in) {
      const T lu = v.u[p - sx] + v.u[p + sx] + v.u[p - sy] + v.u[p + sy] + v.u[p - sz] +
                   v.u[p + sz] - T(6) * v.u[p];
      const T xd = v.da * v.du1[p - sx] + v.db * v.du1[p] + v.dc * v.du1[p + sx];
      const T yd = v.da * v.du2[p - sy] + v.db * v.du2[p] + v.dc * v.du2[p + sy];
      const T zd = v.da * v.du3[p - sz] + v.db * v.du3[p] + v.dc * v.du3[p + sz];
      acc += g1 * (lu - xd) - v.g2[p] * yd - v.g3[p] * zd;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    T s = T(0);
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    v.partial[blockIdx.x] = s;
  }
}

// *lbar += sum of the n partials, in a fixed order
template <typename T>
__global__ void __launch_bounds__(256) adi_vjp_sum_kernel(const T *__restrict__ partial, int n,
                                                          T *lbar) {
  __shared__ T red[256];
  T s = T(0);
  for (int q = threadIdx.x; q < n; q += 256) s += partial[q];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *lbar += red[0];
}

// ------------------------------------------------------------- launchers --
template <typename T, int M>
static cudaError_t adi_x_m(const AdiArgs<T> &g, bool stencil, bool trans, bool inc,
                           cudaStream_t st) {
  const int64_t lines = (int64_t)g.ny * g.nz;
  const dim3 grid((unsigned)((lines + 3) / 4)), block(128);
  if (stencil && !trans && !inc) return launch_pdl(adi_x_kernel<T, M, true, false>, grid, block, 0, st, g);
  if (!stencil && !trans && !inc) return launch_pdl(adi_x_kernel<T, M, false, false>, grid, block, 0, st, g);
  if (!stencil && trans && !inc) return launch_pdl(adi_x_kernel<T, M, false, true>, grid, block, 0, st, g);
  return cudaErrorInvalidValue;
}

// y/z lines: M rows per chunk, NCH chunks per line (16 lines per CTA with
// NCH = 16, else 8)
template <typename T, int M, int NCH>
static cudaError_t adi_s_m(const AdiArgs<T> &g, int axis, bool trans, bool inc, cudaStream_t st) {
  constexpr int SB = (NCH == kWarp) ? 8 : 16;
  const int ntx = (g.nx + SB - 1) / SB;
  const int other = (axis == 1) ? g.nz : g.ny;
  const dim3 grid((unsigned)((int64_t)ntx * other)), block(SB * NCH);
#define ADI_S(AX)                                                                            \
  if (!trans && !inc)                                                                        \
    return launch_pdl(adi_s_kernel<T, M, SB, NCH, AX, false, false>, grid, block, 0, st, g);  \
  if (!trans && inc)                                                                         \
    return launch_pdl(adi_s_kernel<T, M, SB, NCH, AX, false, true>, grid, block, 0, st, g);   \
  if (trans && !inc)                                                                         \
    return launch_pdl(adi_s_kernel<T, M, SB, NCH, AX, true, false>, grid, block, 0, st, g);   \
  return cudaErrorInvalidValue;
  if (axis == 1) {
    ADI_S(1)
  } else {
    ADI_S(2)
  }
#undef ADI_S
}

template <typename T>
cudaError_t adi_axis(const AdiArgs<T> &g, int axis, bool stencil, bool trans, bool inc,
                     cudaStream_t st) {
  const int n = axis == 0 ? g.nx : (axis == 1 ? g.ny : g.nz);
  if (axis == 0) {
    if (n <= 64) return adi_x_m<T, 2>(g, stencil, trans, inc, st);
    if (n <= 128) return adi_x_m<T, 4>(g, stencil, trans, inc, st);
    if (n <= 256) return adi_x_m<T, 8>(g, stencil, trans, inc, st);
    if (n <= 512) return adi_x_m<T, 16>(g, stencil, trans, inc, st);
    return cudaErrorNotSupported;
  }
  if (stencil) return cudaErrorInvalidValue;
  // 16 chunks of up to 8 rows for y lines of at most 128 rows and z lines of
  // at most 64 (per launch at 128^3: y 15.5 -> 14.3 us, z 18.5 -> 19.5 us; at
  // 64^3: y 14.4 -> 12.9, z 12.7 -> 11.7)
  if (n <= (axis == 1 ? 128 : 64)) {
    if (n <= 32) return adi_s_m<T, 2, 16>(g, axis, trans, inc, st);
    if (n <= 64) return adi_s_m<T, 4, 16>(g, axis, trans, inc, st);
    return adi_s_m<T, 8, 16>(g, axis, trans, inc, st);
  }
  if (n <= 64) return adi_s_m<T, 2, 32>(g, axis, trans, inc, st);
  if (n <= 128) return adi_s_m<T, 4, 32>(g, axis, trans, inc, st);
  if (n <= 256) return adi_s_m<T, 8, 32>(g, axis, trans, inc, st);
  if (n <= 512) return adi_s_m<T, 16, 32>(g, axis, trans, inc, st);
  return cudaErrorNotSupported;
}

template <typename T>
cudaError_t adi_lt(const AdiArgs<T> &g, const T *gin, cudaStream_t st) {
  const int64_t total = (int64_t)g.nx * g.ny * g.nz;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  adi_lt_kernel<T><<<dim3((unsigned)blocks), dim3(256), 0, st>>>(g, gin);
  return cudaGetLastError();
}

template <typename T>
cudaError_t adi_vjp(AdiVjpArgs<T> v, T *lbar, cudaStream_t st) {
  const int64_t total = (int64_t)v.nx * v.ny * v.nz;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  const Scratch sc((size_t)blocks * sizeof(T), 0, st);
  v.partial = (T *)sc.get();
  if (!v.partial) return cudaErrorMemoryAllocation;
  adi_vjp_kernel<T><<<dim3((unsigned)blocks), dim3(256), 0, st>>>(v);
  adi_vjp_sum_kernel<T><<<1, 256, 0, st>>>(v.partial, (int)blocks, lbar);
  return cudaGetLastError();
}

}  // namespace tridb200

using namespace tridb200;

static bool adi_dims_ok(int nx, int ny, int nz) {
  return nx >= 1 && ny >= 1 && nz >= 1 && nx <= 512 && ny <= 512 && nz <= 512;
}

template <typename T>
static tridStatus_t adi_solve_entry(const T *rhs, T *out, int nx, int ny, int nz, int axis,
                                    int stencil, int transpose, int inc, T lam, T ca, T cb, T cc) {
  if (!adi_dims_ok(nx, ny, nz) || axis < 0 || axis > 2 || !rhs || !out) return TRID_STATUS_INVALID_VALUE;
  if ((stencil && (axis != 0 || transpose || inc)) || (inc && (transpose || axis == 0)))
    return TRID_STATUS_INVALID_VALUE;
  AdiArgs<T> g = {nx, ny, nz, lam, ca, cb, cc, rhs, out};
  return adi_axis<T>(g, axis, stencil != 0, transpose != 0, inc != 0, current_stream()) == cudaSuccess
             ? TRID_STATUS_SUCCESS
             : TRID_STATUS_EXECUTION_FAILED;
}

template <typename T>
static tridStatus_t adi_steps_entry(T *u, T *work, int nx, int ny, int nz, int nsteps, T lam, T ca,
                                    T cb, T cc) {
  if (!adi_dims_ok(nx, ny, nz) || !u || nsteps < 0) return TRID_STATUS_INVALID_VALUE;
  const size_t npts = (size_t)nx * ny * nz;
  const cudaStream_t st = current_stream();
  const Scratch sc(work ? 0 : 2 * npts * sizeof(T), 0, st);
  if (!work) {
    work = (T *)sc.get();
    if (!work) return TRID_STATUS_ALLOC_FAILED;
  }
  T *w1 = work, *w2 = work + npts;
  for (int s = 0; s < nsteps; ++s) {
    AdiArgs<T> gx = {nx, ny, nz, lam, ca, cb, cc, u, w1};
    AdiArgs<T> gy = {nx, ny, nz, lam, ca, cb, cc, w1, w2};
    AdiArgs<T> gz = {nx, ny, nz, lam, ca, cb, cc, w2, u};
    if (adi_axis<T>(gx, 0, true, false, false, st) != cudaSuccess ||
        adi_axis<T>(gy, 1, false, false, false, st) != cudaSuccess ||
        adi_axis<T>(gz, 2, false, false, true, st) != cudaSuccess)
      return TRID_STATUS_EXECUTION_FAILED;
  }
  return TRID_STATUS_SUCCESS;
}

extern "C" tridStatus_t tridDadiSolve(const double *rhs, double *out, int nx, int ny, int nz,
                                      int axis, int stencil, int transpose, int inc, double lambda,
                                      double a, double b, double c) {
  return adi_solve_entry<double>(rhs, out, nx, ny, nz, axis, stencil, transpose, inc, lambda, a, b, c);
}
extern "C" tridStatus_t tridSadiSolve(const float *rhs, float *out, int nx, int ny, int nz,
                                      int axis, int stencil, int transpose, int inc, float lambda,
                                      float a, float b, float c) {
  return adi_solve_entry<float>(rhs, out, nx, ny, nz, axis, stencil, transpose, inc, lambda, a, b, c);
}
extern "C" tridStatus_t tridDadiSteps(double *u, double *work, int nx, int ny, int nz, int nsteps,
                                      double lambda, double a, double b, double c) {
  return adi_steps_entry<double>(u, work, nx, ny, nz, nsteps, lambda, a, b, c);
}
extern "C" tridStatus_t tridSadiSteps(float *u, float *work, int nx, int ny, int nz, int nsteps,
                                      float lambda, float a, float b, float c) {
  return adi_steps_entry<float>(u, work, nx, ny, nz, nsteps, lambda, a, b, c);
}
extern "C" tridStatus_t tridDadiLaplacianT(const double *g, double *out, int nx, int ny, int nz,
                                           double lambda) {
  if (!adi_dims_ok(nx, ny, nz) || !g || !out) return TRID_STATUS_INVALID_VALUE;
  AdiArgs<double> a = {nx, ny, nz, lambda, 0.0, 1.0, 0.0, nullptr, out};
  return adi_lt<double>(a, g, current_stream()) == cudaSuccess ? TRID_STATUS_SUCCESS
                                                               : TRID_STATUS_EXECUTION_FAILED;
}

extern "C" tridStatus_t tridDadiStepVjp(const double *u, const double *du1, const double *du2,
                                        const double *du3, const double *g1, const double *g2,
                                        const double *g3, double *ubar, int nx, int ny, int nz,
                                        double lambda, double da, double db, double dc,
                                        double *lbar) {
  if (!adi_dims_ok(nx, ny, nz) || !u || !du1 || !du2 || !du3 || !g1 || !g2 || !g3 || !ubar ||
      !lbar)
    return TRID_STATUS_INVALID_VALUE;
  AdiVjpArgs<double> v = {nx, ny, nz, lambda, da, db, dc, u, du1, du2, du3, g1, g2, g3, ubar,
                          nullptr};
  const cudaError_t e = adi_vjp<double>(v, lbar, current_stream());
  if (e == cudaErrorMemoryAllocation) return TRID_STATUS_ALLOC_FAILED;
  return e == cudaSuccess ? TRID_STATUS_SUCCESS : TRID_STATUS_EXECUTION_FAILED;
}
