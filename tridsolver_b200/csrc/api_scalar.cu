// Scalar strided-batch C ABI (9-argument form over device pointers) and the
// library's host runtime: per-thread stream and method override, per-stream
// scratch, tuning table, argument validation and dispatch.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "dispatch.cuh"

namespace tridb200 {

// ------------------------------------------------------------------ state --
static thread_local cudaStream_t tl_stream = nullptr;
static thread_local MethodChoice tl_force = {0, 0, 0};

cudaStream_t current_stream() { return tl_stream; }

struct ScratchBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
};
constexpr int kScratchLevels = 5;
constexpr int kSplitScratch = kScratchLevels - 1;  // split finish (the solves recurse below it)
// One buffer per (device, stream, nesting level): calls on different streams
// may run at the same time on the GPU, so they never share scratch.  The
// per-thread default stream is one stream per thread under a single handle,
// so for it the calling thread is part of the key.
using ScratchKey = std::tuple<int, uintptr_t, std::thread::id, int>;
static std::mutex g_scratch_mu;
static std::map<ScratchKey, ScratchBuf> g_scratch;

static void *persistent_scratch(size_t bytes, int level, cudaStream_t st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  const ScratchKey key{dev, (uintptr_t)st,
                       st == cudaStreamPerThread ? std::this_thread::get_id() : std::thread::id(),
                       level};
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  ScratchBuf &s = g_scratch[key];
  if (s.bytes >= bytes) return s.ptr;
  if (s.ptr) {
    // only work queued on this stream may still read the old buffer
    if (cudaStreamSynchronize(st) != cudaSuccess) return nullptr;
    cudaFree(s.ptr);
    s.ptr = nullptr;
    s.bytes = 0;
  }
  void *p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  s.ptr = p;
  s.bytes = bytes;
  return p;
}

Scratch::Scratch(size_t bytes, int level, cudaStream_t stream) : stream_(stream) {
  if (bytes == 0 || level < 0 || level >= kScratchLevels) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream_, &cs) != cudaSuccess) {
    cudaGetLastError();
    cs = cudaStreamCaptureStatusNone;
  }
  if (cs == cudaStreamCaptureStatusNone) {
    ptr_ = persistent_scratch(bytes, level, stream_);
    return;
  }
  // captured: allocate and free in stream order (graph memory nodes)
  if (cudaMallocAsync(&ptr_, bytes, stream_) != cudaSuccess) {
    cudaGetLastError();
    ptr_ = nullptr;
    return;
  }
  stream_ordered_ = true;
}

Scratch::~Scratch() {
  if (stream_ordered_ && ptr_) cudaFreeAsync(ptr_, stream_);
}

// Frees every scratch buffer of the current device (after the work queued on
// it has finished).
static tridStatus_t release_scratch() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return TRID_STATUS_EXECUTION_FAILED;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (cudaDeviceSynchronize() != cudaSuccess) return TRID_STATUS_EXECUTION_FAILED;
  for (auto it = g_scratch.begin(); it != g_scratch.end();) {
    if (std::get<0>(it->first) == dev) {
      if (it->second.ptr) cudaFree(it->second.ptr);
      it = g_scratch.erase(it);
    } else {
      ++it;
    }
  }
  return TRID_STATUS_SUCCESS;
}

static std::mutex g_err_mu;
static std::vector<unsigned *> g_err;  // indexed by device

unsigned *device_error_flags() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(g_err_mu);
  if ((int)g_err.size() <= dev) g_err.resize(dev + 1, nullptr);
  if (!g_err[dev]) {
    unsigned *p = nullptr;
    if (cudaMalloc(&p, sizeof(unsigned)) != cudaSuccess || cudaMemset(p, 0, sizeof(unsigned)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    g_err[dev] = p;
  }
  return g_err[dev];
}

unsigned *device_error_flags_if_present() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(g_err_mu);
  return (int)g_err.size() > dev ? g_err[dev] : nullptr;
}

struct TuneEntry {
  int dtype_bytes, axis, nmax, method, chunk, spc;
};
static std::mutex g_tune_mu;
static std::vector<TuneEntry> g_tune;

static tridStatus_t parse_tuning_table(const char *path, std::vector<TuneEntry> &table) {
  FILE *f = fopen(path, "r");
  if (!f) return TRID_STATUS_INVALID_VALUE;
  char line[256];
  while (fgets(line, sizeof(line), f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    char dt[16];
    TuneEntry e;
    if (sscanf(line, "%15s %d %d %d %d %d", dt, &e.axis, &e.nmax, &e.method, &e.chunk, &e.spc) !=
        6) {
      fclose(f);
      return TRID_STATUS_INVALID_VALUE;
    }
    e.dtype_bytes = (strcmp(dt, "f64") == 0) ? 8 : (strcmp(dt, "f32") == 0 ? 4 : 0);
    const bool chunk_ok = e.chunk == 0 || e.chunk == 2 || e.chunk == 4 || e.chunk == 8 || e.chunk == 16;
    const bool spc_ok = e.spc == 0 || e.spc == 4 || e.spc == 8 || e.spc == 16 || e.spc == 32;
    // axis class 4: the variable-length batch's length buckets (method 2,
    // chunk 2/4/8 for the lengths up to nmax)
    const bool vl_ok = e.axis != 4 || (e.method == 2 && e.chunk >= 2 && e.chunk <= 8);
    if (e.dtype_bytes == 0 || e.method < 1 || e.method > 6 || e.method == 4 || e.method == 5 ||
        e.axis < 0 || e.axis > 4 || !vl_ok ||
        !chunk_ok || !spc_ok) {
      fclose(f);
      return TRID_STATUS_INVALID_VALUE;
    }
    table.push_back(e);
  }
  fclose(f);
  std::stable_sort(table.begin(), table.end(),
                   [](const TuneEntry &x, const TuneEntry &y) { return x.nmax < y.nmax; });
  return TRID_STATUS_SUCCESS;
}

static std::once_flag g_env_tune_once;
static void load_env_tuning() {
  const char *p = getenv("TRID_B200_TUNING");
  if (!p || !*p) return;
  std::vector<TuneEntry> table;
  if (parse_tuning_table(p, table) == TRID_STATUS_SUCCESS) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.swap(table);
  }
}

// ------------------------------------------------------- method selection --
static int chunk_for(int n, int dtype_bytes) {
  (void)dtype_bytes;
  if (n <= 64) return 2;
  if (n <= 128) return 4;
  if (n <= 256) return 8;
  if (n <= 512) return 16;
  return 0;  // too long for a register-resident partition
}

// Length buckets of the variable-length batch: systems of at most m2max rows
// take 2 rows per lane, at most m4max 4, longer ones 8 (64 / 128 built in).
// A tuning table's axis-class-4 entries (lengths up to nmax use `chunk`)
// move the cut-offs: the leading run of chunk-2 entries sets m2max (at most
// 64 rows fit), the chunk-4 entries after it m4max (at most 128).
void varlen_buckets(int dtype_bytes, int &m2max, int &m4max) {
  std::call_once(g_env_tune_once, load_env_tuning);
  m2max = 64;
  m4max = 128;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  bool any = false;
  int a2 = 0, a4 = 0, stage = 2;
  for (const TuneEntry &e : g_tune) {  // sorted by nmax
    if (e.dtype_bytes != dtype_bytes || e.axis != 4) continue;
    any = true;
    if (e.chunk < stage) continue;  // not monotone: ignored
    stage = e.chunk;
    if (e.chunk == 2) a2 = std::min(e.nmax, 64);
    if (e.chunk == 4) a4 = std::min(e.nmax, 128);
  }
  if (any) {
    m2max = a2;
    m4max = std::max(a2, a4);
  }
}

MethodChoice choose_method(int dtype_bytes, int axis, int n, int opt_hint) {
  std::call_once(g_env_tune_once, load_env_tuning);
  MethodChoice m = tl_force;
  if (m.method == 0 && opt_hint != 0) {
    // reference opts: 1/2 = plain Thomas kernels, 3/4 = Thomas-PCR hybrid
    if (opt_hint == 1 || opt_hint == 2) m.method = 1;
    if (opt_hint == 3 || opt_hint == 4) m.method = 2;
  }
  if (m.method == 0) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const TuneEntry &e : g_tune) {
      if (e.dtype_bytes == dtype_bytes && e.axis == axis && n <= e.nmax) {
        m = {e.method, e.chunk, e.spc};
        break;
      }
    }
  }
  if (m.method == 0) {
    // built-in defaults, from the B200 sweeps of tridsolver_b200.autotune:
    // TMA staging on axis 0; on strided axes the streamed kernel with a full
    // 128-byte line of systems per tile (16 FP64 / 32 FP32), fastest at every
    // row stride measured (DRAM serves 64-byte row segments far slower once
    // the stride reaches 64 KiB).  Where it does not apply (more than 256
    // rows, a narrow or misaligned axis 0) the narrow-tile kernel that was
    // best for the class takes over: plain coalesced loads with 8 systems
    // per CTA up to 64 KiB strides, TMA tiles of 8 systems up to 1 MiB, plain
    // loads with 16 systems beyond that and in FP32.  Long axis-0 systems
    // take one CTA each, longer ones the blocked partition (blocks of
    // 32*chunk rows).
    if (axis == 0) {
      // systems of at most 64 rows: plain coalesced loads beat the TMA
      // staging (sweep: 1.28-1.45x at n = 32 and 64, FP64 and FP32)
      m.method = n <= 64 ? 3 : 2;
    } else {
      m.method = 2;
      m.spc = 128 / dtype_bytes;
      if (dtype_bytes == 4 || axis == 3) {
        m.fb_method = 3;
        m.fb_spc = 16;
      } else {
        m.fb_method = (axis == 1) ? 3 : 2;
        m.fb_spc = 8;
      }
      // 257..512 rows (past the streamed tiles): the narrow plain-load tiles
      // that won the sweep (FP64 class 1: 4 systems per CTA, 1.14x; class 2:
      // 16, 1.11x; FP32 class 1: 8, 1.19x)
      if (n > 256 && n <= 512 && axis <= 2) {
        m.fb_method = 3;
        m.fb_spc = dtype_bytes == 8 ? (axis == 1 ? 4 : 16) : (axis == 1 ? 8 : 16);
      }
    }
  }
  if (m.method >= 2) {
    const int need = chunk_for(n, dtype_bytes);
    if (need == 0) {
      // long system: blocks of 256 rows (FP32 along axis 0: 512, which
      // won the B200 sweep there, 2,048 x 65,536 FP32 0.134 ms against 0.137)
      if (m.chunk == 0) m.chunk = (dtype_bytes == 4 && axis == 0) ? 16 : 8;
    } else if (m.chunk < need) {
      m.chunk = need;
    }
    if (m.spc == 0) m.spc = 8;
  }
  return m;
}

// ------------------------------------------------------------- validation --
tridStatus_t make_geom(int ndim, int solvedim, const int *dims, const int *const pads[5],
                       bool inc, Geom &g) {
  if (ndim < 1 || ndim > kMaxDim || solvedim < 0 || solvedim >= ndim || dims == nullptr)
    return TRID_STATUS_INVALID_VALUE;
  for (int q = 0; q < 5; ++q)
    if (pads[q] == nullptr && (q < 4 || inc)) return TRID_STATUS_INVALID_VALUE;
  int64_t total = 1;
  for (int k = 0; k < ndim; ++k) {
    if (dims[k] < 0) return TRID_STATUS_INVALID_VALUE;
    for (int q = 0; q < 5; ++q)
      if (pads[q] && (q < 4 || inc) && pads[q][k] < dims[k]) return TRID_STATUS_INVALID_VALUE;
    total *= (dims[k] > 0 ? dims[k] : 1);
    if (total > ((int64_t)1 << 46)) return TRID_STATUS_INVALID_VALUE;
  }
  memset(&g, 0, sizeof(g));
  g.n = dims[solvedim];
  g.nod = 0;
  g.nsys = 1;
  for (int k = 0; k < ndim; ++k) {
    if (k == solvedim) continue;
    g.odims[g.nod] = dims[k];
    g.nsys *= dims[k];
    g.nod++;
  }
  g.fastdiv = g.nsys < ((int64_t)1 << 32);
  for (int k = 0; k < g.nod; ++k) fastdiv_setup((uint32_t)g.odims[k], g.dmul[k], g.dshift[k]);
  for (int q = 0; q < 5; ++q) {
    if (!pads[q] || (q == 4 && !inc)) continue;
    int64_t cum = 1;
    int o = 0;
    for (int k = 0; k < ndim; ++k) {
      if (k == solvedim)
        g.stride[q] = cum;
      else
        g.ocum[q][o++] = cum;
      cum *= pads[q][k];
    }
  }
  return TRID_STATUS_SUCCESS;
}

template <typename T>
static bool aligned_ptr(const T *p) {
  return p != nullptr && ((uintptr_t)p % sizeof(T)) == 0;
}

template <typename T, int INC>
static tridStatus_t solve_level(const T *a, const T *b, const T *c, T *d, T *u, int ndim,
                                int solvedim, const int *dims, const int *const pads[5],
                                const int *opts, int sync, int level);

// Blocked partition for any length (and the adjoint): block reduction ->
// block system solved recursively at the next scratch level -> finish.
template <typename T, int MODE>
static tridStatus_t run_general(const Geom &g, GenArgs<T> A, int axis, int chunk, int spc,
                                int level, cudaStream_t stream) {
  const int B = 32 * chunk;
  const int64_t nblk = (g.n + B - 1) / B;
  if (nblk > 0x3fffffff || g.nsys > 0x7fffffff) return TRID_STATUS_INVALID_VALUE;
  A.nblk = (int)nblk;
  const int ax = axis == 0 ? 0 : 1;
  if (nblk == 1) {
    return launch_general_phase<T, MODE>(g, A, ax, chunk, spc, kGenSingle, stream) == cudaSuccess
               ? TRID_STATUS_SUCCESS
               : TRID_STATUS_EXECUTION_FAILED;
  }
  const int64_t len = g.nsys * 2 * nblk;
  const Scratch sc((size_t)4 * len * sizeof(T), level, stream);
  T *red = (T *)sc.get();
  if (!red) return TRID_STATUS_ALLOC_FAILED;
  A.red = red;
  if (launch_general_phase<T, MODE>(g, A, ax, chunk, spc, kGenReduce, stream) != cudaSuccess)
    return TRID_STATUS_EXECUTION_FAILED;
  // block system: nsys contiguous systems of 2*nblk rows, solution into its d
  int bd[2] = {(int)(2 * nblk), (int)g.nsys};
  const int *bp[5] = {bd, bd, bd, bd, bd};
  const tridStatus_t st = solve_level<T, 0>(red, red + len, red + 2 * len, red + 3 * len, nullptr,
                                            2, 0, bd, bp, nullptr, 0, level + 1);
  if (st != TRID_STATUS_SUCCESS) return st;
  A.bsol = red + 3 * len;
  return launch_general_phase<T, MODE>(g, A, ax, chunk, spc, kGenFinish, stream) == cudaSuccess
             ? TRID_STATUS_SUCCESS
             : TRID_STATUS_EXECUTION_FAILED;
}

static int axis_class(const Geom &g, int solvedim, int elem_bytes) {
  // 0 = unit stride inside a system, 1 = strided with a row stride of at most
  // 64 KiB, 2 = up to 1 MiB (the outermost axis of a big cube, where DRAM-page
  // and TLB locality differ), 3 = larger (every row in its own 2 MiB page)
  if (solvedim == 0) return 0;
  const int64_t bytes = g.stride[kD] * (int64_t)elem_bytes;
  return bytes <= 65536 ? 1 : (bytes <= (1 << 20) ? 2 : 3);
}

// Axis-0 systems solved whole by one CTA each (method 6, and the default up
// to 4096 rows).  cudaErrorNotSupported when it does not apply.
template <typename T, int MODE>
static cudaError_t launch_x_whole(const Geom &g, const XArgs<T> &A, const MethodChoice &m,
                                  cudaStream_t st) {
  if (g.n <= 4096) return launch_xcta<T, MODE>(g, A, m.method == 6 ? m.chunk : 0, st);
  return cudaErrorNotSupported;
}

template <typename T, int INC>
static tridStatus_t solve_level(const T *a, const T *b, const T *c, T *d, T *u, int ndim,
                                int solvedim, const int *dims, const int *const pads[5],
                                const int *opts, int sync, int level) {
  Geom g;
  const tridStatus_t st = make_geom(ndim, solvedim, dims, pads, INC != 0, g);
  if (st != TRID_STATUS_SUCCESS) return st;
  if (!aligned_ptr(a) || !aligned_ptr(b) || !aligned_ptr(c) || !aligned_ptr(d))
    return TRID_STATUS_INVALID_VALUE;
  if (INC && !aligned_ptr(u)) return TRID_STATUS_INVALID_VALUE;
  const int opt = opts ? opts[solvedim] : 0;
  if (opt < 0 || opt > 5) return TRID_STATUS_INVALID_VALUE;
  if (g.n == 0 || g.nsys == 0) return TRID_STATUS_SUCCESS;
  if (level >= kScratchLevels) return TRID_STATUS_INTERNAL_ERROR;

  const cudaStream_t stream = current_stream();
  const int axis = axis_class(g, solvedim, (int)sizeof(T));
  const MethodChoice m = choose_method((int)sizeof(T), axis, g.n, opt);
  const bool fits = g.n <= 32 * m.chunk;
  cudaError_t e = cudaErrorNotSupported;
  if (m.method >= 2 && axis == 0 && (!fits || m.method == 6) &&
             (e = launch_x_whole<T, INC ? kXcFwdInc : kXcFwd>(
                  g, XArgs<T>{a, b, c, d, nullptr, nullptr, INC ? u : d, nullptr, nullptr, nullptr,
                              nullptr},
                  m, stream)) != cudaErrorNotSupported) {
    // one CTA per system: done (or failed) above
  } else if (m.method >= 2 && !fits) {
    GenArgs<T> A = {};
    A.a = a;
    A.b = b;
    A.c = c;
    A.rhs = d;
    A.out = INC ? u : d;
    const int spc = narrow_spc(m);
    const tridStatus_t s2 = INC ? run_general<T, kGenFwdInc>(g, A, axis, m.chunk, spc, level, stream)
                                : run_general<T, kGenFwd>(g, A, axis, m.chunk, spc, level, stream);
    if (s2 != TRID_STATUS_SUCCESS) return s2;
    e = cudaSuccess;
  } else if (m.method >= 2) {
    if (axis == 0) {
      if (m.method == 2) {
        unsigned *err = device_error_flags();
        if (!err) return TRID_STATUS_ALLOC_FAILED;
        e = launch_xsolve_tma<T, INC>(g, pads, ndim, a, b, c, d, u, m.chunk, err, stream);
        // rows off the TMA grid (pads[0] not a multiple of the 128-byte
        // row): past 128 rows the one-CTA kernel beats the plain
        // one-warp-per-system loads (B200 sweep, FP64 / FP32: 300 rows
        // 5.19 / 3.49 TB/s against 2.10 / 1.99, 500 rows 6.56 / 5.70 against
        // 2.14 / 1.97; at 100 rows the plain kernel wins, 5.02 / 4.68 against
        // 4.23 / 3.35)
        if (e == cudaErrorNotSupported && g.n > 128)
          e = launch_xcta<T, INC ? kXcFwdInc : kXcFwd>(
              g, XArgs<T>{a, b, c, d, nullptr, nullptr, INC ? u : d, nullptr, nullptr, nullptr,
                          nullptr},
              0, stream);
      }
      if (e == cudaErrorNotSupported) e = launch_xsolve<T, INC>(g, a, b, c, d, u, m.chunk, stream);
    } else {
      if (m.method == 2) {
        unsigned *err = device_error_flags();
        if (!err) return TRID_STATUS_ALLOC_FAILED;
        e = launch_strided_part_tma<T, INC>(g, dims, pads, ndim, solvedim, a, b, c, d, u, m.chunk,
                                            m.spc, true, err, stream);
        if (e == cudaErrorNotSupported && m.fb_method == 2)
          e = launch_strided_part_tma<T, INC>(g, dims, pads, ndim, solvedim, a, b, c, d, u,
                                              m.chunk, m.fb_spc, true, err, stream);
      }
      if (e == cudaErrorNotSupported)
        e = launch_strided<T, INC>(g, a, b, c, d, u, m.chunk, narrow_spc(m), stream);
    }
  } else {
    // Thomas with c'/d' in scratch, in batches of systems bounded to ~1 GiB
    const size_t per_sys = (size_t)2 * g.n * sizeof(T);
    int64_t ws = (int64_t)(((size_t)1 << 30) / per_sys);
    ws = std::max<int64_t>(1, std::min<int64_t>(ws, g.nsys));
    const Scratch sc(per_sys * (size_t)ws, level, stream);
    T *work = (T *)sc.get();
    if (!work) return TRID_STATUS_ALLOC_FAILED;
    e = launch_generic<T, INC>(g, a, b, c, d, u, work, ws, stream);
  }
  if (e != cudaSuccess) return TRID_STATUS_EXECUTION_FAILED;
  if (sync == 1 && cudaStreamSynchronize(stream) != cudaSuccess) return TRID_STATUS_EXECUTION_FAILED;
  return TRID_STATUS_SUCCESS;
}

template <typename T, int INC>
tridStatus_t solve_strided_batch(const T *a, const T *b, const T *c, T *d, T *u, int ndim,
                                 int solvedim, const int *dims, const int *const pads[5],
                                 const int *opts, int sync) {
  return solve_level<T, INC>(a, b, c, d, u, ndim, solvedim, dims, pads, opts, sync, 0);
}

// Adjoint of the strided-batch solve (one pads array for every operand).
template <typename T>
tridStatus_t solve_adjoint(const T *a, const T *b, const T *c, const T *u, const T *w, T *ga,
                           T *gb, T *gc, T *gd, int ndim, int solvedim, const int *dims,
                           const int *pads) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  Geom g;
  const tridStatus_t st = make_geom(ndim, solvedim, dims, p, true, g);
  if (st != TRID_STATUS_SUCCESS) return st;
  if (!aligned_ptr(a) || !aligned_ptr(b) || !aligned_ptr(c) || !aligned_ptr(u) || !aligned_ptr(w))
    return TRID_STATUS_INVALID_VALUE;
  for (const T *o : {(const T *)ga, (const T *)gb, (const T *)gc, (const T *)gd})
    if (o && ((uintptr_t)o % sizeof(T)) != 0) return TRID_STATUS_INVALID_VALUE;
  if (g.n == 0 || g.nsys == 0) return TRID_STATUS_SUCCESS;
  const cudaStream_t stream = current_stream();
  const int axis = axis_class(g, solvedim, (int)sizeof(T));
  MethodChoice m = choose_method((int)sizeof(T), axis, g.n, 0);
  if (m.chunk == 0) m.chunk = 8;
  if (m.spc == 0) m.spc = 8;
  if (axis == 0 && (g.n > 64 || m.method == 6)) {
    const cudaError_t e = launch_x_whole<T, kXcAdj>(
        g, XArgs<T>{a, b, c, nullptr, w, u, nullptr, ga, gb, gc, gd}, m, stream);
    if (e != cudaErrorNotSupported)
      return e == cudaSuccess ? TRID_STATUS_SUCCESS : TRID_STATUS_EXECUTION_FAILED;
  }
  GenArgs<T> A = {};
  A.a = a;
  A.b = b;
  A.c = c;
  A.rhs = w;
  A.usol = u;
  A.ga = ga;
  A.gb = gb;
  A.gc = gc;
  A.gd = gd;
  return run_general<T, kGenAdj>(g, A, axis, m.chunk, narrow_spc(m), 0, stream);
}
// Forward solve and adjoint of the linear loss <w, x> in one pass where a
// one-warp or one-CTA-per-system kernel applies (axis 0, n <= 4096); otherwise the
// forward solve followed by the adjoint.
template <typename T>
tridStatus_t solve_fwd_adj(const T *a, const T *b, const T *c, const T *d, const T *w, T *x,
                           T *ga, T *gb, T *gc, T *gd, int ndim, int solvedim, const int *dims,
                           const int *pads) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  Geom g;
  const tridStatus_t st = make_geom(ndim, solvedim, dims, p, true, g);
  if (st != TRID_STATUS_SUCCESS) return st;
  if (!aligned_ptr(a) || !aligned_ptr(b) || !aligned_ptr(c) || !aligned_ptr(d) ||
      !aligned_ptr(w) || !aligned_ptr((const T *)x))
    return TRID_STATUS_INVALID_VALUE;
  for (const T *o : {(const T *)ga, (const T *)gb, (const T *)gc, (const T *)gd})
    if (o && ((uintptr_t)o % sizeof(T)) != 0) return TRID_STATUS_INVALID_VALUE;
  if (g.n == 0 || g.nsys == 0) return TRID_STATUS_SUCCESS;
  const cudaStream_t stream = current_stream();
  const int axis = axis_class(g, solvedim, (int)sizeof(T));
  MethodChoice m = choose_method((int)sizeof(T), axis, g.n, 0);
  if (m.chunk == 0) m.chunk = 8;
  if (m.spc == 0) m.spc = 8;
  if (axis == 0) {
    const cudaError_t e = launch_x_whole<T, kXcFused>(
        g, XArgs<T>{a, b, c, d, w, nullptr, x, ga, gb, gc, gd}, m, stream);
    if (e != cudaErrorNotSupported)
      return e == cudaSuccess ? TRID_STATUS_SUCCESS : TRID_STATUS_EXECUTION_FAILED;
  }
  // two passes: x = A^{-1} d (blocked partition, d left intact), then the
  // adjoint at x
  GenArgs<T> A = {};
  A.a = a;
  A.b = b;
  A.c = c;
  A.rhs = d;
  A.out = x;
  const tridStatus_t s1 = run_general<T, kGenFwd>(g, A, axis, m.chunk, narrow_spc(m), 0, stream);
  if (s1 != TRID_STATUS_SUCCESS) return s1;
  return solve_adjoint<T>(a, b, c, x, w, ga, gb, gc, gd, ndim, solvedim, dims, pads);
}
// Out-of-place forward solve x = A^{-1} d (d left intact, one pads array
// for every operand): the one-CTA kernel on axis 0 up to 4096 rows, the
// blocked partition (which reads the right-hand side and writes the
// solution separately) elsewhere; x == d is the ordinary in-place solve.
template <typename T>
static tridStatus_t solve_out(const T *a, const T *b, const T *c, const T *d, T *x, int ndim,
                              int solvedim, const int *dims, const int *pads) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  if (x == d) return solve_level<T, 0>(a, b, c, x, nullptr, ndim, solvedim, dims, p, nullptr, 0, 0);
  Geom g;
  const tridStatus_t st = make_geom(ndim, solvedim, dims, p, true, g);
  if (st != TRID_STATUS_SUCCESS) return st;
  if (!aligned_ptr(a) || !aligned_ptr(b) || !aligned_ptr(c) || !aligned_ptr(d) ||
      !aligned_ptr((const T *)x))
    return TRID_STATUS_INVALID_VALUE;
  if (g.n == 0 || g.nsys == 0) return TRID_STATUS_SUCCESS;
  const cudaStream_t stream = current_stream();
  const int axis = axis_class(g, solvedim, (int)sizeof(T));
  MethodChoice m = choose_method((int)sizeof(T), axis, g.n, 0);
  if (m.chunk == 0) m.chunk = 8;
  if (m.spc == 0) m.spc = 8;
  if (axis == 0 && m.method != 1) {
    const cudaError_t e = launch_x_whole<T, kXcFwd>(
        g, XArgs<T>{a, b, c, d, nullptr, nullptr, x, nullptr, nullptr, nullptr, nullptr}, m,
        stream);
    if (e != cudaErrorNotSupported)
      return e == cudaSuccess ? TRID_STATUS_SUCCESS : TRID_STATUS_EXECUTION_FAILED;
  }
  GenArgs<T> A = {};
  A.a = a;
  A.b = b;
  A.c = c;
  A.rhs = d;
  A.out = x;
  return run_general<T, kGenFwd>(g, A, axis, m.chunk, narrow_spc(m), 0, stream);
}

template tridStatus_t solve_fwd_adj<float>(const float *, const float *, const float *,
                                           const float *, const float *, float *, float *, float *,
                                           float *, float *, int, int, const int *, const int *);
template tridStatus_t solve_fwd_adj<double>(const double *, const double *, const double *,
                                            const double *, const double *, double *, double *,
                                            double *, double *, double *, int, int, const int *,
                                            const int *);

// Systems split along the solve axis across ranks (reference:
// scalar/src/cuda/trid_cuda_mpi.cu:473-583 and include/trid_mpi_cuda.hpp):
// this rank's slab reduced to six boundary numbers per system, and the finish
// from the slabs of every rank gathered in rank order.  The exchange between
// the two is the caller's (tridsolver_b200/mpi.py: an all-gather over the
// ranks of the solve dimension).
template <typename T>
static tridStatus_t split_reduce(const T *a, const T *b, const T *c, const T *d, int ndim,
                                 int solvedim, const int *dims, const int *pads, double *bnd) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  Geom g;
  const tridStatus_t st = make_geom(ndim, solvedim, dims, p, false, g);
  if (st != TRID_STATUS_SUCCESS) return st;
  if (!aligned_ptr(a) || !aligned_ptr(b) || !aligned_ptr(c) || !aligned_ptr(d) || !bnd ||
      ((uintptr_t)bnd % sizeof(double)) != 0)
    return TRID_STATUS_INVALID_VALUE;
  if (g.nsys == 0) return TRID_STATUS_SUCCESS;
  if (g.n < 2) return TRID_STATUS_INVALID_VALUE;  // one row: both ends are the same unknown
  return launch_split_reduce<T>(g, a, b, c, d, bnd, current_stream()) == cudaSuccess
             ? TRID_STATUS_SUCCESS
             : TRID_STATUS_EXECUTION_FAILED;
}

template <typename T, int INC>
static tridStatus_t split_finish(const T *a, const T *b, const T *c, T *d, T *u, int ndim,
                                 int solvedim, const int *dims, const int *pads,
                                 const double *bnd_all, int nranks, int rank) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  Geom g;
  tridStatus_t st = make_geom(ndim, solvedim, dims, p, INC != 0, g);
  if (st != TRID_STATUS_SUCCESS) return st;
  if (!aligned_ptr(a) || !aligned_ptr(b) || !aligned_ptr(c) || !aligned_ptr(d) ||
      (INC && !aligned_ptr(u)) || !bnd_all || ((uintptr_t)bnd_all % sizeof(double)) != 0 ||
      nranks < 1 || rank < 0 || rank >= nranks)
    return TRID_STATUS_INVALID_VALUE;
  if (g.nsys == 0) return TRID_STATUS_SUCCESS;
  if (g.n < 2) return TRID_STATUS_INVALID_VALUE;
  const cudaStream_t stream = current_stream();
  // Inc leaves d as it was: the patched entries come back
  const Scratch sc(INC ? (size_t)2 * g.nsys * sizeof(T) : 0, kSplitScratch, stream);
  T *saved = (T *)sc.get();
  if (INC && !saved) return TRID_STATUS_ALLOC_FAILED;
  if (launch_split_patch<T>(g, a, c, d, bnd_all, nranks, rank, saved, stream) != cudaSuccess)
    return TRID_STATUS_EXECUTION_FAILED;
  st = solve_level<T, INC>(a, b, c, d, u, ndim, solvedim, dims, p, nullptr, 0, 0);
  if (INC && launch_split_restore<T>(g, d, saved, stream) != cudaSuccess)
    return TRID_STATUS_EXECUTION_FAILED;
  return st;
}

template tridStatus_t solve_adjoint<float>(const float *, const float *, const float *,
                                           const float *, const float *, float *, float *,
                                           float *, float *, int, int, const int *, const int *);
template tridStatus_t solve_adjoint<double>(const double *, const double *, const double *,
                                            const double *, const double *, double *, double *,
                                            double *, double *, int, int, const int *,
                                            const int *);

template tridStatus_t solve_strided_batch<float, 0>(const float *, const float *, const float *,
                                                    float *, float *, int, int, const int *,
                                                    const int *const[5], const int *, int);
template tridStatus_t solve_strided_batch<float, 1>(const float *, const float *, const float *,
                                                    float *, float *, int, int, const int *,
                                                    const int *const[5], const int *, int);
template tridStatus_t solve_strided_batch<double, 0>(const double *, const double *,
                                                     const double *, double *, double *, int, int,
                                                     const int *, const int *const[5],
                                                     const int *, int);
template tridStatus_t solve_strided_batch<double, 1>(const double *, const double *,
                                                     const double *, double *, double *, int, int,
                                                     const int *, const int *const[5],
                                                     const int *, int);

}  // namespace tridb200

using namespace tridb200;

// ---------------------------------------------------------------- C ABI --
#ifndef TRID_CUDACOMPAT
extern "C" tridStatus_t tridSmtsvStridedBatch(const float *a, const float *b, const float *c,
                                              float *d, float *u, int ndim, int solvedim,
                                              int *dims, int *pads) {
  (void)u;
  const int *p[5] = {pads, pads, pads, pads, pads};
  return solve_strided_batch<float, 0>(a, b, c, d, nullptr, ndim, solvedim, dims, p, nullptr, 0);
}
extern "C" tridStatus_t tridDmtsvStridedBatch(const double *a, const double *b, const double *c,
                                              double *d, double *u, int ndim, int solvedim,
                                              int *dims, int *pads) {
  (void)u;
  const int *p[5] = {pads, pads, pads, pads, pads};
  return solve_strided_batch<double, 0>(a, b, c, d, nullptr, ndim, solvedim, dims, p, nullptr, 0);
}
extern "C" tridStatus_t tridSmtsvStridedBatchInc(const float *a, const float *b, const float *c,
                                                 float *d, float *u, int ndim, int solvedim,
                                                 int *dims, int *pads) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  return solve_strided_batch<float, 1>(a, b, c, d, u, ndim, solvedim, dims, p, nullptr, 0);
}
extern "C" tridStatus_t tridDmtsvStridedBatchInc(const double *a, const double *b,
                                                 const double *c, double *d, double *u, int ndim,
                                                 int solvedim, int *dims, int *pads) {
  const int *p[5] = {pads, pads, pads, pads, pads};
  return solve_strided_batch<double, 1>(a, b, c, d, u, ndim, solvedim, dims, p, nullptr, 0);
}
#endif

#define TRID_PADDED(NAME, T, INC)                                                              \
  extern "C" tridStatus_t NAME(const T *a, const int *a_pads, const T *b, const int *b_pads,   \
                               const T *c, const int *c_pads, T *d, const int *d_pads, T *u,   \
                               const int *u_pads, int ndim, int solvedim, int *dims,           \
                               int *opts, int sync) {                                          \
    const int *p[5] = {a_pads, b_pads, c_pads, d_pads, INC ? u_pads : d_pads};                 \
    return solve_strided_batch<T, INC>(a, b, c, d, INC ? u : nullptr, ndim, solvedim, dims, p, \
                                       opts, sync);                                            \
  }
TRID_PADDED(tridDmtsvStridedBatchPadded, double, 0)
TRID_PADDED(tridDmtsvStridedBatchPaddedInc, double, 1)
TRID_PADDED(tridSmtsvStridedBatchPadded, float, 0)
TRID_PADDED(tridSmtsvStridedBatchPaddedInc, float, 1)

extern "C" tridStatus_t tridDmtsvStridedBatchAdjoint(const double *a, const double *b,
                                                     const double *c, const double *u,
                                                     const double *w, double *da, double *db,
                                                     double *dc, double *dd, int ndim,
                                                     int solvedim, int *dims, int *pads) {
  return solve_adjoint<double>(a, b, c, u, w, da, db, dc, dd, ndim, solvedim, dims, pads);
}

extern "C" tridStatus_t tridSmtsvStridedBatchAdjoint(const float *a, const float *b,
                                                     const float *c, const float *u,
                                                     const float *w, float *da, float *db,
                                                     float *dc, float *dd, int ndim, int solvedim,
                                                     int *dims, int *pads) {
  return solve_adjoint<float>(a, b, c, u, w, da, db, dc, dd, ndim, solvedim, dims, pads);
}

extern "C" tridStatus_t tridDmtsvStridedBatchOut(const double *a, const double *b,
                                                 const double *c, const double *d, double *x,
                                                 int ndim, int solvedim, int *dims, int *pads) {
  return solve_out<double>(a, b, c, d, x, ndim, solvedim, dims, pads);
}
extern "C" tridStatus_t tridSmtsvStridedBatchOut(const float *a, const float *b, const float *c,
                                                 const float *d, float *x, int ndim, int solvedim,
                                                 int *dims, int *pads) {
  return solve_out<float>(a, b, c, d, x, ndim, solvedim, dims, pads);
}

extern "C" tridStatus_t tridDmtsvStridedBatchFwdAdj(const double *a, const double *b,
                                                    const double *c, const double *d,
                                                    const double *w, double *x, double *da,
                                                    double *db, double *dc, double *dd, int ndim,
                                                    int solvedim, int *dims, int *pads) {
  return solve_fwd_adj<double>(a, b, c, d, w, x, da, db, dc, dd, ndim, solvedim, dims, pads);
}

extern "C" tridStatus_t tridSmtsvStridedBatchFwdAdj(const float *a, const float *b,
                                                    const float *c, const float *d,
                                                    const float *w, float *x, float *da,
                                                    float *db, float *dc, float *dd, int ndim,
                                                    int solvedim, int *dims, int *pads) {
  return solve_fwd_adj<float>(a, b, c, d, w, x, da, db, dc, dd, ndim, solvedim, dims, pads);
}

#define TRID_SPLIT(TAG, T)                                                                     \
  extern "C" tridStatus_t trid##TAG##mtsvStridedBatchSplitReduce(                              \
      const T *a, const T *b, const T *c, const T *d, int ndim, int solvedim, const int *dims,  \
      const int *pads, double *bnd) {                                                          \
    return split_reduce<T>(a, b, c, d, ndim, solvedim, dims, pads, bnd);                       \
  }                                                                                            \
  extern "C" tridStatus_t trid##TAG##mtsvStridedBatchSplitFinish(                              \
      const T *a, const T *b, const T *c, T *d, T *u, int ndim, int solvedim, const int *dims, \
      const int *pads, const double *bnd_all, int nranks, int rank, int inc) {                 \
    return inc ? split_finish<T, 1>(a, b, c, d, u, ndim, solvedim, dims, pads, bnd_all, nranks, \
                                    rank)                                                      \
               : split_finish<T, 0>(a, b, c, d, nullptr, ndim, solvedim, dims, pads, bnd_all,  \
                                    nranks, rank);                                             \
  }
TRID_SPLIT(D, double)
TRID_SPLIT(S, float)

extern "C" void initTridMultiDimBatchSolve(int ndim, int *dims, int *pads) {
  (void)ndim;
  (void)dims;
  (void)pads;
}

extern "C" tridStatus_t tridSetStream(void *stream) {
  tl_stream = (cudaStream_t)stream;
  return TRID_STATUS_SUCCESS;
}

extern "C" void *tridGetStream(void) { return (void *)tl_stream; }

extern "C" tridStatus_t tridReleaseScratch(void) { return release_scratch(); }

extern "C" const char *tridGetStatusString(tridStatus_t s) {
  switch (s) {
    case TRID_STATUS_SUCCESS: return "TRID_STATUS_SUCCESS";
    case TRID_STATUS_NOT_INITIALIZED: return "TRID_STATUS_NOT_INITIALIZED";
    case TRID_STATUS_ALLOC_FAILED: return "TRID_STATUS_ALLOC_FAILED";
    case TRID_STATUS_INVALID_VALUE: return "TRID_STATUS_INVALID_VALUE";
    case TRID_STATUS_ARCH_MISMATCH: return "TRID_STATUS_ARCH_MISMATCH";
    case TRID_STATUS_MAPPING_ERROR: return "TRID_STATUS_MAPPING_ERROR";
    case TRID_STATUS_EXECUTION_FAILED: return "TRID_STATUS_EXECUTION_FAILED";
    case TRID_STATUS_INTERNAL_ERROR: return "TRID_STATUS_INTERNAL_ERROR";
    case TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED: return "TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED";
    case TRID_STATUS_ZERO_PIVOT: return "TRID_STATUS_ZERO_PIVOT";
  }
  return "unknown tridStatus_t";
}

extern "C" tridStatus_t tridSetMethod(int method, int chunk, int sys_per_cta) {
  if (method < 0 || method > 6 || method == 4 || method == 5) return TRID_STATUS_INVALID_VALUE;
  if (chunk != 0 && chunk != 2 && chunk != 4 && chunk != 8 && chunk != 16)
    return TRID_STATUS_INVALID_VALUE;
  if (sys_per_cta != 0 && sys_per_cta != 4 && sys_per_cta != 8 && sys_per_cta != 16 &&
      sys_per_cta != 32)
    return TRID_STATUS_INVALID_VALUE;
  tl_force = {method, chunk, sys_per_cta};
  return TRID_STATUS_SUCCESS;
}

// Reads and clears both error words of the current device: the library's
// (made by the first kernel that needs it) and the allocation-free varlen
// solve's (inside its static array).  Allocates nothing: a word that does not
// exist yet has recorded nothing.
extern "C" tridStatus_t tridGetDeviceErrors(unsigned *flags) {
  if (!flags) return TRID_STATUS_INVALID_VALUE;
  unsigned acc = 0;
  unsigned *words[2] = {device_error_flags_if_present(), noalloc_error_word()};
  for (unsigned *p : words) {
    if (!p) continue;
    unsigned v = 0;
    if (cudaMemcpy(&v, p, sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemset(p, 0, sizeof(unsigned)) != cudaSuccess)
      return TRID_STATUS_EXECUTION_FAILED;
    acc |= v;
  }
  *flags = acc;
  return TRID_STATUS_SUCCESS;
}

extern "C" tridStatus_t tridLoadTuningTable(const char *path) {
  std::call_once(g_env_tune_once, load_env_tuning);  // an explicit table wins
  std::vector<TuneEntry> table;
  if (path) {
    const tridStatus_t st = parse_tuning_table(path, table);
    if (st != TRID_STATUS_SUCCESS) return st;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.swap(table);
  return TRID_STATUS_SUCCESS;
}

extern "C" tridStatus_t tridQueryMethod(int dtype_bytes, int axis, int n, int *method, int *chunk,
                                        int *sys_per_cta) {
  if ((dtype_bytes != 4 && dtype_bytes != 8) || axis < 0 || axis > 4 || n < 0 || !method ||
      !chunk || !sys_per_cta)
    return TRID_STATUS_INVALID_VALUE;
  if (axis == 4) {  // the variable-length batch's bucket for a system of n rows
    int m2 = 0, m4 = 0;
    varlen_buckets(dtype_bytes, m2, m4);
    *method = 2;
    *chunk = n <= m2 ? 2 : (n <= m4 ? 4 : 8);
    *sys_per_cta = 0;
    return TRID_STATUS_SUCCESS;
  }
  const MethodChoice m = choose_method(dtype_bytes, axis, n, 0);
  *method = m.method;
  *chunk = m.chunk;
  *sys_per_cta = m.spc;
  return TRID_STATUS_SUCCESS;
}
