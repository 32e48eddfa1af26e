// Host-side dispatcher for the scalar strided-batch solves (C++17).
//
// Follows the reference's per-axis dispatch (trid_cpu.cpp:406-531 and
// trid_cuda.cu:191-445) but with one B200 kernel family per axis class and no
// transposes: validate -> flatten geometry -> pick method -> launch on the
// caller's stream.
#pragma once

#include <stdint.h>

#include "trid_internal.cuh"

namespace tridb200 {

struct MethodChoice {
  int method;   // 1 = Thomas (generic), 2 = partitioned
  int chunk;    // rows per thread (method 2)
  int spc;      // systems per CTA (method 2, strided axes)
  // where the built-in default is the streamed full-line kernel (method 2
  // with 128 bytes of systems per CTA) and that kernel does not apply: the
  // narrow-tile method and systems per CTA to use instead (0 = none)
  int fb_method = 0;
  int fb_spc = 0;
};

// Systems per CTA for the narrow-tile kernels (plain strided, blocked
// partition), which take 4, 8 or 16.
inline int narrow_spc(const MethodChoice &m) {
  if (m.fb_method != 0) return m.fb_spc;
  return m.spc > 16 ? 16 : m.spc;
}

// Pick the method for (dtype bytes, axis class, n); honours the per-thread
// override and the tuning table.
MethodChoice choose_method(int dtype_bytes, int axis, int n, int opt_hint);

// Validate and flatten; returns TRID_STATUS_SUCCESS with g filled, or an error.
// pads[q] are the per-array pads (q = a,b,c,d,u); pads[4] may be null when !inc.
tridStatus_t make_geom(int ndim, int solvedim, const int *dims, const int *const pads[5],
                       bool inc, Geom &g);

template <typename T, int INC>
tridStatus_t solve_strided_batch(const T *a, const T *b, const T *c, T *d, T *u, int ndim,
                                 int solvedim, const int *dims, const int *const pads[5],
                                 const int *opts, int sync);

}  // namespace tridb200
