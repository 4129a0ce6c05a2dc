// cuda_host_shim.h -- lets two of the reference's CUDA sources compile as
// plain host C++ so that they can run serially on the CPU (TEST ONLY).
//
// Used for del-splat-cuda-kernels/cuda/tile_acceleration.h (tile span and
// key bits), splat_point.cu (point z-buffer), and splat_gauss.cu /
// splat_circle.cu (projection, blend, circle painter; their del-geo includes
// resolve to oracle/ref/del_geo/, which forwards to the oracle's
// restatement).  The grid is emulated by the drivers (ref_*.cpp) one thread
// at a time (per host thread: the built-in indices are thread_local), so the
// reference's atomics reduce to ordinary read-modify-writes.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>

// The reference's sources repeat tile_acceleration.h and the kernel names;
// a translation unit that compiles one of them next to the others defines
// DSPLAT_SHIM_INTERNAL first (device functions get internal linkage) and
// renames the extern "C" kernels with macros.
#ifdef DSPLAT_SHIM_INTERNAL
#define __device__ static inline
#else
#define __device__
#endif
#define __global__
#define __host__

namespace cuda {
namespace std {
using ::std::array;
}  // namespace std
}  // namespace cuda

struct dsplat_shim_dim3 {
  unsigned x = 0, y = 0, z = 0;
};
extern thread_local dsplat_shim_dim3 threadIdx, blockIdx, blockDim;

inline unsigned atomicAdd(unsigned* p, unsigned v) {
  unsigned o = *p;
  *p = o + v;
  return o;
}
inline unsigned atomicCAS(unsigned* p, unsigned cmp, unsigned val) {
  unsigned o = *p;
  if (o == cmp) *p = val;
  return o;
}
inline float __uint_as_float(unsigned u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
inline unsigned __float_as_uint(float f) {
  unsigned u;
  std::memcpy(&u, &f, 4);
  return u;
}
