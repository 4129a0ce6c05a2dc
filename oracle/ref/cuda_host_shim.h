// cuda_host_shim.h -- lets two of the reference's CUDA sources compile as
// plain host C++ so that they can run serially on the CPU (TEST ONLY).
//
// Used for del-splat-cuda-kernels/cuda/tile_acceleration.h (tile span and
// key bits) and del-splat-cuda-kernels/cuda/splat_point.cu (point z-buffer);
// both need nothing beyond CUDA built-ins.  The grid is emulated by looping
// over threadIdx in oracle/ref/ref_driver.cpp, one thread at a time, so the
// reference's atomics reduce to ordinary read-modify-writes.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>

#define __device__
#define __global__
#define __host__

namespace cuda {
namespace std {
using ::std::array;
}  // namespace std
}  // namespace cuda

struct dsplat_shim_dim3 {
  unsigned x, y, z;
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
