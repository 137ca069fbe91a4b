// Internal helpers shared by the CUDA translation units: launch checks, the library's
// last-error text, exact order-independent max/min reductions through integer keys.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

namespace wb {

// Status codes of the C ABI (also in include/wellbalanced_b200.h).
enum Status : int {
  kOk = 0,
  kBadArgument = -1,
  kCudaError = -2,
  kUnsupported = -3,
  kTooLarge = -4,
};

void set_error(const char* fmt, ...);
const char* last_error();

inline int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: CUDA launch failed: %s", what, cudaGetErrorString(e));
    return kCudaError;
  }
  return kOk;
}

// Order-preserving map of a double onto uint64: a < b  <=>  key(a) < key(b) (non-NaN).
__device__ __forceinline__ unsigned long long double_to_key(double x) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__host__ __device__ __forceinline__ double key_to_double_bits(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double out;
  memcpy(&out, &b, sizeof(out));
  return out;
}

__device__ __forceinline__ double key_to_double(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double(static_cast<long long>(b));
}

// keys[0] = key(0) (running max of a non-negative rate), keys[1] = key(+inf) (running min)
__global__ void init_keys_kernel(unsigned long long* keys);

// Block-wide max of `largest` and min of `smallest`, one atomic per warp; the min also
// into *level_min when given.
__device__ __forceinline__ void block_reduce_keys(double largest, double smallest,
                                                  unsigned long long* keys,
                                                  unsigned long long* level_min = nullptr) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    largest = fmax(largest, __shfl_xor_sync(0xffffffffu, largest, o));
    smallest = fmin(smallest, __shfl_xor_sync(0xffffffffu, smallest, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&keys[0], double_to_key(largest));
    atomicMin(&keys[1], double_to_key(smallest));
    if (level_min) atomicMin(level_min, double_to_key(smallest));
  }
}

}  // namespace wb
