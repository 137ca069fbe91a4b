// wb_rate_static: the stable-rate reduction of wb_rate with its per-instance keys in a
// file-scope static device array instead of a caller-provided buffer, so the call
// allocates nothing and needs no scratch from the caller. The per-cell work is the rate
// kernel of rate.cu (launch_rate_chunks), run on that static scratch; a last kernel
// decodes the keys into the caller's float64 output, out[2k] = largest rate and
// out[2k+1] = smallest density of instance k (the reference's mhd_rate out[2] per
// instance: carafe/kernels/mhd_rate/mhd_rate_pyccel.py:30-83).
//
// Scratch: kRateStaticMaxInstances instances x 2 keys x 8 bytes = 64 KiB, plus one status
// word, one copy per device (a __device__ variable exists once in every device context).
// No part of it has to start at zero: every call first writes the reduction identities
// into the slots of its instances and clears the status word, and reads only those.
// A patch whose instance index is not below the call's instance count is skipped by the
// rate kernel (it never writes outside the slots) and sets the status word; the decode
// kernel then writes NaN to every output value, so the caller sees the failure.
//
// Set-up: the first call on each device resolves the scratch's device address with
// cudaGetSymbolAddress and caches it (host memory, under a mutex); later calls on that
// device reuse the cached pointer. Make that first call before any stream capture that
// includes this entry point. The cached address belongs to the device's primary context:
// it does not survive cudaDeviceReset, after which this entry point must not be called
// in the same process.
//
// Overlap: all calls on one device share the one scratch array. Two calls in flight at
// the same time (on different streams, or from different host threads without ordering
// between their streams) race on it and may both return wrong values. Calls ordered on
// one stream do not overlap.
#include <mutex>

#include "layout.cuh"
#include "stage.cuh"
#include "wb_internal.cuh"

namespace wb {

constexpr int kRateStaticMaxInstances = 4096;
constexpr int kRateStaticMaxDevices = 64;

// [0, 2 * max): the key pairs; [2 * max]: the status word (low 32 bits)
static __device__ __align__(256) unsigned long long g_rate_scratch[2 * kRateStaticMaxInstances + 1];

__global__ void clear_rate_status_kernel(unsigned long long* status) { *status = 0ull; }

__global__ void decode_rate_keys_kernel(const unsigned long long* __restrict__ keys, int n,
                                        const unsigned long long* __restrict__ status, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 2 * n) out[i] = *status ? __longlong_as_double(0x7ff8000000000000ll) : key_to_double(keys[i]);
}

namespace {

std::mutex g_setup_mutex;
unsigned long long* g_scratch[kRateStaticMaxDevices] = {};

// The device address of g_rate_scratch on the current device (resolved once per device).
int rate_scratch(unsigned long long** ptr) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) {
    set_error("rate_static: cudaGetDevice failed: %s", cudaGetErrorString(e));
    return kCudaError;
  }
  if (device < 0 || device >= kRateStaticMaxDevices) {
    set_error("rate_static: device %d is beyond the %d devices the set-up table holds", device,
              kRateStaticMaxDevices);
    return kUnsupported;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch[device]) {
    void* address = nullptr;
    e = cudaGetSymbolAddress(&address, g_rate_scratch);
    if (e != cudaSuccess || !address) {
      set_error("rate_static: cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
      return kCudaError;
    }
    g_scratch[device] = static_cast<unsigned long long*>(address);
  }
  *ptr = g_scratch[device];
  return kOk;
}

}  // namespace
}  // namespace wb

extern "C" int wb_rate_static(int precision, int ndim, const void* state, const void* patches, int npatches,
                              const int* chunk_patch, const int* chunk_start, int nchunks, double b0x, double b0y,
                              double b0z, double gamma, int ninstances, double* out, void* stream) {
  using namespace wb;
  set_error("");
  if (precision != 32 && precision != 64 && precision != kMath32State64) {
    set_error("rate_static: precision is 32, 64 or %d (a float64 state), not %d", kMath32State64, precision);
    return kBadArgument;
  }
  if (!state || !patches || !out) {
    set_error("rate_static: null state, patch table or output pointer");
    return kBadArgument;
  }
  if ((ndim != 2 && ndim != 3) || ninstances <= 0 || npatches <= 0 || nchunks < 0 ||
      (nchunks > 0 && (!chunk_patch || !chunk_start))) {
    set_error("rate_static: bad ndim / ninstances / patch count / work list");
    return kBadArgument;
  }
  if (ninstances > kRateStaticMaxInstances) {
    set_error("rate_static: %d instances exceed the static scratch of %d instances (%d KiB); use wb_rate with a "
              "caller-provided key buffer",
              ninstances, kRateStaticMaxInstances, int(2 * kRateStaticMaxInstances * sizeof(unsigned long long) / 1024));
    return kTooLarge;
  }
  unsigned long long* keys = nullptr;
  int status = rate_scratch(&keys);
  if (status != kOk) return status;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const double b0[3] = {b0x, b0y, b0z};
  unsigned long long* word = keys + 2 * kRateStaticMaxInstances;
  // the status word's low half, as the rate kernels' error flag (little-endian)
  unsigned* flag = reinterpret_cast<unsigned*>(word);
  clear_rate_status_kernel<<<1, 1, 0, s>>>(word);
  status = precision == 32
               ? launch_rate_chunks<float>(static_cast<const float*>(state), static_cast<const PatchDesc*>(patches),
                                           npatches, ndim, chunk_patch, chunk_start, nchunks, b0, gamma, keys,
                                           ninstances, s, nullptr, 0, flag)
               : launch_rate_chunks<double>(static_cast<const double*>(state), static_cast<const PatchDesc*>(patches),
                                            npatches, ndim, chunk_patch, chunk_start, nchunks, b0, gamma, keys,
                                            ninstances, s, nullptr, 0, flag);
  if (status != kOk) return status;
  decode_rate_keys_kernel<<<(2 * ninstances + 255) / 256, 256, 0, s>>>(keys, ninstances, word, out);
  return check_launch("rate_static decode");
}
