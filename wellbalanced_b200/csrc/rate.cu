// Stable time step on device: the fast-wave rate of every cell reduced per instance
// (carafe/kernels/mhd_rate/mhd_rate_pyccel.py:30-83 in 2D, carafe/mhd3d.py:674-724 in
// 3D), then dt = cfl / max rate with the diffusion limit (carafe/mhd.py:930-963).
// Works on the patch pool; no host synchronisation, so a step can be captured in a graph.
// The per-chunk and per-instance bodies are in ratecell.cuh.
#include "layout.cuh"
#include "numerics.cuh"
#include "ratecell.cuh"
#include "stage.cuh"
#include "wb_internal.cuh"

namespace wb {

__global__ void init_keys_kernel(unsigned long long* keys) {
  keys[0] = double_to_key(0.0);
  keys[1] = rate_min_identity();
}

// Reduction identities of n instances' (max rate, min density) keys and, when
// level_keys is given, of their per-level density minima (n x nlevels keys).
__global__ void init_keys_n_kernel(unsigned long long* keys, int n, unsigned long long* level_keys, int nlevels) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    keys[2 * i] = double_to_key(0.0);
    keys[2 * i + 1] = rate_min_identity();
  }
  if (level_keys && i < n * nlevels) level_keys[i] = rate_min_identity();
}

constexpr int kRateThreads = 256;  // threads of a rate block (8 rounds: 2048 cells)

// One block per (patch, chunk of cells).
template <typename S>
__global__ void __launch_bounds__(kRateThreads) rate2d_kernel(const S* __restrict__ pool, const PatchDesc* patches,
                                                    int npatches, const int* chunk_patch,
                                                    const int* chunk_start, double b0x, double b0y,
                                                    double gamma, const RateSlots slots) {
  rate_chunk2d<S, kRateThreads>(pool, patches, chunk_patch[blockIdx.x], chunk_start[blockIdx.x], b0x, b0y, gamma,
                                slots);
}

template <typename S>
__global__ void __launch_bounds__(kRateThreads) rate3d_kernel(const S* __restrict__ pool, const PatchDesc* patches,
                                                    int npatches, const int* chunk_patch,
                                                    const int* chunk_start, double b0x, double b0y,
                                                    double b0z, double gamma, const RateSlots slots) {
  rate_chunk3d<S, kRateThreads>(pool, patches, chunk_patch[blockIdx.x], chunk_start[blockIdx.x], b0x, b0y, b0z,
                                gamma, slots);
}

// The work list of the rate kernels is derived from the patch table on the host and
// kept by the caller (chunks of 2048 cells).
template <typename S>
int launch_rate_chunks(const S* state, const PatchDesc* patches, int npatches, int ndim, const int* chunk_patch,
                       const int* chunk_start, int nchunks, const double* b0, double gamma,
                       unsigned long long* keys, int ninstances, cudaStream_t stream,
                       unsigned long long* level_keys, int nlevels, unsigned* error) {
  const int slots_n = level_keys ? max(ninstances, ninstances * nlevels) : ninstances;
  init_keys_n_kernel<<<(slots_n + 255) / 256, 256, 0, stream>>>(keys, ninstances, level_keys, nlevels);
  const RateSlots slots{keys, ninstances, level_keys, nlevels, error};
  if (nchunks > 0) {
    if (ndim == 2)
      rate2d_kernel<S><<<nchunks, kRateThreads, 0, stream>>>(state, patches, npatches, chunk_patch, chunk_start, b0[0], b0[1],
                                                    gamma, slots);
    else
      rate3d_kernel<S><<<nchunks, kRateThreads, 0, stream>>>(state, patches, npatches, chunk_patch, chunk_start, b0[0], b0[1],
                                                    b0[2], gamma, slots);
  }
  return check_launch("rate");
}

template int launch_rate_chunks<float>(const float*, const PatchDesc*, int, int, const int*, const int*, int,
                                       const double*, double, unsigned long long*, int, cudaStream_t,
                                       unsigned long long*, int, unsigned*);
template int launch_rate_chunks<double>(const double*, const PatchDesc*, int, int, const int*, const int*, int,
                                        const double*, double, unsigned long long*, int, cudaStream_t,
                                        unsigned long long*, int, unsigned*);

__global__ void finalize_dt_kernel(const unsigned long long* keys, int n, double cfl, double eta, double kappa,
                                   double gamma, const double* inv_dx2_sum, const unsigned long long* level_keys,
                                   const double* inv_dx2_levels, int nlevels, double* time, const double* end,
                                   double* dt, int advance) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    finalize_dt_one(i, keys, cfl, eta, kappa, gamma, inv_dx2_sum, level_keys, inv_dx2_levels, nlevels, time, end, dt,
                    advance);
}

int launch_finalize_dt(const unsigned long long* keys, int ninstances, double cfl, double eta, double kappa,
                       double gamma, const double* inv_dx2_sum, double* time, const double* end, double* dt,
                       int advance_time, cudaStream_t stream, const unsigned long long* level_keys,
                       const double* inv_dx2_levels, int nlevels) {
  if (ninstances > 0)
    finalize_dt_kernel<<<(ninstances + 255) / 256, 256, 0, stream>>>(keys, ninstances, cfl, eta, kappa, gamma,
                                                                     inv_dx2_sum, level_keys, inv_dx2_levels,
                                                                     nlevels, time, end, dt, advance_time);
  return check_launch("finalize_dt");
}

}  // namespace wb
