// Stable time step on device: the fast-wave rate of every cell reduced per instance
// (carafe/kernels/mhd_rate/mhd_rate_pyccel.py:30-83 in 2D, carafe/mhd3d.py:674-724 in
// 3D), then dt = cfl / max rate with the diffusion limit (carafe/mhd.py:930-963).
// Works on the patch pool; no host synchronisation, so a step can be captured in a graph.
#include "layout.cuh"
#include "numerics.cuh"
#include "stage.cuh"
#include "wb_internal.cuh"

namespace wb {

__global__ void init_keys_kernel(unsigned long long* keys) {
  keys[0] = double_to_key(0.0);
  keys[1] = double_to_key(__longlong_as_double(0x7ff0000000000000ll));
}

// Reduction identities of n instances' (max rate, min density) keys and, when
// level_keys is given, of their per-level density minima (n x nlevels keys).
__global__ void init_keys_n_kernel(unsigned long long* keys, int n, unsigned long long* level_keys, int nlevels) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    keys[2 * i] = double_to_key(0.0);
    keys[2 * i + 1] = double_to_key(__longlong_as_double(0x7ff0000000000000ll));
  }
  if (level_keys && i < n * nlevels) level_keys[i] = double_to_key(__longlong_as_double(0x7ff0000000000000ll));
}

// Where a rate block reduces: the instance's key pair and, optionally, the density-minimum
// key of the patch's level. A patch whose instance or level lies outside the key arrays
// is skipped (its block reduces nothing) and flagged in `error` (nullable).
struct RateSlots {
  unsigned long long* keys;        // [2 * ninstances]
  int ninstances;
  unsigned long long* level_keys;  // [ninstances * nlevels] or null
  int nlevels;
  unsigned* error;                 // nullable
};

__device__ __forceinline__ bool rate_slot(const PatchDesc& P, const RateSlots& r, unsigned long long** keys,
                                          unsigned long long** level_min) {
  const bool ok = P.instance >= 0 && P.instance < r.ninstances && (!r.level_keys || (P.level >= 0 && P.level < r.nlevels));
  if (!ok) {
    if (r.error && threadIdx.x == 0) atomicOr(r.error, 1u);
    return false;
  }
  *keys = r.keys + 2 * P.instance;
  *level_min = r.level_keys ? r.level_keys + P.instance * r.nlevels + P.level : nullptr;
  return true;
}

constexpr unsigned kRateThreads = 256;  // threads of a rate block (8 rounds: 2048 cells)

// 2D: one block per (patch, chunk of cells); grid.y unused.
template <typename S>
__global__ void __launch_bounds__(kRateThreads) rate2d_kernel(const S* __restrict__ pool, const PatchDesc* patches,
                                                    int npatches, const int* chunk_patch,
                                                    const int* chunk_start, double b0x, double b0y,
                                                    double gamma, const RateSlots slots) {
  const int pi = chunk_patch[blockIdx.x];
  const PatchDesc P = patches[pi];
  unsigned long long *keys, *level_min;
  if (!rate_slot(P, slots, &keys, &level_min)) return;  // uniform over the block
  const int nx = P.n[0], ny = P.n[1];
  const S* src = pool + P.off;
  const int64_t pitch = P.pitch0, fs = P.fstride;
  using M = Math<S>;
  const S dx = S(P.dx[0]), dy = S(P.dx[1]);
  const S idx = M::inv(dx), idy = M::inv(dy);
  const S g = S(gamma), bx0 = S(b0x), by0 = S(b0y);
  S largest = S(0), smallest = S(INFINITY);  // converted once, exactly (as in 3D)
  // work-list indices are 32-bit (chunk_start is int): 32-bit index arithmetic
  const unsigned total = unsigned(nx) * unsigned(ny);
  const unsigned start = unsigned(chunk_start[blockIdx.x]);
#pragma unroll 2
  for (int s = 0; s < 8; ++s) {
    const unsigned t = start + unsigned(s) * kRateThreads + threadIdx.x;
    if (t >= total) continue;
    const unsigned row = t / unsigned(ny);
    const int i = int(row) + kHalo, j = int(t - row * unsigned(ny)) + kHalo;
    const int64_t c = int64_t(i) * pitch + j;
    const S* A = src + 6 * fs;
    const S r = src[c];
    const S ir = M::inv(r);
    const S u = M::div(src[fs + c], r, ir), v = M::div(src[2 * fs + c], r, ir), w = M::div(src[3 * fs + c], r, ir);
    const S bx = S(0.5) * (M::div(A[c + 1] - A[c], dy, idy) + bx0 + (M::div(A[c + pitch + 1] - A[c + pitch], dy, idy) + bx0));
    const S by = S(0.5) * (-M::div(A[c + pitch] - A[c], dx, idx) + by0 + (-M::div(A[c + pitch + 1] - A[c + 1], dx, idx) + by0));
    const S bz = src[5 * fs + c];
    const S p = (g - S(1)) * (src[4 * fs + c] - S(0.5) * r * (u * u + v * v + w * w) - S(0.5) * (bx * bx + by * by + bz * bz));
    const S rate = M::div(rabs(u) + fast_speed(r, p, bx, by, bz, g), dx, idx) +
                   M::div(rabs(v) + fast_speed(r, p, by, bx, bz, g), dy, idy);
    largest = rmax(largest, rate);
    smallest = rmin(smallest, r);
  }
  block_reduce_keys(double(largest), double(smallest), keys, level_min);
}

template <typename S>
__global__ void __launch_bounds__(kRateThreads) rate3d_kernel(const S* __restrict__ pool, const PatchDesc* patches,
                                                    int npatches, const int* chunk_patch,
                                                    const int* chunk_start, double b0x, double b0y,
                                                    double b0z, double gamma, const RateSlots slots) {
  const int pi = chunk_patch[blockIdx.x];
  const PatchDesc P = patches[pi];
  unsigned long long *keys, *level_min;
  if (!rate_slot(P, slots, &keys, &level_min)) return;  // uniform over the block
  const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
  const S* src = pool + P.off;
  const int64_t p0 = P.pitch0, p1 = P.pitch1, fs = P.fstride;
  using M = Math<S>;
  const S dx = S(P.dx[0]), dy = S(P.dx[1]), dz = S(P.dx[2]);
  const S idx = M::inv(dx), idy = M::inv(dy), idz = M::inv(dz);
  const S g = S(gamma);
  // the max / min in the state's type (exact: the max of the float rates converts to the
  // max of their double images), converted once for the block reduction
  S largest = S(0), smallest = S(INFINITY);
  // work-list indices are 32-bit (chunk_start is int): 32-bit index arithmetic
  const unsigned total = unsigned(nx) * unsigned(ny) * unsigned(nz);
  const unsigned start = unsigned(chunk_start[blockIdx.x]);
#pragma unroll 2
  for (int s = 0; s < 8; ++s) {
    const unsigned t = start + unsigned(s) * kRateThreads + threadIdx.x;
    if (t >= total) continue;
    const unsigned line = t / unsigned(nz);
    const unsigned plane = line / unsigned(ny);
    const int i = int(plane) + kHalo;
    const int j = int(line - plane * unsigned(ny)) + kHalo;
    const int k = int(t - line * unsigned(nz)) + kHalo;
    const int64_t o = int64_t(i) * p0 + int64_t(j) * p1 + k;
    const S* Ax = src + 5 * fs;
    const S* Ay = src + 6 * fs;
    const S* Az = src + 7 * fs;
    const S bxl = M::div(Az[o + p1] - Az[o], dy, idy) - M::div(Ay[o + 1] - Ay[o], dz, idz) + S(b0x);
    const S bxh = M::div(Az[o + p0 + p1] - Az[o + p0], dy, idy) - M::div(Ay[o + p0 + 1] - Ay[o + p0], dz, idz) + S(b0x);
    const S byl = M::div(Ax[o + 1] - Ax[o], dz, idz) - M::div(Az[o + p0] - Az[o], dx, idx) + S(b0y);
    const S byh = M::div(Ax[o + p1 + 1] - Ax[o + p1], dz, idz) - M::div(Az[o + p1 + p0] - Az[o + p1], dx, idx) + S(b0y);
    const S bzl = M::div(Ay[o + p0] - Ay[o], dx, idx) - M::div(Ax[o + p1] - Ax[o], dy, idy) + S(b0z);
    const S bzh = M::div(Ay[o + p0 + 1] - Ay[o + 1], dx, idx) - M::div(Ax[o + p1 + 1] - Ax[o + 1], dy, idy) + S(b0z);
    const S bx = S(0.5) * (bxl + bxh), by = S(0.5) * (byl + byh), bz = S(0.5) * (bzl + bzh);
    const S r = src[o];
    const S ir = M::inv(r);
    const S u = M::div(src[fs + o], r, ir), v = M::div(src[2 * fs + o], r, ir), w = M::div(src[3 * fs + o], r, ir);
    const S p = (g - S(1)) * (src[4 * fs + o] - S(0.5) * r * (u * u + v * v + w * w) - S(0.5) * (bx * bx + by * by + bz * bz));
    const S rate = M::div(rabs(u) + fast_speed(r, p, bx, by, bz, g), dx, idx) +
                   M::div(rabs(v) + fast_speed(r, p, by, bz, bx, g), dy, idy) +
                   M::div(rabs(w) + fast_speed(r, p, bz, bx, by, g), dz, idz);
    largest = rmax(largest, rate);
    smallest = rmin(smallest, r);
  }
  block_reduce_keys(double(largest), double(smallest), keys, level_min);
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

// dt of instance i: cfl times the smaller of the fast-wave crossing time 1 / rate and the
// explicit diffusion limit 0.5 / (D (dx^-2 + dy^-2 [+ dz^-2])), D = max(eta, (gamma - 1)
// kappa / rho_min). With per-level keys the limit is taken level by level, each level's
// smallest density with that level's spacing, as the reference takes it patch by patch
// (carafe/mhd.py:942-960: patches of one level share the spacing, so the smallest
// density of the level decides); without them, the instance's smallest density with its
// finest spacing.
__global__ void finalize_dt_kernel(const unsigned long long* keys, int n, double cfl, double eta, double kappa,
                                   double gamma, const double* inv_dx2_sum, const unsigned long long* level_keys,
                                   const double* inv_dx2_levels, int nlevels, double* time, const double* end,
                                   double* dt, int advance) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double rate = key_to_double(keys[2 * i]);
  double smallest = 1.0 / rate;
  if (eta > 0.0 || kappa > 0.0) {
    if (level_keys) {
      for (int l = 0; l < nlevels; ++l) {
        const double inv = inv_dx2_levels[i * nlevels + l];
        if (!(inv > 0.0)) continue;  // no patch of the instance on this level
        const double rho_min = key_to_double(level_keys[i * nlevels + l]);
        const double diffusivity = fmax(eta, (gamma - 1.0) * kappa / rho_min);
        if (diffusivity > 0.0) smallest = fmin(smallest, 0.5 / (diffusivity * inv));
      }
    } else {
      const double rho_min = key_to_double(keys[2 * i + 1]);
      const double diffusivity = fmax(eta, (gamma - 1.0) * kappa / rho_min);
      if (diffusivity > 0.0) smallest = fmin(smallest, 0.5 / (diffusivity * inv_dx2_sum[i]));
    }
  }
  double step = cfl * smallest;
  if (end) {
    const double remaining = end[i] - time[i];
    if (!(time[i] < end[i] * (1.0 - 1e-14))) step = 0.0;
    step = fmin(step, fmax(remaining, 0.0));
  }
  dt[i] = step;
  if (advance && time) time[i] += step;
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
