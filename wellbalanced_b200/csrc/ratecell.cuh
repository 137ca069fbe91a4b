// Device bodies of the stable-time-step reduction (carafe/kernels/mhd_rate/mhd_rate_pyccel.py:30-83
// in 2D, carafe/mhd3d.py:674-724 in 3D; dt as carafe/mhd.py:930-963): one chunk of cells
// over the threads of a block, and the step of one instance. Shared by the rate kernels
// and the op program.
#pragma once

#include "layout.cuh"
#include "numerics.cuh"
#include "wb_internal.cuh"

namespace wb {

// Cells per work item of the rate reduction (the host cuts every patch into such chunks).
constexpr unsigned kRateChunk = 2048;

__device__ __forceinline__ unsigned long long rate_min_identity() {
  return double_to_key(__longlong_as_double(0x7ff0000000000000ll));
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

// The cells of one chunk (kRateChunk cells of patch pi from `chunk_start`) over the NT
// threads of a block, reduced into the chunk's slots. 2D:
template <typename S, int NT>
__device__ __forceinline__ void rate_chunk2d(const S* __restrict__ pool, const PatchDesc* patches, int pi,
                                             int chunk_start, double b0x, double b0y, double gamma,
                                             const RateSlots& slots) {
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
  const unsigned start = unsigned(chunk_start);
#pragma unroll 2
  for (int s = 0; s < int(kRateChunk / NT); ++s) {
    const unsigned t = start + unsigned(s) * NT + threadIdx.x;
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

// 3D:
template <typename S, int NT>
__device__ __forceinline__ void rate_chunk3d(const S* __restrict__ pool, const PatchDesc* patches, int pi,
                                             int chunk_start, double b0x, double b0y, double b0z, double gamma,
                                             const RateSlots& slots) {
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
  const unsigned start = unsigned(chunk_start);
#pragma unroll 2
  for (int s = 0; s < int(kRateChunk / NT); ++s) {
    const unsigned t = start + unsigned(s) * NT + threadIdx.x;
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

// dt of instance i: cfl times the smaller of the fast-wave crossing time 1 / rate and the
// explicit diffusion limit 0.5 / (D (dx^-2 + dy^-2 [+ dz^-2])), D = max(eta, (gamma - 1)
// kappa / rho_min). With per-level keys the limit is taken level by level, each level's
// smallest density with that level's spacing, as the reference takes it patch by patch
// (carafe/mhd.py:942-960: patches of one level share the spacing, so the smallest
// density of the level decides); without them, the instance's smallest density with its
// finest spacing.
__device__ __forceinline__ void finalize_dt_one(int i, const unsigned long long* keys, double cfl, double eta,
                                                double kappa, double gamma, const double* inv_dx2_sum,
                                                const unsigned long long* level_keys, const double* inv_dx2_levels,
                                                int nlevels, double* time, const double* end, double* dt,
                                                int advance) {
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

}  // namespace wb
