// Arguments and launchers of the fused stage kernels and the per-step rate kernels.
#pragma once

#include <cuda_runtime.h>

#include "layout.cuh"

namespace wb {

// One RK stage over a work list of tiles:
//   stage 1 (base == nullptr): dst = src - dt L(src)
//   stage 2 (base != nullptr): dst = (src - dt L(src) + base) / 2   (Heun combine)
// src is read with its halos; base and dst only at the tile's own cells / nodes, so
// dst may alias base (stage 2 writes the new state over the start state in place).
template <typename S>
struct StageArgs {
  const S* src;
  const S* base;
  S* dst;
  const PatchDesc* patches;
  const Tile* tiles;
  const double* dt;             // per instance
  double gamma, inv_gm1;
  double b0[3];
  unsigned long long* bad;      // count of non-positive / non-finite cells
  double* bflux;                // boundary-face fluxes of each patch (nullable)
  int lx;                       // 3D: cell planes per tile along x
  // non-ideal terms (zero: ideal MHD): resistivity, Braginskii conduction along and
  // across the field (2D only), gravity
  double eta = 0.0, kappa_par = 0.0, kappa_perp = 0.0;
  double gravity[3] = {0.0, 0.0, 0.0};
};

// The precision code of a float64 state advanced with float32 arithmetic (the C ABI's
// WB_MATH32_STATE64); the other codes are 32 (float32 state and arithmetic) and 64.
constexpr int kMath32State64 = 6432;

// S: the state's type; R: the arithmetic of the face work (R = S, or S = double with
// R = float). tx x ty: the tile shape the work list was cut with (one of tile_shapes_2d)
template <typename S, typename R = S>
int launch_stage2d(const StageArgs<S>& args, int ntiles, int limiter, int tx, int ty, cudaStream_t stream);
// ty x tz: the tile shape the work list was cut with (one of tile_shapes_3d)
template <typename S, typename R = S>
int launch_stage3d(const StageArgs<S>& args, int ntiles, int limiter, int ty, int tz, cudaStream_t stream);

// mode: 0 float32, 1 float64, kMath32State64 the float64 state with float32 arithmetic
void tile_shape_2d(int mode, int* tx, int* ty);
// The 2D tile shapes built, (tx, ty) pairs, the default first; returns their count.
int tile_shapes_2d(int mode, int* shapes, int max);
// The 3D tile shapes built, (ty, tz) pairs, the default first; returns their count.
int tile_shapes_3d(int mode, int* shapes, int max);
void tile_shape_3d(int mode, int* ty, int* tz);

// Fast-wave rate max and density min of every patch's cells, per instance, as
// order-preserving keys: keys[2 * instance] (max rate), keys[2 * instance + 1] (min rho);
// with level_keys (nullable), also the density min of each (instance, level) at
// level_keys[instance * nlevels + level]. Work list: chunks of up to 2048 cells
// (chunk_patch[c], chunk_start[c]). Patches whose instance (or level) lies outside the
// key arrays are skipped and flagged in *error (nullable).
template <typename S>
int launch_rate_chunks(const S* state, const PatchDesc* patches, int npatches, int ndim, const int* chunk_patch,
                       const int* chunk_start, int nchunks, const double* b0, double gamma,
                       unsigned long long* keys, int ninstances, cudaStream_t stream,
                       unsigned long long* level_keys = nullptr, int nlevels = 0, unsigned* error = nullptr);

// dt[i] = min(cfl / rate_i, diffusion limit_i, remaining_i); advances time[i] by it. The
// diffusion limit is per level when level_keys / inv_dx2_levels are given.
int launch_finalize_dt(const unsigned long long* keys, int ninstances, double cfl, double diffusivity,
                       double conduction, double gamma, const double* inv_dx2_sum, double* time,
                       const double* end, double* dt, int advance_time, cudaStream_t stream,
                       const unsigned long long* level_keys = nullptr, const double* inv_dx2_levels = nullptr,
                       int nlevels = 0);

}  // namespace wb
