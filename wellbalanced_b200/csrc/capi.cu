// extern "C" entry points of libwb200.so (declared in include/wellbalanced_b200.h):
// argument validation, error text, dispatch to the kernel launchers.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/wellbalanced_b200.h"
#include "halo.cuh"
#include "layout.cuh"
#include "stage.cuh"
#include "wb_internal.cuh"

namespace wb {

static thread_local char g_error[512] = "";

void set_error(const char* fmt, ...) {
  va_list args;
  va_start(args, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, args);
  va_end(args);
}

const char* last_error() { return g_error; }

int launch_primitive_fp64(const double*, const double*, const double*, const double*, const double*,
                          const double*, const double*, int, int, double, double, double, double, double,
                          double*, double*, double*, double*, unsigned long long*, cudaStream_t);
int launch_sweep_fp64(const double*, const double*, int, int, double, int, int, double*, cudaStream_t);
int launch_ct_fp64(const double*, const double*, const double*, const double*, const double*, int, int, int,
                   int, double*, cudaStream_t);
int launch_ct_planes_fp64(const double*, const double*, const double*, const double*, const double*, int, int,
                          int, int, int, double*, cudaStream_t);
int launch_rate_fp64(const double*, const double*, const double*, const double*, const double*, const double*,
                     const double*, int, int, int, double, double, double, double, double, double*,
                     cudaStream_t);
int launch_resistive_fp64(const double*, const double*, const double*, int, int, double, double, double,
                          double*, double*, double*, cudaStream_t);
int launch_conductive_fp64(const double*, const double*, const double*, int, int, double, double, double,
                           double, double*, double*, cudaStream_t);

}  // namespace wb

using namespace wb;

namespace {

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

bool block_ok(int64_t X, int64_t Y, const char* what) {
  if (X < 4 || Y < 4 || X > (1 << 30) || Y > (1 << 30) || X * Y > (int64_t(1) << 40)) {
    set_error("%s: block shape (%lld, %lld) out of range (each side >= 4)", what, (long long)X, (long long)Y);
    return false;
  }
  return true;
}

bool ptrs_ok(std::initializer_list<const void*> ptrs, const char* what) {
  for (const void* p : ptrs)
    if (!p) {
      set_error("%s: a required pointer is NULL", what);
      return false;
    }
  return true;
}

// Precision codes: 32 (float32 state and arithmetic), 64 (float64), and
// WB_MATH32_STATE64 (a float64 state advanced with float32 arithmetic). Kernels that only
// move or reduce the state (halos, restriction, reflux, rate) take the state's type.
bool precision_ok(int precision, const char* what) {
  if (precision != 32 && precision != 64 && precision != kMath32State64) {
    set_error("%s: precision must be 32, 64 or %d, got %d", what, kMath32State64, precision);
    return false;
  }
  return true;
}

// the tile-shape table of a precision code
int shape_mode(int precision) { return precision == 32 ? 0 : (precision == 64 ? 1 : kMath32State64); }

}  // namespace

extern "C" {

const char* wb_version(void) { return "wellbalanced_b200 0.1.0 (sm_100a)"; }

const char* wb_last_error(void) { return last_error(); }

int wb_mhd_primitive(const double* rho, const double* mx, const double* my, const double* mz, const double* energy,
                     const double* bz, const double* az, int64_t X, int64_t Y, double dx, double dy, double b0x,
                     double b0y, double gamma, double* prim, double* bxf, double* byf, double* ecc,
                     unsigned long long* bad, void* stream) {
  set_error("");
  if (!block_ok(X, Y, "mhd_primitive") ||
      !ptrs_ok({rho, mx, my, mz, energy, bz, az, prim, bxf, byf, ecc, bad}, "mhd_primitive"))
    return kBadArgument;
  return launch_primitive_fp64(rho, mx, my, mz, energy, bz, az, int(X), int(Y), dx, dy, b0x, b0y, gamma, prim, bxf,
                               byf, ecc, bad, as_stream(stream));
}

int wb_mhd_sweep(const double* prim, const double* bn, int axis, int limiter, double gamma, int64_t X, int64_t Y,
                 double* flux, void* stream) {
  set_error("");
  if (!block_ok(X, Y, "mhd_sweep") || !ptrs_ok({prim, bn, flux}, "mhd_sweep")) return kBadArgument;
  if (axis != 0 && axis != 1) {
    set_error("mhd_sweep: axis must be 0 or 1, got %d", axis);
    return kBadArgument;
  }
  if (limiter < 0 || limiter > 3) {
    set_error("mhd_sweep: limiter code %d is not one of 0..3", limiter);
    return kBadArgument;
  }
  return launch_sweep_fp64(prim, bn, axis, limiter, gamma, int(X), int(Y), flux, as_stream(stream));
}

int wb_ct_contact(const double* fx_by, const double* gy_bx, const double* fx_rho, const double* gy_rho,
                  const double* ecc, int64_t X, int64_t Y, int64_t na, int64_t nb, double* ez, void* stream) {
  set_error("");
  if (!block_ok(X, Y, "ct_contact") || !ptrs_ok({fx_by, gy_bx, fx_rho, gy_rho, ecc, ez}, "ct_contact"))
    return kBadArgument;
  if (na < 0 || nb < 0 || na > X - 3 || nb > Y - 3) {
    set_error("ct_contact: ez shape (%lld, %lld) exceeds (X-3, Y-3)", (long long)na, (long long)nb);
    return kBadArgument;
  }
  return launch_ct_fp64(fx_by, gy_bx, fx_rho, gy_rho, ecc, int(X), int(Y), int(na), int(nb), ez, as_stream(stream));
}

int wb_ct_contact_planes(const double* fx_by, const double* gy_bx, const double* fx_rho, const double* gy_rho,
                         const double* ecc, int64_t X, int64_t Y, int64_t na, int64_t nb, int64_t planes, double* ez,
                         void* stream) {
  set_error("");
  if (!block_ok(X, Y, "ct_contact_planes") || !ptrs_ok({fx_by, gy_bx, fx_rho, gy_rho, ecc, ez}, "ct_contact_planes"))
    return kBadArgument;
  if (na < 0 || nb < 0 || na > X - 3 || nb > Y - 3 || planes < 0 || planes > 65535) {
    set_error("ct_contact_planes: ez shape (%lld, %lld) x %lld planes out of range", (long long)na, (long long)nb,
              (long long)planes);
    return kBadArgument;
  }
  return launch_ct_planes_fp64(fx_by, gy_bx, fx_rho, gy_rho, ecc, int(X), int(Y), int(na), int(nb), int(planes), ez,
                               as_stream(stream));
}

int wb_mhd_rate(const double* rho, const double* mx, const double* my, const double* mz, const double* energy,
                const double* bz, const double* az, int64_t X, int64_t Y, int halo, double dx, double dy,
                double b0x, double b0y, double gamma, double* out, void* stream) {
  set_error("");
  if (!block_ok(X, Y, "mhd_rate") || !ptrs_ok({rho, mx, my, mz, energy, bz, az, out}, "mhd_rate"))
    return kBadArgument;
  if (halo < 0 || 2 * halo >= X || 2 * halo >= Y) {
    set_error("mhd_rate: halo %d leaves no cells", halo);
    return kBadArgument;
  }
  return launch_rate_fp64(rho, mx, my, mz, energy, bz, az, int(X), int(Y), halo, dx, dy, b0x, b0y, gamma, out,
                          as_stream(stream));
}

int wb_mhd_resistive(const double* prim, const double* bxf, const double* byf, int64_t X, int64_t Y, double dx,
                     double dy, double eta, double* fx, double* fy, double* ez, void* stream) {
  set_error("");
  if (!block_ok(X, Y, "mhd_resistive") || !ptrs_ok({prim, bxf, byf, fx, fy, ez}, "mhd_resistive"))
    return kBadArgument;
  return launch_resistive_fp64(prim, bxf, byf, int(X), int(Y), dx, dy, eta, fx, fy, ez, as_stream(stream));
}

int wb_mhd_conductive(const double* prim, const double* bxf, const double* byf, int64_t X, int64_t Y, double dx,
                      double dy, double parallel, double perpendicular, double* fx, double* fy, void* stream) {
  set_error("");
  if (!block_ok(X, Y, "mhd_conductive") || !ptrs_ok({prim, bxf, byf, fx, fy}, "mhd_conductive"))
    return kBadArgument;
  return launch_conductive_fp64(prim, bxf, byf, int(X), int(Y), dx, dy, parallel, perpendicular, fx, fy,
                                as_stream(stream));
}

static int stage2d(int precision, const void* src, const void* base, void* dst, const void* patches,
                   const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y, int limiter,
                   int tx, int ty, unsigned long long* bad, double* bflux, void* stream) {
  if (!precision_ok(precision, "stage2d") || !ptrs_ok({src, dst, patches, tiles, dt, bad}, "stage2d"))
    return kBadArgument;
  if (ntiles < 0 || !(gamma > 1.0)) {
    set_error("stage2d: ntiles must be >= 0 and gamma > 1");
    return kBadArgument;
  }
  if (precision == 32) {
    StageArgs<float> a{static_cast<const float*>(src), static_cast<const float*>(base), static_cast<float*>(dst),
                       static_cast<const PatchDesc*>(patches), static_cast<const Tile*>(tiles), dt, gamma,
                       1.0 / (gamma - 1.0), {b0x, b0y, 0.0}, bad, bflux, 0};
    return launch_stage2d<float>(a, ntiles, limiter, tx, ty, as_stream(stream));
  }
  StageArgs<double> a{static_cast<const double*>(src), static_cast<const double*>(base), static_cast<double*>(dst),
                      static_cast<const PatchDesc*>(patches), static_cast<const Tile*>(tiles), dt, gamma,
                      1.0 / (gamma - 1.0), {b0x, b0y, 0.0}, bad, bflux, 0};
  return precision == 64 ? launch_stage2d<double, double>(a, ntiles, limiter, tx, ty, as_stream(stream))
                         : launch_stage2d<double, float>(a, ntiles, limiter, tx, ty, as_stream(stream));
}

int wb_stage2d(int precision, const void* src, const void* base, void* dst, const void* patches, const void* tiles,
               int ntiles, const double* dt, double gamma, double b0x, double b0y, int limiter,
               unsigned long long* bad, double* bflux, void* stream) {
  set_error("");
  int tx, ty;
  tile_shape_2d(shape_mode(precision), &tx, &ty);
  return stage2d(precision, src, base, dst, patches, tiles, ntiles, dt, gamma, b0x, b0y, limiter, tx, ty, bad, bflux,
                 stream);
}

int wb_stage2d_tiled(int precision, const void* src, const void* base, void* dst, const void* patches,
                     const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y, int limiter,
                     int tx, int ty, unsigned long long* bad, double* bflux, void* stream) {
  set_error("");
  return stage2d(precision, src, base, dst, patches, tiles, ntiles, dt, gamma, b0x, b0y, limiter, tx, ty, bad, bflux,
                 stream);
}

int wb_tile_shapes(int ndim, int precision, int* shapes, int max) {
  set_error("");
  if (!precision_ok(precision, "tile_shapes") || (max > 0 && !shapes)) return kBadArgument;
  if (ndim != 2 && ndim != 3) {
    set_error("tile_shapes: ndim must be 2 or 3");
    return kBadArgument;
  }
  return ndim == 2 ? tile_shapes_2d(shape_mode(precision), shapes, max)
                   : tile_shapes_3d(shape_mode(precision), shapes, max);
}

int wb_stage2d_physics(int precision, const void* src, const void* base, void* dst, const void* patches,
                       const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y, int limiter,
                       double eta, double kappa_par, double kappa_perp, double gx, double gy,
                       unsigned long long* bad, void* stream) {
  set_error("");
  if (!precision_ok(precision, "stage2d_physics") ||
      !ptrs_ok({src, dst, patches, tiles, dt, bad}, "stage2d_physics"))
    return kBadArgument;
  if (ntiles < 0 || !(gamma > 1.0) || !(eta >= 0.0) || !(kappa_par >= 0.0) || !(kappa_perp >= 0.0)) {
    set_error("stage2d_physics: ntiles must be >= 0, gamma > 1, and eta and the conductivities >= 0");
    return kBadArgument;
  }
  int tx, ty;  // the non-ideal kernel runs on the default tiles
  tile_shape_2d(shape_mode(precision), &tx, &ty);
  if (precision == 32) {
    StageArgs<float> a{static_cast<const float*>(src), static_cast<const float*>(base), static_cast<float*>(dst),
                       static_cast<const PatchDesc*>(patches), static_cast<const Tile*>(tiles), dt, gamma,
                       1.0 / (gamma - 1.0), {b0x, b0y, 0.0}, bad, nullptr, 0};
    a.eta = eta, a.kappa_par = kappa_par, a.kappa_perp = kappa_perp, a.gravity[0] = gx, a.gravity[1] = gy;
    return launch_stage2d<float>(a, ntiles, limiter, tx, ty, as_stream(stream));
  }
  StageArgs<double> a{static_cast<const double*>(src), static_cast<const double*>(base), static_cast<double*>(dst),
                      static_cast<const PatchDesc*>(patches), static_cast<const Tile*>(tiles), dt, gamma,
                      1.0 / (gamma - 1.0), {b0x, b0y, 0.0}, bad, nullptr, 0};
  a.eta = eta, a.kappa_par = kappa_par, a.kappa_perp = kappa_perp, a.gravity[0] = gx, a.gravity[1] = gy;
  return precision == 64 ? launch_stage2d<double, double>(a, ntiles, limiter, tx, ty, as_stream(stream))
                         : launch_stage2d<double, float>(a, ntiles, limiter, tx, ty, as_stream(stream));
}

static int stage3d(int precision, const void* src, const void* base, void* dst, const void* patches,
                   const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y, double b0z,
                   int limiter, int lx, int ty, int tz, unsigned long long* bad, double* bflux, void* stream) {
  if (!precision_ok(precision, "stage3d") || !ptrs_ok({src, dst, patches, tiles, dt, bad}, "stage3d"))
    return kBadArgument;
  if (ntiles < 0 || !(gamma > 1.0) || lx <= 0) {
    set_error("stage3d: ntiles must be >= 0, gamma > 1 and lx > 0");
    return kBadArgument;
  }
  if (precision == 32) {
    StageArgs<float> a{static_cast<const float*>(src), static_cast<const float*>(base), static_cast<float*>(dst),
                       static_cast<const PatchDesc*>(patches), static_cast<const Tile*>(tiles), dt, gamma,
                       1.0 / (gamma - 1.0), {b0x, b0y, b0z}, bad, bflux, lx};
    return launch_stage3d<float>(a, ntiles, limiter, ty, tz, as_stream(stream));
  }
  StageArgs<double> a{static_cast<const double*>(src), static_cast<const double*>(base), static_cast<double*>(dst),
                      static_cast<const PatchDesc*>(patches), static_cast<const Tile*>(tiles), dt, gamma,
                      1.0 / (gamma - 1.0), {b0x, b0y, b0z}, bad, bflux, lx};
  return precision == 64 ? launch_stage3d<double, double>(a, ntiles, limiter, ty, tz, as_stream(stream))
                         : launch_stage3d<double, float>(a, ntiles, limiter, ty, tz, as_stream(stream));
}

int wb_stage3d(int precision, const void* src, const void* base, void* dst, const void* patches, const void* tiles,
               int ntiles, const double* dt, double gamma, double b0x, double b0y, double b0z, int limiter, int lx,
               unsigned long long* bad, double* bflux, void* stream) {
  set_error("");
  int ty, tz;
  tile_shape_3d(shape_mode(precision), &ty, &tz);
  return stage3d(precision, src, base, dst, patches, tiles, ntiles, dt, gamma, b0x, b0y, b0z, limiter, lx, ty, tz,
                 bad, bflux, stream);
}

int wb_stage3d_tiled(int precision, const void* src, const void* base, void* dst, const void* patches,
                     const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y, double b0z,
                     int limiter, int lx, int ty, int tz, unsigned long long* bad, double* bflux, void* stream) {
  set_error("");
  return stage3d(precision, src, base, dst, patches, tiles, ntiles, dt, gamma, b0x, b0y, b0z, limiter, lx, ty, tz,
                 bad, bflux, stream);
}

int wb_stage3d_physics(int precision, const void* src, const void* base, void* dst, const void* patches,
                       const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y, double b0z,
                       int limiter, int lx, double eta, double gx, double gy, double gz, unsigned long long* bad,
                       void* stream) {
  set_error("");
  if (!precision_ok(precision, "stage3d_physics") ||
      !ptrs_ok({src, dst, patches, tiles, dt, bad}, "stage3d_physics"))
    return kBadArgument;
  if (ntiles < 0 || !(gamma > 1.0) || lx <= 0 || !(eta >= 0.0)) {
    set_error("stage3d_physics: ntiles must be >= 0, gamma > 1, lx > 0 and eta >= 0");
    return kBadArgument;
  }
  int ty, tz;  // the non-ideal kernel runs on the default tiles
  tile_shape_3d(shape_mode(precision), &ty, &tz);
  if (precision == 32) {
    StageArgs<float> a{static_cast<const float*>(src), static_cast<const float*>(base), static_cast<float*>(dst),
                       static_cast<const PatchDesc*>(patches), static_cast<const Tile*>(tiles), dt, gamma,
                       1.0 / (gamma - 1.0), {b0x, b0y, b0z}, bad, nullptr, lx};
    a.eta = eta, a.gravity[0] = gx, a.gravity[1] = gy, a.gravity[2] = gz;
    return launch_stage3d<float>(a, ntiles, limiter, ty, tz, as_stream(stream));
  }
  StageArgs<double> a{static_cast<const double*>(src), static_cast<const double*>(base), static_cast<double*>(dst),
                      static_cast<const PatchDesc*>(patches), static_cast<const Tile*>(tiles), dt, gamma,
                      1.0 / (gamma - 1.0), {b0x, b0y, b0z}, bad, nullptr, lx};
  a.eta = eta, a.gravity[0] = gx, a.gravity[1] = gy, a.gravity[2] = gz;
  return precision == 64 ? launch_stage3d<double, double>(a, ntiles, limiter, ty, tz, as_stream(stream))
                         : launch_stage3d<double, float>(a, ntiles, limiter, ty, tz, as_stream(stream));
}

int wb_tile_shape(int ndim, int precision, int* a, int* b) {
  set_error("");
  if (!precision_ok(precision, "tile_shape") || !a || !b || (ndim != 2 && ndim != 3)) {
    set_error("tile_shape: ndim must be 2 or 3 and outputs non-NULL");
    return kBadArgument;
  }
  if (ndim == 2)
    tile_shape_2d(shape_mode(precision), a, b);
  else
    tile_shape_3d(shape_mode(precision), a, b);
  return kOk;
}

int wb_rate(int precision, int ndim, const void* state, const void* patches, int npatches, const int* chunk_patch,
            const int* chunk_start, int nchunks, double b0x, double b0y, double b0z, double gamma,
            unsigned long long* keys, int ninstances, void* stream) {
  set_error("");
  if (!precision_ok(precision, "rate") || !ptrs_ok({state, patches, keys}, "rate")) return kBadArgument;
  if ((ndim != 2 && ndim != 3) || ninstances <= 0 || nchunks < 0 || (nchunks > 0 && (!chunk_patch || !chunk_start))) {
    set_error("rate: bad ndim / ninstances / work list");
    return kBadArgument;
  }
  const double b0[3] = {b0x, b0y, b0z};
  if (precision == 32)
    return launch_rate_chunks<float>(static_cast<const float*>(state), static_cast<const PatchDesc*>(patches), npatches,
                                     ndim, chunk_patch, chunk_start, nchunks, b0, gamma, keys, ninstances,
                                     as_stream(stream));
  return launch_rate_chunks<double>(static_cast<const double*>(state), static_cast<const PatchDesc*>(patches),
                                    npatches, ndim, chunk_patch, chunk_start, nchunks, b0, gamma, keys, ninstances,
                                    as_stream(stream));
}

int wb_finalize_dt(const unsigned long long* keys, int ninstances, double cfl, double eta, double kappa, double gamma,
                   const double* inv_dx2_sum, double* time, const double* end, double* dt, int advance, void* stream) {
  set_error("");
  if (!ptrs_ok({keys, inv_dx2_sum, dt}, "finalize_dt")) return kBadArgument;
  if ((end || advance) && !time) {
    set_error("finalize_dt: time is required with end or advance");
    return kBadArgument;
  }
  return launch_finalize_dt(keys, ninstances, cfl, eta, kappa, gamma, inv_dx2_sum, time, end, dt, advance,
                            as_stream(stream));
}

int wb_rate_levels(int precision, int ndim, const void* state, const void* patches, int npatches,
                   const int* chunk_patch, const int* chunk_start, int nchunks, double b0x, double b0y, double b0z,
                   double gamma, unsigned long long* keys, int ninstances, unsigned long long* level_keys,
                   int nlevels, void* stream) {
  set_error("");
  if (!precision_ok(precision, "rate_levels") || !ptrs_ok({state, patches, keys, level_keys}, "rate_levels"))
    return kBadArgument;
  if ((ndim != 2 && ndim != 3) || ninstances <= 0 || nlevels <= 0 || nchunks < 0 ||
      (nchunks > 0 && (!chunk_patch || !chunk_start))) {
    set_error("rate_levels: bad ndim / ninstances / nlevels / work list");
    return kBadArgument;
  }
  if (int64_t(ninstances) * nlevels >= (int64_t(1) << 31)) {
    set_error("rate_levels: %d instances x %d levels exceed 2^31 keys", ninstances, nlevels);
    return kTooLarge;
  }
  const double b0[3] = {b0x, b0y, b0z};
  if (precision == 32)
    return launch_rate_chunks<float>(static_cast<const float*>(state), static_cast<const PatchDesc*>(patches), npatches,
                                     ndim, chunk_patch, chunk_start, nchunks, b0, gamma, keys, ninstances,
                                     as_stream(stream), level_keys, nlevels);
  return launch_rate_chunks<double>(static_cast<const double*>(state), static_cast<const PatchDesc*>(patches),
                                    npatches, ndim, chunk_patch, chunk_start, nchunks, b0, gamma, keys, ninstances,
                                    as_stream(stream), level_keys, nlevels);
}

int wb_finalize_dt_levels(const unsigned long long* keys, int ninstances, double cfl, double eta, double kappa,
                          double gamma, const unsigned long long* level_keys, const double* inv_dx2_levels,
                          int nlevels, double* time, const double* end, double* dt, int advance, void* stream) {
  set_error("");
  if (!ptrs_ok({keys, level_keys, inv_dx2_levels, dt}, "finalize_dt_levels")) return kBadArgument;
  if (nlevels <= 0) {
    set_error("finalize_dt_levels: nlevels must be positive");
    return kBadArgument;
  }
  if ((end || advance) && !time) {
    set_error("finalize_dt_levels: time is required with end or advance");
    return kBadArgument;
  }
  return launch_finalize_dt(keys, ninstances, cfl, eta, kappa, gamma, nullptr, time, end, dt, advance,
                            as_stream(stream), level_keys, inv_dx2_levels, nlevels);
}

int wb_copy_ops(int precision, void* pool, const void* patches, const void* ops, int nops, void* stream) {
  set_error("");
  if (!precision_ok(precision, "copy_ops") || !ptrs_ok({pool, patches}, "copy_ops") || (nops > 0 && !ops))
    return kBadArgument;
  if (precision == 32)
    return launch_copy_ops<float>(static_cast<float*>(pool), static_cast<const PatchDesc*>(patches),
                                  static_cast<const CopyOp*>(ops), nops, as_stream(stream));
  return launch_copy_ops<double>(static_cast<double*>(pool), static_cast<const PatchDesc*>(patches),
                                 static_cast<const CopyOp*>(ops), nops, as_stream(stream));
}

int wb_interp_ops(int precision, void* pool, const void* patches, const void* ops, int nops, void* stream) {
  set_error("");
  if (!precision_ok(precision, "interp_ops") || !ptrs_ok({pool, patches}, "interp_ops") || (nops > 0 && !ops))
    return kBadArgument;
  if (precision == 32)
    return launch_interp_ops<float>(static_cast<float*>(pool), static_cast<const PatchDesc*>(patches),
                                    static_cast<const InterpOp*>(ops), nops, as_stream(stream));
  return launch_interp_ops<double>(static_cast<double*>(pool), static_cast<const PatchDesc*>(patches),
                                   static_cast<const InterpOp*>(ops), nops, as_stream(stream));
}

int wb_fill_ops(int precision, void* pool, const void* patches, const void* interp, int ninterp, const void* copies,
                int ncopies, void* stream) {
  set_error("");
  if (!precision_ok(precision, "fill_ops") || !ptrs_ok({pool, patches}, "fill_ops") || (ninterp > 0 && !interp) ||
      (ncopies > 0 && !copies) || ninterp < 0 || ncopies < 0)
    return kBadArgument;
  if (precision == 32)
    return launch_fill_ops<float>(static_cast<float*>(pool), static_cast<const PatchDesc*>(patches),
                                  static_cast<const InterpOp*>(interp), ninterp, static_cast<const CopyOp*>(copies),
                                  ncopies, as_stream(stream));
  return launch_fill_ops<double>(static_cast<double*>(pool), static_cast<const PatchDesc*>(patches),
                                 static_cast<const InterpOp*>(interp), ninterp, static_cast<const CopyOp*>(copies),
                                 ncopies, as_stream(stream));
}

int wb_restrict_ops(int precision, void* pool, const void* patches, const void* ops, int nops, void* stream) {
  set_error("");
  if (!precision_ok(precision, "restrict_ops") || !ptrs_ok({pool, patches}, "restrict_ops") || (nops > 0 && !ops))
    return kBadArgument;
  if (precision == 32)
    return launch_restrict_ops<float>(static_cast<float*>(pool), static_cast<const PatchDesc*>(patches),
                                      static_cast<const RestrictOp*>(ops), nops, as_stream(stream));
  return launch_restrict_ops<double>(static_cast<double*>(pool), static_cast<const PatchDesc*>(patches),
                                     static_cast<const RestrictOp*>(ops), nops, as_stream(stream));
}

static int face_flux_ops(int precision, const void* pool, const void* patches, const void* ops, int nops,
                         int nfaces, const double* b0, double gamma, int limiter, const double* physics,
                         const double* bflux, double* reg, void* stream) {
  if (!precision_ok(precision, "face_flux_ops") || (nops > 0 && !ptrs_ok({pool, patches, ops, reg}, "face_flux_ops")))
    return kBadArgument;
  if (limiter < 0 || limiter > 3) {
    set_error("face_flux_ops: limiter code %d is not one of 0..3", limiter);
    return kBadArgument;
  }
  if (precision == 32)
    return launch_face_flux_ops<float>(static_cast<const float*>(pool), static_cast<const PatchDesc*>(patches),
                                       static_cast<const FaceFluxOp*>(ops), nops, nfaces, b0, gamma, limiter, physics, bflux,
                                       reg, as_stream(stream));
  if (precision == kMath32State64)
    return launch_face_flux_ops<double, float>(static_cast<const double*>(pool), static_cast<const PatchDesc*>(patches),
                                               static_cast<const FaceFluxOp*>(ops), nops, nfaces, b0, gamma, limiter,
                                               physics, bflux, reg, as_stream(stream));
  return launch_face_flux_ops<double>(static_cast<const double*>(pool), static_cast<const PatchDesc*>(patches),
                                      static_cast<const FaceFluxOp*>(ops), nops, nfaces, b0, gamma, limiter, physics, bflux,
                                      reg, as_stream(stream));
}

int wb_face_flux_ops(int precision, const void* pool, const void* patches, const void* ops, int nops, double b0x,
                     double b0y, double b0z, double gamma, int limiter, double* reg, void* stream) {
  set_error("");
  const double b0[3] = {b0x, b0y, b0z};
  return face_flux_ops(precision, pool, patches, ops, nops, 0, b0, gamma, limiter, nullptr, nullptr, reg, stream);
}

int wb_face_flux_ops_staged(int precision, const void* pool, const void* patches, const void* ops, int nops,
                            int nfaces, double b0x, double b0y, double b0z, double gamma, int limiter,
                            const double* bflux, double* reg, void* stream) {
  set_error("");
  if (nops > 0 && (!bflux || nfaces < 0)) {
    set_error("face_flux_ops_staged: NULL boundary-face fluxes or a negative face count");
    return kBadArgument;
  }
  const double b0[3] = {b0x, b0y, b0z};
  return face_flux_ops(precision, pool, patches, ops, nops, nfaces, b0, gamma, limiter, nullptr, bflux, reg, stream);
}

int wb_face_flux_ops_physics(int precision, const void* pool, const void* patches, const void* ops, int nops,
                             double b0x, double b0y, double b0z, double gamma, int limiter, double eta,
                             double kappa_par, double kappa_perp, double* reg, void* stream) {
  set_error("");
  if (!(eta >= 0.0) || !(kappa_par >= 0.0) || !(kappa_perp >= 0.0)) {
    set_error("face_flux_ops_physics: eta %g, kappa_par %g, kappa_perp %g must be non-negative", eta, kappa_par,
              kappa_perp);
    return kBadArgument;
  }
  const double b0[3] = {b0x, b0y, b0z};
  const double physics[3] = {eta, kappa_par, kappa_perp};
  return face_flux_ops(precision, pool, patches, ops, nops, 0, b0, gamma, limiter, physics, nullptr, reg, stream);
}

int wb_reflux_apply(int precision, void* pool, const void* patches, const void* ops, int nops, double* reg,
                    const double* dt, void* stream) {
  set_error("");
  if (!precision_ok(precision, "reflux_apply") || (nops > 0 && !ptrs_ok({pool, patches, ops, reg, dt}, "reflux_apply")))
    return kBadArgument;
  if (precision == 32)
    return launch_reflux_apply<float>(static_cast<float*>(pool), static_cast<const PatchDesc*>(patches),
                                      static_cast<const RefluxOp*>(ops), nops, reg, dt, as_stream(stream));
  return launch_reflux_apply<double>(static_cast<double*>(pool), static_cast<const PatchDesc*>(patches),
                                     static_cast<const RefluxOp*>(ops), nops, reg, dt, as_stream(stream));
}

int wb_struct_sizes(int64_t* sizes_host, int n) {
  set_error("");
  if (!sizes_host || n < 7) {
    set_error("struct_sizes: needs room for 7 sizes (9 with the op-program structs)");
    return kBadArgument;
  }
  if (n >= 9) {
    sizes_host[7] = sizeof(wb_program_segment);
    sizes_host[8] = sizeof(wb_program_params);
  }
  sizes_host[0] = sizeof(PatchDesc);
  sizes_host[1] = sizeof(Tile);
  sizes_host[2] = sizeof(CopyOp);
  sizes_host[3] = sizeof(InterpOp);
  sizes_host[4] = sizeof(RestrictOp);
  sizes_host[5] = sizeof(FaceFluxOp);
  sizes_host[6] = sizeof(RefluxOp);
  return kOk;
}

}  // extern "C"
