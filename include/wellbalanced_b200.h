/*
 * wellbalanced_b200 — C ABI of the B200 ideal-MHD step (libwb200.so).
 *
 * Every pointer argument is a DEVICE pointer unless its name ends in `_host`; arrays are
 * C-contiguous (row-major, the last index fastest). `stream` is a cudaStream_t (NULL:
 * the legacy default stream). Functions return 0 on success or a negative status
 * (WB_BAD_ARGUMENT, WB_CUDA_ERROR, WB_UNSUPPORTED, WB_TOO_LARGE); wb_last_error() then
 * describes the failure (thread-local). Nothing here allocates device memory except
 * where a function says so.
 *
 * Two groups of entry points:
 *
 *  1. The reference's six block kernels, same arguments and out-parameter convention
 *     as `carafe.kernels.<name>.kernel` (float64, one haloed block of X x Y cells):
 *     the drop-in for the cunumpy kernel slot of carafe/kernels/<name>/__init__.py:9-10.
 *
 *  2. The fused engine used by the whole-step path (MHD2D / MHD3D): stage kernels over
 *     a device work list of patch tiles, the per-step rate / dt reduction, and the
 *     halo / restriction / flux-register op lists. Structs are laid out as in
 *     wellbalanced_b200/csrc/layout.cuh and halo.cuh (mirrored by the Python host).
 */
#ifndef WELLBALANCED_B200_H
#define WELLBALANCED_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WB_OK 0
#define WB_BAD_ARGUMENT (-1)
#define WB_CUDA_ERROR (-2)
#define WB_UNSUPPORTED (-3)
#define WB_TOO_LARGE (-4)

/* Version string of the library. */
const char* wb_version(void);
/* Text of the last failure on the calling thread ("" if none). */
const char* wb_last_error(void);

/* ---- 1. the reference's block kernels (float64) ------------------------------------ */

/* carafe/kernels/mhd_primitive/mhd_primitive_pyccel.py:23-87 — mhd_primitive(rho, mx, my,
 * mz, energy, bz, az, dx, dy, b0x, b0y, gamma, prim, bxf, byf, ecc) -> int.
 * Cells (X, Y); az (X+1, Y+1); prim (8, X, Y); bxf (X+1, Y); byf (X, Y+1); ecc (X, Y).
 * The bad-cell count is ADDED to *bad (a device counter the caller zeroes); the
 * reference returns it. */
int wb_mhd_primitive(const double* rho, const double* mx, const double* my, const double* mz,
                     const double* energy, const double* bz, const double* az, int64_t X, int64_t Y,
                     double dx, double dy, double b0x, double b0y, double gamma, double* prim,
                     double* bxf, double* byf, double* ecc, unsigned long long* bad, void* stream);

/* carafe/kernels/mhd_sweep/mhd_sweep_pyccel.py:254-319 — mhd_sweep(prim, bn, axis, limiter,
 * gamma, flux). prim (8, X, Y); bn (X+1, Y) for axis 0, (X, Y+1) for axis 1; flux
 * (7, X-3, Y) or (7, X, Y-3). limiter: 0 minmod, 1 vanleer, 2 mc, 3 none. */
int wb_mhd_sweep(const double* prim, const double* bn, int axis, int limiter, double gamma, int64_t X,
                 int64_t Y, double* flux, void* stream);

/* carafe/kernels/ct_contact/ct_contact_pyccel.py:26-61 — ct_contact(fx_by, gy_bx, fx_rho,
 * gy_rho, ecc, ez). fx_* (X-3, Y); gy_* (X, Y-3); ecc (X, Y); ez (na, nb). */
int wb_ct_contact(const double* fx_by, const double* gy_bx, const double* fx_rho, const double* gy_rho,
                  const double* ecc, int64_t X, int64_t Y, int64_t na, int64_t nb, double* ez, void* stream);

/* The per-plane ct_contact calls of carafe/mhd3d.py:544-557 (MHD3D._edge_field) in one
 * launch: `planes` stacked blocks, plane q of each array at q times its plane size
 * (fx_* (planes, X-3, Y), gy_* (planes, X, Y-3), ecc (planes, X, Y), ez (planes, na, nb)). */
int wb_ct_contact_planes(const double* fx_by, const double* gy_bx, const double* fx_rho, const double* gy_rho,
                         const double* ecc, int64_t X, int64_t Y, int64_t na, int64_t nb, int64_t planes, double* ez,
                         void* stream);

/* carafe/kernels/mhd_rate/mhd_rate_pyccel.py:30-83 — mhd_rate(rho, mx, my, mz, energy, bz, az,
 * halo, dx, dy, b0x, b0y, gamma, out). out: device double[2] = (largest rate, smallest rho). */
int wb_mhd_rate(const double* rho, const double* mx, const double* my, const double* mz,
                const double* energy, const double* bz, const double* az, int64_t X, int64_t Y, int halo,
                double dx, double dy, double b0x, double b0y, double gamma, double* out, void* stream);

/* carafe/kernels/mhd_resistive/mhd_resistive_pyccel.py:21-67 — mhd_resistive(prim, bxf, byf,
 * dx, dy, eta, fx, fy, ez): adds the resistive terms in place. */
int wb_mhd_resistive(const double* prim, const double* bxf, const double* byf, int64_t X, int64_t Y,
                     double dx, double dy, double eta, double* fx, double* fy, double* ez, void* stream);

/* carafe/kernels/mhd_conductive/mhd_conductive_pyccel.py:38-100 — mhd_conductive(prim, bxf,
 * byf, dx, dy, parallel, perpendicular, fx, fy): subtracts the heat flux in place. */
int wb_mhd_conductive(const double* prim, const double* bxf, const double* byf, int64_t X, int64_t Y,
                      double dx, double dy, double parallel, double perpendicular, double* fx, double* fy,
                      void* stream);

/* ---- 2. the fused engine -------------------------------------------------------------- */

/* One RK stage of every tile in `tiles` (struct Tile[ntiles]) of the patches in `patches`
 * (struct PatchDesc[]), replacing carafe/mhd.py:889-927 (_advance) for MHD2D and
 * carafe/mhd3d.py:635-671 for MHD3D, with the Heun combine of mhd.py:983-988:
 *   base == NULL: dst = src - dt L(src);   else dst = (src - dt L(src) + base) / 2.
 * `precision`: 32 (float state and arithmetic), 64 (double state and arithmetic) or
 * WB_MATH32_STATE64 (a double state advanced with float arithmetic: primitive variables
 * and face fields formed in double and rounded to float, reconstruction / HLLD / CT in
 * float, flux differences and the updates of U, A and the Heun combine in double);
 * src/base/dst are pools of the state's type. */
#define WB_MATH32_STATE64 6432
/*
 * dt: device double per instance. bad: device counter of bad cells (added to).
 * bflux: device double array of boundary-face fluxes (NULL to skip).
 * lx (3D only): cell planes per tile along x. */
int wb_stage2d(int precision, const void* src, const void* base, void* dst, const void* patches,
               const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y,
               int limiter, unsigned long long* bad, double* bflux, void* stream);
int wb_stage3d(int precision, const void* src, const void* base, void* dst, const void* patches,
               const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y,
               double b0z, int limiter, int lx, unsigned long long* bad, double* bflux, void* stream);

/* wb_stage2d with the reference's non-ideal terms in the same pass (carafe/mhd.py:844-927):
 * resistivity eta (carafe/kernels/mhd_resistive/mhd_resistive_pyccel.py:21-67), Braginskii
 * conduction along / across the field (mhd_conductive_pyccel.py:38-100) and gravity
 * (gx, gy); all zero gives the ideal kernel. */
int wb_stage2d_physics(int precision, const void* src, const void* base, void* dst, const void* patches,
                       const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y,
                       int limiter, double eta, double kappa_par, double kappa_perp, double gx, double gy,
                       unsigned long long* bad, void* stream);

/* wb_stage3d with the reference's resistivity and gravity in the same pass
 * (carafe/mhd3d.py:561-600, 639-671): E += eta J on every edge and eta (J x B) on every
 * face's energy flux, J = curl B on the edges from the face fields and B the mean of the
 * four faces around each face; rho g and m . g on the cells. All zero gives the ideal
 * kernel. */
int wb_stage3d_physics(int precision, const void* src, const void* base, void* dst, const void* patches,
                       const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y,
                       double b0z, int limiter, int lx, double eta, double gx, double gy, double gz,
                       unsigned long long* bad, void* stream);

/* wb_stage2d on a work list cut into tx x ty tiles, one of the shapes wb_tile_shapes lists
 * (no counterpart in the reference: the tile shape is this implementation's schedule,
 * picked by the autotuner). Ideal MHD; the non-ideal kernel runs on the default shape. */
int wb_stage2d_tiled(int precision, const void* src, const void* base, void* dst, const void* patches,
                     const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y,
                     int limiter, int tx, int ty, unsigned long long* bad, double* bflux, void* stream);

/* wb_stage3d on a work list cut into ty x tz columns, one of the shapes wb_tile_shapes
 * lists (no counterpart in the reference: the autotuner's schedule). Ideal MHD; the
 * non-ideal kernel runs on the default shape. */
int wb_stage3d_tiled(int precision, const void* src, const void* base, void* dst, const void* patches,
                     const void* tiles, int ntiles, const double* dt, double gamma, double b0x, double b0y,
                     double b0z, int limiter, int lx, int ty, int tz, unsigned long long* bad, double* bflux,
                     void* stream);

/* Tile shape of the stage kernels: 2D (TX, TY); 3D (TY, TZ). */
int wb_tile_shape(int ndim, int precision, int* a, int* b);

/* The tile shapes the 2D / 3D stage kernel is built for: up to `max` pairs ((tx, ty) in
 * 2D, (ty, tz) in 3D) into shapes[2 * i], shapes[2 * i + 1], the default first; returns
 * how many there are. */
int wb_tile_shapes(int ndim, int precision, int* shapes, int max);

/* Per-instance max fast-wave rate and min density (carafe/mhd.py:930-963,
 * carafe/mhd3d.py:674-724) as order-preserving keys: keys[2i], keys[2i+1]. Work list:
 * chunk_patch[c], chunk_start[c] (up to 2048 cells per chunk). */
int wb_rate(int precision, int ndim, const void* state, const void* patches, int npatches,
            const int* chunk_patch, const int* chunk_start, int nchunks, double b0x, double b0y, double b0z,
            double gamma, unsigned long long* keys, int ninstances, void* stream);

/* dt[i] = cfl * min(1 / rate_i, 0.5 / (D_i * inv_dx2_sum[i])), D_i = max(eta, (gamma - 1)
 * kappa / min rho_i); with end != NULL clipped to end[i] - time[i] (0 once reached);
 * advance != 0 adds dt[i] to time[i]. */
int wb_finalize_dt(const unsigned long long* keys, int ninstances, double cfl, double eta, double kappa,
                   double gamma, const double* inv_dx2_sum, double* time, const double* end, double* dt,
                   int advance, void* stream);

/* wb_rate that also reduces the smallest density of every (instance, level):
 * level_keys[instance * nlevels + level] (order-preserving keys, nlevels * ninstances).
 * With wb_finalize_dt_levels it takes the diffusion limit level by level, each level's
 * smallest density with that level's spacing, as carafe/mhd.py:942-960 does patch by
 * patch (patches of one level share their spacing). A patch whose instance or level lies
 * outside the key arrays is skipped (as in wb_rate). */
int wb_rate_levels(int precision, int ndim, const void* state, const void* patches, int npatches,
                   const int* chunk_patch, const int* chunk_start, int nchunks, double b0x, double b0y,
                   double b0z, double gamma, unsigned long long* keys, int ninstances,
                   unsigned long long* level_keys, int nlevels, void* stream);
/* wb_finalize_dt with the diffusion limit min over levels l of 0.5 / (D_l * inv_dx2_levels[i
 * * nlevels + l]), D_l = max(eta, (gamma - 1) kappa / min rho of level l); levels with
 * inv_dx2_levels 0 hold no patch of the instance and are skipped. */
int wb_finalize_dt_levels(const unsigned long long* keys, int ninstances, double cfl, double eta, double kappa,
                          double gamma, const unsigned long long* level_keys, const double* inv_dx2_levels,
                          int nlevels, double* time, const double* end, double* dt, int advance, void* stream);

/* Halo and restriction op lists (struct CopyOp / InterpOp / RestrictOp), replacing
 * patchwork's exchange_halos and restrict (carafe/mhd.py:744-777, 981, 991). An op covers
 * fewer than 2^31 points of fields 0..7, and never writes a point it reads. One 64-thread
 * block runs one op: lists of small ops (64 points or fewer) run in one wave, and large
 * boxes are best cut into ops of up to ~1024 points (wellbalanced_b200.mesh.size_ops). */
int wb_copy_ops(int precision, void* pool, const void* patches, const void* ops, int nops, void* stream);
int wb_interp_ops(int precision, void* pool, const void* patches, const void* ops, int nops, void* stream);
int wb_restrict_ops(int precision, void* pool, const void* patches, const void* ops, int nops, void* stream);
/* wb_interp_ops and wb_copy_ops of one level in a single launch. Valid only when no op of
 * the two lists writes a point another op of them writes or reads: the interpolation ops
 * cover just the halo points no same-level copy fills (wellbalanced_b200.mesh.Layout builds
 * them so), and the copies read only their sources' computed points. */
int wb_fill_ops(int precision, void* pool, const void* patches, const void* interp, int ninterp, const void* copies,
                int ncopies, void* stream);

/* Refluxing, replacing patchwork's FluxRegister (carafe/mhd.py:906-919, 989-990): after
 * a stage, reg += (mean of the fine faces - the coarse face) of every coarse-fine
 * interface face, recomputed from the stage's input pool (struct FaceFluxOp); after the
 * step, the coarse cells beside the interfaces take U -= sign * 0.5 dt * reg / dx and reg
 * is cleared (struct RefluxOp; dt per instance on the device). The ops of one
 * wb_reflux_apply call run concurrently and must not share a coarse cell: a cell between
 * fine patches takes its corrections from separate calls (per axis and side, or grouped so
 * that no call holds two ops of one cell, as wellbalanced_b200.mesh.Layout does). */
int wb_face_flux_ops(int precision, const void* pool, const void* patches, const void* ops, int nops, double b0x,
                     double b0y, double b0z, double gamma, int limiter, double* reg, void* stream);
/* The same register update for 2D ideal MHD with the fine faces read from `bflux`, the
 * boundary-face fluxes the stage kernel of that stage wrote (wb_stage2d's bflux argument,
 * float64 rows per patch at PatchDesc.bflux: for x then y, side (low, high), conserved row,
 * face along the side); only the coarse faces are recomputed, one thread per coarse face of
 * all ops: each op's FaceFluxOp.first holds its first face in that flat numbering (the
 * prefix sum of the ops' lengths, in list order) and nfaces their total. The fluxes read are those the
 * fine cells were advanced with: with float32 face arithmetic the register equals
 * wb_face_flux_ops' bit for bit, in float64 to rounding.
 * No counterpart in the reference (whose register records the fluxes as its sweeps form
 * them). 3D ops and non-ideal terms are not read from bflux: use wb_face_flux_ops(_physics). */
int wb_face_flux_ops_staged(int precision, const void* pool, const void* patches, const void* ops, int nops,
                            int nfaces, double b0x, double b0y, double b0z, double gamma, int limiter,
                            const double* bflux, double* reg, void* stream);
/* The same register update with the non-ideal face terms of wb_stage2d_physics /
 * wb_stage3d_physics: each recomputed face flux carries the resistive terms (and, in 2D,
 * the Braginskii heat flux), as the reference's fluxes do when its register records them
 * (carafe/mhd.py:866-872, 906-919; carafe/mhd3d.py:630-632). 3D interfaces take eta only
 * (the reference's MHD3D has no conduction). */
int wb_face_flux_ops_physics(int precision, const void* pool, const void* patches, const void* ops, int nops,
                             double b0x, double b0y, double b0z, double gamma, int limiter, double eta,
                             double kappa_par, double kappa_perp, double* reg, void* stream);
int wb_reflux_apply(int precision, void* pool, const void* patches, const void* ops, int nops, double* reg,
                    const double* dt, void* stream);

/* ---- 3. op programs ------------------------------------------------------------------ */

/* The small-op phases between two stage kernels of a refined step in one launch: reflux
 * (wb_reflux_apply), restriction (wb_restrict_ops), the halo fill of every level
 * (wb_fill_ops / wb_copy_ops) and the stable step (wb_rate, wb_finalize_dt): patchwork's
 * exchange_halos, FluxRegister.reflux and restrict, and stable_step, as
 * carafe/mhd.py:889-994 (and carafe/mhd3d.py:635-754) call them between and after the
 * stages. The register's face fluxes (wb_face_flux_ops) keep their own launch. A program
 * is a list of segments, each one op list of one kind on one of two pools; the segments
 * of one phase run together (their ops must touch disjoint points), the phases one after
 * the other. Each item runs the arithmetic of the standalone kernel of its kind, so the
 * results are those of the standalone launches, bit for bit. `counters`: device array of
 * 3 + (phases) unsigned words, zero before the first call; every call leaves them zero
 * except word 2, the error bits (2: a phase wait ran out after a second; 1: a rate chunk's
 * instance or level lay outside the keys), which the caller reads and clears. Calls that
 * share one `counters` array must not overlap on the GPU. `segments` and `params` are host
 * memory (copied into the launch); the op records, work lists, pools and the arrays
 * `params` points at are device memory. */
#define WB_PROGRAM_MAX_SEGMENTS 64
enum {
  WB_SEG_COPY = 0,        /* ops: struct CopyOp[count] */
  WB_SEG_INTERP = 1,      /* ops: struct InterpOp[count] */
  WB_SEG_RESTRICT = 2,    /* ops: struct RestrictOp[count] */
  WB_SEG_REFLUX = 3,      /* ops: struct RefluxOp[count]; params: reg, dt */
  WB_SEG_INIT_KEYS = 4,   /* one item: the keys' (and level keys') reduction identities */
  WB_SEG_RATE = 5,        /* ops: int chunk_patch[count], aux: int chunk_start[count] (as wb_rate) */
  WB_SEG_FINALIZE_DT = 6, /* one item: wb_finalize_dt (wb_finalize_dt_levels when level_keys is set) */
  WB_SEG_ADVANCE_TIME = 7 /* one item: time[i] += dt[i] */
};
typedef struct wb_program_segment {
  int32_t kind;  /* WB_SEG_* */
  int32_t pool;  /* 0: pool0, 1: pool1 */
  int32_t phase; /* 0 for the first segment, then equal to or one above the previous one */
  int32_t count; /* items */
  int32_t first; /* set by wb_run_program */
  int32_t pad;   /* set by wb_run_program (ops per work item) */
  const void* ops;
  const void* aux;
} wb_program_segment;
typedef struct wb_program_params {
  double b0[3];
  double gamma;
  double cfl, dt_eta, dt_kappa; /* the stable step's cfl, resistivity and conductivity */
  int32_t ndim, ninstances, nlevels, advance;
  double* reg;
  double* dt;
  double* time;
  const double* end;
  unsigned long long* keys;
  unsigned long long* level_keys; /* NULL: one density minimum per instance */
  const double* inv_dx2_sum;
  const double* inv_dx2_levels;
} wb_program_params;
int wb_run_program(int precision, void* pool0, void* pool1, const void* patches, const wb_program_segment* segments,
                   int nsegments, const wb_program_params* params, unsigned* counters, void* stream);

/* ---- 4. regrid on the device ---------------------------------------------------------- */

/* The plain refinement tagger, replacing the per-patch loops of carafe/mhd.py:1011-1041
 * (|J_z| at the cell's four nodes, averaged, times max(dx, dy)) and carafe/mhd3d.py:771-801
 * (|curl B| of the cell field by central differences, times max(dx, dy, dz)): every cell of
 * the patches below level `levels`, in float64 from the stored state, over the rate work
 * list (chunks of 2048 cells). A tagged cell sets tags[base + i s0 + j s1 + k] = 1 (2D:
 * base + i s0 + j) with {int64 base, s0, s1} of its patch in `place` (device, one record
 * per patch); the caller zeroes `tags` (the levels' dense arrays) first. */
int wb_current_tags(int precision, int ndim, const void* pool, const void* patches, const int* chunk_patch,
                    const int* chunk_start, int nchunks, const void* place, int levels, double b0x, double b0y,
                    double b0z, double threshold, unsigned char* tags, void* stream);
/* The state transfer of a regrid (patchwork's AMRHierarchy.regrid as carafe/mhd.py:1043-1056
 * calls it), level by level on the new hierarchy's pool:
 * - wb_prolong_ops: the new fine patches from the new coarser level (struct ProlongOp of
 *   csrc/transfer.cu: fine, coarse, field range, node mask, ndim, n[3], d[3] haloed fine
 *   start, fine_lo[3], coarse_lo[3] level indices, coarse_n[3] level shape, periodic mask):
 *   cells minmod-limited (children c -/+ s/4 per axis), potentials linear along node axes;
 * - wb_kept_ops: the points an old patch of the same level held, from the old pool (struct
 *   CopyOp: dst a new patch, src1 an old patch in old_patches, unit weights and strides);
 * - wb_positivity_ops: after both, every prolonged parent (struct PositivityOp of
 *   csrc/transfer.cu: fine, coarse, ndim, pad, n[3] parents, f0[3] haloed first child,
 *   c0[3] haloed first parent) whose children include a non-positive density or pressure
 *   gives them its density, momentum (2D: B_z) and an energy that keeps the pressure
 *   positive: E + M_i - mean(M) while that pressure is positive (the integral kept), else
 *   p / (gamma - 1) + K + M_i (M_i a child's magnetic energy from the fine potential). No
 *   counterpart in the reference, whose transfer leaves such children to fail the next
 *   step's check; elsewhere the transfer is unchanged. */
int wb_prolong_ops(int precision, void* pool, const void* patches, const void* ops, int nops, void* stream);
int wb_kept_ops(int precision, void* pool, const void* patches, const void* old_pool, const void* old_patches,
                const void* ops, int nops, void* stream);
int wb_positivity_ops(int precision, void* pool, const void* patches, const void* ops, int nops, double b0x,
                      double b0y, double b0z, double gamma, void* stream);

/* Sizes of the engine structs, for callers that mirror them: PatchDesc, Tile, CopyOp,
 * InterpOp, RestrictOp, FaceFluxOp, RefluxOp, and with n >= 9 wb_program_segment and
 * wb_program_params. */
int wb_struct_sizes(int64_t* sizes_host, int n);

/* Learned refinement tagger. No counterpart in the reference: it predicts the cells the
 * current tagger (|J| dx > threshold, carafe/mhd3d.py:771-801) flags a few steps ahead.
 * Parameters are one float32 vector of 5313 values (W1 [64][16] | b1 | W2 [64][64] | b2 |
 * W3 [64] | b3); the kernels use them rounded to bfloat16, with float32 accumulation.
 * - wb_tag_features: 16 stencil features of every interior cell of the 3D patches of a
 *   pool, written as float32 rows out[(row_start[p] + t) * 16 + c] (t the cell's index
 *   in (i, j, k) order), normalised as (f - mean[c]) * inv_std[c]; work list as wb_rate;
 * - wb_mlp_forward: logits of n feature rows (tensor-core mma, bf16 x float32);
 * - wb_mlp_backward: adds the gradient of the summed weighted binary cross-entropy
 *   (weight pos_weight where targets[r] = 1) to grads and the loss to *loss;
 * - wb_mlp_adam: one Adam step with the gradients scaled by `scale`; clears grads. */
int wb_tag_features(int precision, const void* pool, const void* patches, const int* chunk_patch,
                    const int* chunk_start, int nchunks, const int64_t* row_start, double b0x, double b0y,
                    double b0z, double gamma, const float* mean, const float* inv_std, float* out, void* stream);
int wb_mlp_forward(const float* features, int64_t n, const float* params, float* logits, void* stream);
int wb_mlp_backward(const float* features, const float* targets, int64_t n, const float* params, float pos_weight,
                    float* grads, double* loss, void* stream);
int wb_mlp_adam(float* params, float* grads, float* m, float* v, int count, float lr, float beta1, float beta2,
                float eps, int step, float scale, void* stream);

/* wb_rate without a caller-provided key buffer: allocates nothing. No counterpart in the
 * reference (its rate kernel returns into a caller-allocated out[2]). Same work list and
 * state as wb_rate; the per-instance keys live in a static device array of 4096
 * instances (64 KiB per device), and the result is decoded into `out` (device float64,
 * 2 * ninstances): out[2k] = largest rate, out[2k+1] = smallest density of instance k.
 * - ninstances > 4096 returns WB_TOO_LARGE with a message (use wb_rate for more);
 * - a patch whose instance index is not below ninstances is skipped and makes every
 *   value of `out` NaN (a call that cannot give the rate of every instance gives none);
 * - nothing must start at zero: each call initialises the slots it uses;
 * - the first call on a device resolves the scratch address (cudaGetSymbolAddress) and
 *   caches it; make that call before any stream capture that includes this function;
 *   the cached address belongs to the device's primary context and does not survive
 *   cudaDeviceReset (do not call this function after a reset in the same process);
 * - all calls on a device share the scratch: calls in flight at the same time (other
 *   streams, other threads) race and may return wrong values. */
int wb_rate_static(int precision, int ndim, const void* state, const void* patches, int npatches,
                   const int* chunk_patch, const int* chunk_start, int nchunks, double b0x, double b0y,
                   double b0z, double gamma, int ninstances, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WELLBALANCED_B200_H */
