// Op lists of the halo, restriction and reflux kernels (built by the host per layout).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "layout.cuh"

namespace wb {

// dst[d + p] = w1 * src1[s1 + m1 * p] + w2 * src2[s2 + m2 * p], p over the box n,
// fields [field_lo, field_hi), field `negate` negated. Indices are haloed patch indices.
// (every op: fewer than 2^31 points, fields within 0..7, no point both read and written)
struct CopyOp {
  int32_t dst, src1, src2;
  int32_t field_lo, field_hi, negate;
  int32_t n[3];
  int32_t d[3];
  int32_t s1[3], m1[3];
  int32_t s2[3], m2[3];
  double w1, w2;
};

// Fine halo box d .. d + n (haloed fine indices) interpolated from the coarse patch.
struct InterpOp {
  int32_t fine, coarse;
  int32_t field_lo, field_hi;
  int32_t node_mask;  // bit a: axis a is node-centred for these fields
  int32_t ndim;
  int32_t n[3];
  int32_t d[3];
  int32_t fine_lo[3];    // level index of the fine patch's first interior cell
  int32_t coarse_lo[3];  // level index of the coarse patch's first interior cell
};

// Coarse box c .. c + n (haloed coarse indices) from the fine values starting at f.
struct RestrictOp {
  int32_t fine, coarse;
  int32_t field_lo, field_hi;
  int32_t node_mask;
  int32_t ndim;
  int32_t n[3];
  int32_t c[3];
  int32_t f[3];
};

// One coarse-fine interface side: the coarse faces (haloed index coarse_plane along
// `axis` of the coarse patch, transverse start coarse_t0) and the fine faces over them
// (2 per coarse face along each transverse axis), accumulated into reg[reg_off ...].
struct FaceFluxOp {
  int32_t coarse, fine;
  int32_t ndim, axis, t1, t2;
  int32_t coarse_plane, fine_plane;
  int32_t coarse_t0[2], fine_t0[2];
  int32_t len, width;
  int32_t first;  // the op's first coarse face in the flat numbering of all ops' faces
  int32_t pad1;
  int64_t reg_off;
};

// Apply the register of one interface to the coarse cells beside it.
struct RefluxOp {
  int32_t coarse;
  int32_t len, width, ncomp;
  int32_t c[3];   // haloed index of the first coarse cell
  int32_t t1, t2; // transverse axes (t2 = -1 in 2D)
  int32_t field[8];
  double sign, dx;
  int64_t reg_off;
};

template <typename S>
int launch_copy_ops(S* pool, const PatchDesc* patches, const CopyOp* ops, int nops, cudaStream_t stream);
template <typename S>
int launch_interp_ops(S* pool, const PatchDesc* patches, const InterpOp* ops, int nops, cudaStream_t stream);
template <typename S>
int launch_fill_ops(S* pool, const PatchDesc* patches, const InterpOp* interp, int ninterp, const CopyOp* copies,
                    int ncopies, cudaStream_t stream);
template <typename S>
int launch_restrict_ops(S* pool, const PatchDesc* patches, const RestrictOp* ops, int nops, cudaStream_t stream);
// R: the arithmetic of the recomputed face fluxes (the stage kernels' for the state type S);
// bflux: the stage kernel's boundary-face fluxes (2D ideal: the fine faces read there), or null
template <typename S, typename R = S>
int launch_face_flux_ops(const S* pool, const PatchDesc* patches, const FaceFluxOp* ops, int nops, int nfaces,
                         const double* b0, double gamma, int limiter, const double* physics, const double* bflux,
                         double* reg, cudaStream_t stream);
template <typename S>
int launch_reflux_apply(S* pool, const PatchDesc* patches, const RefluxOp* ops, int nops, double* reg,
                        const double* dt, cudaStream_t stream);

}  // namespace wb
