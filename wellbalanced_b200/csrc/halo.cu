// Halo filling, restriction and refluxing on the patch pool, driven by op lists the
// host derives from the patch layout once per regrid.
//
// * Affine copy ops fill halos: dst[d + p] = w1 * src1[s1 + m1 * p] + w2 * src2[s2 + m2 * p]
//   over a box p of points, for a range of fields, with an optional negated field. They
//   express same-level copies and periodic images (w1 = 1, m1 = 1), zero-gradient
//   outflow cells (m = 0 along the normal), mirrored wall cells (m = -1, the normal
//   momentum negated), the linear extrapolation of outflow potentials and the odd
//   reflection of wall potentials (two sources) — carafe/mhd.py:298-353, 744-777.
// * Interpolation ops fill fine halos from the coarse patch below: linear along
//   cell-centred axes, coincident-or-4-point-midpoint along node axes.
// * Restriction ops set coarse values under fine patches: the mean of the fine values
//   along cell-centred axes, the coincident fine value along node axes.
//
// One block of 64 threads runs one op, its threads over the op's points: 32 such blocks
// are resident per SM, so a level's many small halo ops (tens of points each) run in one
// wave. The host cuts boxes into ops sized for the list (rows along the contiguous axis
// first): one point per thread where the list is small, up to 1024 points per op where
// it fills the GPU many times over. A thread issues every load of its point (all fields,
// all interpolation weights) before any store: the stores go through the same pool
// pointer, so loads placed after a store would wait for it.
#include "layout.cuh"
#include "halo.cuh"
#include "ops.cuh"
#include "wb_internal.cuh"

namespace wb {

template <typename S>
__global__ void __launch_bounds__(kOpThreads) copy_ops_kernel(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                                             const CopyOp* __restrict__ ops) {
  copy_op_pairs(pool, patches, ops[blockIdx.x]);
}

template <typename S>
__global__ void __launch_bounds__(kOpThreads) interp_ops_kernel(S* __restrict__ pool,
                                                               const PatchDesc* __restrict__ patches,
                                                               const InterpOp* __restrict__ ops) {
  interp_op(pool, patches, ops[blockIdx.x]);
}

// A level's interpolation and same-level copy ops in one launch (blocks [0, ninterp) the
// interpolation ops, the rest the copies): valid when no op of either list writes a point
// that another op of the launch writes or reads, as for interpolation ops trimmed to the
// halo points no sibling covers (the copies read only their sources' computed points).
template <typename S>
__global__ void __launch_bounds__(kOpThreads) fill_ops_kernel(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                                             const InterpOp* __restrict__ interp, int ninterp,
                                                             const CopyOp* __restrict__ copies) {
  if (int(blockIdx.x) < ninterp)
    interp_op(pool, patches, interp[blockIdx.x]);
  else
    copy_op(pool, patches, copies[blockIdx.x - ninterp]);
}

template <typename S>
__global__ void __launch_bounds__(kOpThreads) restrict_ops_kernel(S* __restrict__ pool,
                                                                 const PatchDesc* __restrict__ patches,
                                                                 const RestrictOp* __restrict__ ops) {
  restrict_op(pool, patches, ops[blockIdx.x]);
}

template <typename S>
int launch_copy_ops(S* pool, const PatchDesc* patches, const CopyOp* ops, int nops, cudaStream_t stream) {
  if (nops > 0) copy_ops_kernel<S><<<nops, kOpThreads, 0, stream>>>(pool, patches, ops);
  return check_launch("halo copy");
}
template <typename S>
int launch_interp_ops(S* pool, const PatchDesc* patches, const InterpOp* ops, int nops, cudaStream_t stream) {
  if (nops > 0) interp_ops_kernel<S><<<nops, kOpThreads, 0, stream>>>(pool, patches, ops);
  return check_launch("halo interpolation");
}
template <typename S>
int launch_fill_ops(S* pool, const PatchDesc* patches, const InterpOp* interp, int ninterp, const CopyOp* copies,
                    int ncopies, cudaStream_t stream) {
  if (ninterp + ncopies > 0)
    fill_ops_kernel<S><<<ninterp + ncopies, kOpThreads, 0, stream>>>(pool, patches, interp, ninterp, copies);
  return check_launch("halo fill");
}

template <typename S>
int launch_restrict_ops(S* pool, const PatchDesc* patches, const RestrictOp* ops, int nops, cudaStream_t stream) {
  if (nops > 0) restrict_ops_kernel<S><<<nops, kOpThreads, 0, stream>>>(pool, patches, ops);
  return check_launch("restrict");
}
template int launch_copy_ops<float>(float*, const PatchDesc*, const CopyOp*, int, cudaStream_t);
template int launch_copy_ops<double>(double*, const PatchDesc*, const CopyOp*, int, cudaStream_t);
template int launch_interp_ops<float>(float*, const PatchDesc*, const InterpOp*, int, cudaStream_t);
template int launch_interp_ops<double>(double*, const PatchDesc*, const InterpOp*, int, cudaStream_t);
template int launch_fill_ops<float>(float*, const PatchDesc*, const InterpOp*, int, const CopyOp*, int, cudaStream_t);
template int launch_fill_ops<double>(double*, const PatchDesc*, const InterpOp*, int, const CopyOp*, int,
                                     cudaStream_t);
template int launch_restrict_ops<float>(float*, const PatchDesc*, const RestrictOp*, int, cudaStream_t);
template int launch_restrict_ops<double>(double*, const PatchDesc*, const RestrictOp*, int, cudaStream_t);

}  // namespace wb
