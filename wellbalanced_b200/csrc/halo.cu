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
#include "wb_internal.cuh"

namespace wb {

// element offset of haloed index (i, j, k) of a patch (k ignored in 2D)
__device__ __forceinline__ int64_t offset_of(const PatchDesc& P, int i, int j, int k) {
  if (P.pitch1) return int64_t(i) * P.pitch0 + int64_t(j) * P.pitch1 + k;
  return int64_t(i) * P.pitch0 + j;
}

constexpr int kOpThreads = 64;  // threads of the block that runs one op

// The points of one copy op, over the threads of the block.
template <typename S>
__device__ __forceinline__ void copy_op(S* __restrict__ pool, const PatchDesc* __restrict__ patches, const CopyOp& op) {
  const PatchDesc D = patches[op.dst];
  const PatchDesc A = patches[op.src1];
  const PatchDesc B = patches[op.src2 >= 0 ? op.src2 : op.src1];
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = threadIdx.x; t < count; t += kOpThreads) {
    const unsigned line = t / n2;
    const int p2 = int(t - line * n2);
    const int p1 = int(line % n1);
    const int p0 = int(line / n1);
    const int64_t od = offset_of(D, op.d[0] + p0, op.d[1] + p1, op.d[2] + p2);
    const int64_t o1 = offset_of(A, op.s1[0] + op.m1[0] * p0, op.s1[1] + op.m1[1] * p1, op.s1[2] + op.m1[2] * p2);
    const int64_t o2 = offset_of(B, op.s2[0] + op.m2[0] * p0, op.s2[1] + op.m2[1] * p1, op.s2[2] + op.m2[2] * p2);
    // every field's value first, then the stores (an op never writes a point it reads)
    S v[8];
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      if (f >= op.field_lo && f < op.field_hi) {
        S x = S(op.w1) * pool[A.off + f * A.fstride + o1];
        if (op.w2 != 0.0) x += S(op.w2) * pool[B.off + f * B.fstride + o2];
        v[f] = f == op.negate ? -x : x;
      }
    }
#pragma unroll
    for (int f = 0; f < 8; ++f)
      if (f >= op.field_lo && f < op.field_hi) pool[D.off + f * D.fstride + od] = v[f];
  }
}

// The points of one copy op, two per thread and pass (the loads of both, every field,
// before the stores; an op never writes a point it reads): for the standalone copy
// launches, whose ops are large where the lists are (a big box's halos).
template <typename S>
__device__ __forceinline__ void copy_op_pairs(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                              const CopyOp& op) {
  const PatchDesc D = patches[op.dst];
  const PatchDesc A = patches[op.src1];
  const PatchDesc B = patches[op.src2 >= 0 ? op.src2 : op.src1];
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t0 = threadIdx.x; t0 < count; t0 += 2 * kOpThreads) {
    S v[2][8];
    int64_t od[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const unsigned t = t0 + u * kOpThreads;
      if (t >= count) continue;
      const unsigned line = t / n2;
      const int p2 = int(t - line * n2);
      const int p1 = int(line % n1);
      const int p0 = int(line / n1);
      od[u] = offset_of(D, op.d[0] + p0, op.d[1] + p1, op.d[2] + p2);
      const int64_t o1 = offset_of(A, op.s1[0] + op.m1[0] * p0, op.s1[1] + op.m1[1] * p1, op.s1[2] + op.m1[2] * p2);
      const int64_t o2 = offset_of(B, op.s2[0] + op.m2[0] * p0, op.s2[1] + op.m2[1] * p1, op.s2[2] + op.m2[2] * p2);
#pragma unroll
      for (int f = 0; f < 8; ++f) {
        if (f >= op.field_lo && f < op.field_hi) {
          S x = S(op.w1) * pool[A.off + f * A.fstride + o1];
          if (op.w2 != 0.0) x += S(op.w2) * pool[B.off + f * B.fstride + o2];
          v[u][f] = f == op.negate ? -x : x;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (t0 + u * kOpThreads >= count) continue;
#pragma unroll
      for (int f = 0; f < 8; ++f)
        if (f >= op.field_lo && f < op.field_hi) pool[D.off + f * D.fstride + od[u]] = v[u][f];
    }
  }
}

template <typename S>
__global__ void __launch_bounds__(kOpThreads) copy_ops_kernel(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                                             const CopyOp* __restrict__ ops) {
  copy_op_pairs(pool, patches, ops[blockIdx.x]);
}

// Fine halo points from the coarse patch below. Fine haloed index f along an axis
// corresponds to level index g = f - 2 + box_lo; the coarse level index is g / 2.
template <typename S>
__device__ __forceinline__ void axis_weights(int node_axis, int g, int& c0, int& cnt, S (&w)[4]) {
  // returns coarse level indices c0 .. c0+cnt-1 with weights w
  if (node_axis) {
    if ((g & 1) == 0) {
      c0 = g >> 1;
      cnt = 1;
      w[0] = S(1);
    } else {
      c0 = (g >> 1) - 1;  // floor for negative g too (arithmetic shift)
      cnt = 4;
      w[0] = S(-1.0 / 16);
      w[1] = S(9.0 / 16);
      w[2] = S(9.0 / 16);
      w[3] = S(-1.0 / 16);
    }
  } else {
    const int c = g >> 1;
    if ((g & 1) == 0) {
      c0 = c - 1;
      w[0] = S(0.25);
      w[1] = S(0.75);
    } else {
      c0 = c;
      w[0] = S(0.75);
      w[1] = S(0.25);
    }
    cnt = 2;
  }
}

// One fine point of an interpolation op: the weights of every axis, then the loads of
// all fields over all weights (fields innermost; each field's terms in the order a0, a1,
// a2), then the stores.
template <typename S, int NDIM>
__device__ __forceinline__ void interp_point(S* __restrict__ pool, const PatchDesc& F, const PatchDesc& C,
                                             const InterpOp& op, unsigned t, unsigned n1, unsigned n2) {
  const unsigned line = t / n2;
  const int q2 = int(t - line * n2);
  const int q1 = int(line % n1);
  const int q0 = int(line / n1);
  const int fi[3] = {op.d[0] + q0, op.d[1] + q1, op.d[2] + q2};  // fine haloed indices
  int c0[3], cnt[3];
  S w[3][4];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (a >= NDIM) {
      c0[a] = 0;
      cnt[a] = 1;
      w[a][0] = S(1);
      continue;
    }
    const int g = fi[a] - kHalo + op.fine_lo[a];  // fine level index
    axis_weights<S>((op.node_mask >> a) & 1, g, c0[a], cnt[a], w[a]);
    c0[a] = c0[a] - op.coarse_lo[a] + kHalo;  // coarse haloed index
  }
  const int lo = op.field_lo, hi = op.field_hi;
  S acc[8];
#pragma unroll
  for (int f = 0; f < 8; ++f) acc[f] = S(0);
  constexpr int K2 = NDIM == 3 ? 4 : 1;
#pragma unroll
  for (int a0 = 0; a0 < 4; ++a0)
#pragma unroll
    for (int a1 = 0; a1 < 4; ++a1)
#pragma unroll
      for (int a2 = 0; a2 < K2; ++a2) {
        if (a0 < cnt[0] && a1 < cnt[1] && a2 < cnt[2]) {
          const S wt = w[0][a0] * w[1][a1] * w[2][a2];
          const S* cf = pool + C.off + offset_of(C, c0[0] + a0, c0[1] + a1, NDIM == 3 ? c0[2] + a2 : 0);
#pragma unroll
          for (int f = 0; f < 8; ++f)
            if (f >= lo && f < hi) acc[f] += wt * cf[f * C.fstride];
        }
      }
  S* out = pool + F.off + offset_of(F, fi[0], fi[1], NDIM == 3 ? fi[2] : 0);
#pragma unroll
  for (int f = 0; f < 8; ++f)
    if (f >= lo && f < hi) out[f * F.fstride] = acc[f];
}

// The points of one interpolation op, over the threads of the block.
template <typename S>
__device__ __forceinline__ void interp_op(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                          const InterpOp& op) {
  const PatchDesc F = patches[op.fine];
  const PatchDesc C = patches[op.coarse];
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = threadIdx.x; t < count; t += kOpThreads) {
    if (op.ndim == 3)
      interp_point<S, 3>(pool, F, C, op, t, n1, n2);
    else
      interp_point<S, 2>(pool, F, C, op, t, n1, n2);
  }
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
  const RestrictOp op = ops[blockIdx.x];
  const PatchDesc F = patches[op.fine];
  const PatchDesc C = patches[op.coarse];
  int cnt[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) cnt[a] = (a < op.ndim && !((op.node_mask >> a) & 1)) ? 2 : 1;
  const int total = cnt[0] * cnt[1] * cnt[2];
  const S scale = S(1) / S(total);
  const int lo = op.field_lo, hi = op.field_hi;
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = threadIdx.x; t < count; t += kOpThreads) {
    const unsigned line = t / n2;
    const int q2 = int(t - line * n2);
    const int q1 = int(line % n1);
    const int q0 = int(line / n1);
    const int ci[3] = {op.c[0] + q0, op.c[1] + q1, op.c[2] + q2};  // coarse haloed
    const int fi[3] = {op.f[0] + 2 * q0, op.f[1] + 2 * q1, op.f[2] + 2 * q2};  // fine haloed start
    // every fine value of every field first (fields innermost; each field's terms in the
    // order a0, a1, a2), then the stores
    S acc[8];
#pragma unroll
    for (int f = 0; f < 8; ++f) acc[f] = S(0);
#pragma unroll
    for (int a0 = 0; a0 < 2; ++a0)
#pragma unroll
      for (int a1 = 0; a1 < 2; ++a1)
#pragma unroll
        for (int a2 = 0; a2 < 2; ++a2) {
          if (a0 < cnt[0] && a1 < cnt[1] && a2 < cnt[2]) {
            const S* ff = pool + F.off + offset_of(F, fi[0] + a0, fi[1] + a1, op.ndim == 3 ? fi[2] + a2 : 0);
#pragma unroll
            for (int f = 0; f < 8; ++f)
              if (f >= lo && f < hi) acc[f] += ff[f * F.fstride];
          }
        }
    S* out = pool + C.off + offset_of(C, ci[0], ci[1], op.ndim == 3 ? ci[2] : 0);
#pragma unroll
    for (int f = 0; f < 8; ++f)
      if (f >= lo && f < hi) out[f * C.fstride] = total == 1 ? acc[f] : acc[f] * scale;
  }
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
