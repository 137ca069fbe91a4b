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
#include "layout.cuh"
#include "halo.cuh"
#include "wb_internal.cuh"

namespace wb {

// element offset of haloed index (i, j, k) of a patch (k ignored in 2D)
__device__ __forceinline__ int64_t offset_of(const PatchDesc& P, int i, int j, int k) {
  if (P.pitch1) return int64_t(i) * P.pitch0 + int64_t(j) * P.pitch1 + k;
  return int64_t(i) * P.pitch0 + j;
}

template <typename S>
__global__ void __launch_bounds__(256) copy_ops_kernel(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                                      const CopyOp* __restrict__ ops) {
  const CopyOp op = ops[blockIdx.x];
  const PatchDesc D = patches[op.dst];
  const PatchDesc A = patches[op.src1];
  const PatchDesc B = patches[op.src2 >= 0 ? op.src2 : op.src1];
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = threadIdx.x; t < count; t += blockDim.x) {
    const unsigned line = t / n2;
    const int p2 = int(t - line * n2);
    const int p1 = int(line % n1);
    const int p0 = int(line / n1);
    const int64_t od = offset_of(D, op.d[0] + p0, op.d[1] + p1, op.d[2] + p2);
    const int64_t o1 = offset_of(A, op.s1[0] + op.m1[0] * p0, op.s1[1] + op.m1[1] * p1, op.s1[2] + op.m1[2] * p2);
    const int64_t o2 = offset_of(B, op.s2[0] + op.m2[0] * p0, op.s2[1] + op.m2[1] * p1, op.s2[2] + op.m2[2] * p2);
    // every field's value first, then the stores: the loads of a point are in flight
    // together (an op never writes a point it reads)
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

template <typename S>
__global__ void __launch_bounds__(256) interp_ops_kernel(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                                        const InterpOp* __restrict__ ops) {
  const InterpOp op = ops[blockIdx.x];
  const PatchDesc F = patches[op.fine];
  const PatchDesc C = patches[op.coarse];
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = threadIdx.x; t < count; t += blockDim.x) {
    const unsigned line = t / n2;
    const int q2 = int(t - line * n2);
    const int q1 = int(line % n1);
    const int q0 = int(line / n1);
    const int fi[3] = {op.d[0] + q0, op.d[1] + q1, op.d[2] + q2};  // fine haloed indices
    int c0[3], cnt[3];
    S w[3][4];
    for (int a = 0; a < 3; ++a) {
      if (a >= op.ndim) {
        c0[a] = 0;
        cnt[a] = 1;
        w[a][0] = S(1);
        continue;
      }
      const int g = fi[a] - kHalo + op.fine_lo[a];  // fine level index
      axis_weights<S>((op.node_mask >> a) & 1, g, c0[a], cnt[a], w[a]);
      c0[a] = c0[a] - op.coarse_lo[a] + kHalo;  // coarse haloed index
    }
    const int64_t od = offset_of(F, fi[0], fi[1], op.ndim == 3 ? fi[2] : 0);
    for (int f = op.field_lo; f < op.field_hi; ++f) {
      const S* cf = pool + C.off + f * C.fstride;
      S acc = S(0);
      for (int a0 = 0; a0 < cnt[0]; ++a0)
        for (int a1 = 0; a1 < cnt[1]; ++a1)
          for (int a2 = 0; a2 < cnt[2]; ++a2)
            acc += w[0][a0] * w[1][a1] * w[2][a2] *
                   cf[offset_of(C, c0[0] + a0, c0[1] + a1, op.ndim == 3 ? c0[2] + a2 : 0)];
      pool[F.off + f * F.fstride + od] = acc;
    }
  }
}

template <typename S>
__global__ void __launch_bounds__(256) restrict_ops_kernel(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                                          const RestrictOp* __restrict__ ops) {
  const RestrictOp op = ops[blockIdx.x];
  const PatchDesc F = patches[op.fine];
  const PatchDesc C = patches[op.coarse];
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = threadIdx.x; t < count; t += blockDim.x) {
    const unsigned line = t / n2;
    const int q2 = int(t - line * n2);
    const int q1 = int(line % n1);
    const int q0 = int(line / n1);
    const int ci[3] = {op.c[0] + q0, op.c[1] + q1, op.c[2] + q2};  // coarse haloed
    const int fi[3] = {op.f[0] + 2 * q0, op.f[1] + 2 * q1, op.f[2] + 2 * q2};  // fine haloed start
    int cnt[3];
    for (int a = 0; a < 3; ++a) cnt[a] = (a < op.ndim && !((op.node_mask >> a) & 1)) ? 2 : 1;
    const S scale = S(1) / S(cnt[0] * cnt[1] * cnt[2]);
    const int64_t oc = offset_of(C, ci[0], ci[1], op.ndim == 3 ? ci[2] : 0);
    for (int f = op.field_lo; f < op.field_hi; ++f) {
      const S* ff = pool + F.off + f * F.fstride;
      S acc = S(0);
      for (int a0 = 0; a0 < cnt[0]; ++a0)
        for (int a1 = 0; a1 < cnt[1]; ++a1)
          for (int a2 = 0; a2 < cnt[2]; ++a2)
            acc += ff[offset_of(F, fi[0] + a0, fi[1] + a1, op.ndim == 3 ? fi[2] + a2 : 0)];
      pool[C.off + f * C.fstride + oc] = cnt[0] * cnt[1] * cnt[2] == 1 ? acc : acc * scale;
    }
  }
}

template <typename S>
int launch_copy_ops(S* pool, const PatchDesc* patches, const CopyOp* ops, int nops, cudaStream_t stream) {
  if (nops > 0) copy_ops_kernel<S><<<nops, 256, 0, stream>>>(pool, patches, ops);
  return check_launch("halo copy");
}
template <typename S>
int launch_interp_ops(S* pool, const PatchDesc* patches, const InterpOp* ops, int nops, cudaStream_t stream) {
  if (nops > 0) interp_ops_kernel<S><<<nops, 256, 0, stream>>>(pool, patches, ops);
  return check_launch("halo interpolation");
}
template <typename S>
int launch_restrict_ops(S* pool, const PatchDesc* patches, const RestrictOp* ops, int nops, cudaStream_t stream) {
  if (nops > 0) restrict_ops_kernel<S><<<nops, 256, 0, stream>>>(pool, patches, ops);
  return check_launch("restrict");
}
template int launch_copy_ops<float>(float*, const PatchDesc*, const CopyOp*, int, cudaStream_t);
template int launch_copy_ops<double>(double*, const PatchDesc*, const CopyOp*, int, cudaStream_t);
template int launch_interp_ops<float>(float*, const PatchDesc*, const InterpOp*, int, cudaStream_t);
template int launch_interp_ops<double>(double*, const PatchDesc*, const InterpOp*, int, cudaStream_t);
template int launch_restrict_ops<float>(float*, const PatchDesc*, const RestrictOp*, int, cudaStream_t);
template int launch_restrict_ops<double>(double*, const PatchDesc*, const RestrictOp*, int, cudaStream_t);

}  // namespace wb
