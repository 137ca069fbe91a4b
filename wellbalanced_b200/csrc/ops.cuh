// Device bodies of the halo, restriction and reflux ops: one op over the NT threads of a
// block. The standalone op kernels launch one op per block; the op program
// (program.cu) runs them inside one launch.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "halo.cuh"
#include "layout.cuh"

namespace wb {

// A thread's place among the NT threads that run one op (a whole block, or one warp of it).
template <int NT>
__device__ __forceinline__ unsigned op_lane() {
  return threadIdx.x % unsigned(NT);
}

// element offset of haloed index (i, j, k) of a patch (k ignored in 2D)
__device__ __forceinline__ int64_t offset_of(const PatchDesc& P, int i, int j, int k) {
  if (P.pitch1) return int64_t(i) * P.pitch0 + int64_t(j) * P.pitch1 + k;
  return int64_t(i) * P.pitch0 + j;
}

constexpr int kOpThreads = 64;  // threads of the block that runs one op

// The points of one copy op, over the NT threads of the block.
template <typename S, int NT = kOpThreads>
__device__ __forceinline__ void copy_op(S* __restrict__ pool, const PatchDesc* __restrict__ patches, const CopyOp& op) {
  const PatchDesc D = patches[op.dst];
  const PatchDesc A = patches[op.src1];
  const PatchDesc B = patches[op.src2 >= 0 ? op.src2 : op.src1];
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = op_lane<NT>(); t < count; t += NT) {
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
template <typename S, int NT = kOpThreads>
__device__ __forceinline__ void copy_op_pairs(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                              const CopyOp& op) {
  const PatchDesc D = patches[op.dst];
  const PatchDesc A = patches[op.src1];
  const PatchDesc B = patches[op.src2 >= 0 ? op.src2 : op.src1];
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t0 = op_lane<NT>(); t0 < count; t0 += 2 * NT) {
    S v[2][8];
    int64_t od[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const unsigned t = t0 + u * NT;
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
      if (t0 + u * NT >= count) continue;
#pragma unroll
      for (int f = 0; f < 8; ++f)
        if (f >= op.field_lo && f < op.field_hi) pool[D.off + f * D.fstride + od[u]] = v[u][f];
    }
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

// The points of one interpolation op, over the NT threads of the block.
template <typename S, int NT = kOpThreads>
__device__ __forceinline__ void interp_op(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                          const InterpOp& op) {
  const PatchDesc F = patches[op.fine];
  const PatchDesc C = patches[op.coarse];
  // 32-bit point index (the host keeps every op below 2^31 points)
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = op_lane<NT>(); t < count; t += NT) {
    if (op.ndim == 3)
      interp_point<S, 3>(pool, F, C, op, t, n1, n2);
    else
      interp_point<S, 2>(pool, F, C, op, t, n1, n2);
  }
}

// The coarse points of one restriction op, over the NT threads of the block: the mean of
// the fine values along cell-centred axes, the coincident fine value along node axes.
template <typename S, int NT = kOpThreads>
__device__ __forceinline__ void restrict_op(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                            const RestrictOp& op) {
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
  for (unsigned t = op_lane<NT>(); t < count; t += NT) {
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

// Apply the register of one interface to the coarse cells beside it, then clear it:
// U -= sign * (0.5 dt) * reg / dx (sign +1 where the interface is the cell's upper face).
// The ops run together must touch disjoint cells (no atomics).
template <typename S, int NT>
__device__ __forceinline__ void reflux_op(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                          const RefluxOp& op, double* __restrict__ reg,
                                          const double* __restrict__ dt) {
  const PatchDesc C = patches[op.coarse];
  const double scale = 0.5 * dt[C.instance];
  const int64_t count = int64_t(op.len) * op.ncomp;
  for (int64_t t = op_lane<NT>(); t < count; t += NT) {
    const int q = int(t / op.len), s = int(t % op.len);
    const int s1 = s / op.width, s2 = s % op.width;
    int idx[3] = {op.c[0], op.c[1], op.c[2]};
    idx[op.t1] += s1;
    if (op.t2 >= 0) idx[op.t2] += s2;
    const int64_t o = offset_of(C, idx[0], idx[1], idx[2]);
    double& r = reg[op.reg_off + int64_t(q) * op.len + s];
    S* u = pool + C.off + int64_t(op.field[q]) * C.fstride + o;
    *u = S(double(*u) - op.sign * scale * r / op.dx);
    r = 0.0;
  }
}

}  // namespace wb
