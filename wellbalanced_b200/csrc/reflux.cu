// Refluxing on the device (Berger–Colella; patchwork's FluxRegister, whose semantics
// tests/unit/test_fluid2d_patches.py:162-240 of the reference pins): after each RK stage
// the fluxes through every coarse-fine interface face are recomputed from the stage's
// input state — the coarse face and the mean of the fine faces over it, with the same
// reconstruction and HLLD as the stage kernels — and their difference is accumulated in
// a float64 register; after the Heun combine the coarse cells outside the fine patches
// take the register's correction (carafe/mhd.py:906-919, 989-990).
#include <type_traits>

#include "halo.cuh"
#include "ops.cuh"
#include "layout.cuh"
#include "numerics.cuh"
#include "wb_internal.cuh"

namespace wb {

__device__ __forceinline__ int64_t cell_offset(const PatchDesc& P, int i, int j, int k) {
  if (P.pitch1) return int64_t(i) * P.pitch0 + int64_t(j) * P.pitch1 + k;
  return int64_t(i) * P.pitch0 + j;
}

// The arithmetic of the primitive variables and face fields: the state's type S, with
// float32-seeded float64 reciprocals where a float64 state is advanced with float32
// arithmetic R (as the stage kernels' cell phase); Math<S> where R = S.
template <typename S, typename R>
using CellMath = typename std::conditional<std::is_same<S, R>::value, Math<S>, MathRefined>::type;

// Primitive variables (rho, u, v, w, p, bx, by, bz) of haloed cell (i, j, k) and the
// field at its lower face along `axis`, with the arithmetic of the stage kernels: formed
// in the state's type S and rounded to the arithmetic type R.
template <typename S, typename R>
__device__ void cell_primitive(const S* src, const PatchDesc& P, int ndim, int i, int j, int k, int axis,
                               const double* b0, double gamma, R (&q)[8], R& bn_lower) {
  using M = CellMath<S, R>;
  const int64_t fs = P.fstride;
  const int64_t o = cell_offset(P, i, j, k);
  const S r = src[o], m0 = src[fs + o], m1 = src[2 * fs + o], m2 = src[3 * fs + o], e = src[4 * fs + o];
  S bx, by, bz, bn;
  if (ndim == 2) {
    const S* A = src + 6 * fs;
    const int64_t p0 = P.pitch0;
    const S dx = S(P.dx[0]), dy = S(P.dx[1]);
    const S idx = M::inv(dx), idy = M::inv(dy);
    const S bxl = M::div(A[o + 1] - A[o], dy, idy) + S(b0[0]);
    const S bxh = M::div(A[o + p0 + 1] - A[o + p0], dy, idy) + S(b0[0]);
    const S byl = -M::div(A[o + p0] - A[o], dx, idx) + S(b0[1]);
    const S byh = -M::div(A[o + p0 + 1] - A[o + 1], dx, idx) + S(b0[1]);
    bx = S(0.5) * (bxl + bxh);
    by = S(0.5) * (byl + byh);
    bz = src[5 * fs + o];
    bn = axis == 0 ? bxl : byl;
  } else {
    const S* Ax = src + 5 * fs;
    const S* Ay = src + 6 * fs;
    const S* Az = src + 7 * fs;
    const int64_t p0 = P.pitch0, p1 = P.pitch1;
    const S dx = S(P.dx[0]), dy = S(P.dx[1]), dz = S(P.dx[2]);
    const S idx = M::inv(dx), idy = M::inv(dy), idz = M::inv(dz);
    auto fx = [&](int64_t c) { return M::div(Az[c + p1] - Az[c], dy, idy) - M::div(Ay[c + 1] - Ay[c], dz, idz) + S(b0[0]); };
    auto fy = [&](int64_t c) { return M::div(Ax[c + 1] - Ax[c], dz, idz) - M::div(Az[c + p0] - Az[c], dx, idx) + S(b0[1]); };
    auto fz = [&](int64_t c) { return M::div(Ay[c + p0] - Ay[c], dx, idx) - M::div(Ax[c + p1] - Ax[c], dy, idy) + S(b0[2]); };
    const S bxl = fx(o), byl = fy(o), bzl = fz(o);
    bx = S(0.5) * (bxl + fx(o + p0));
    by = S(0.5) * (byl + fy(o + p1));
    bz = S(0.5) * (bzl + fz(o + 1));
    bn = axis == 0 ? bxl : (axis == 1 ? byl : bzl);
  }
  const S ir = M::inv(r);
  const S u = M::div(m0, r, ir), v = M::div(m1, r, ir), w = M::div(m2, r, ir);
  q[0] = R(r);
  q[1] = R(u);
  q[2] = R(v);
  q[3] = R(w);
  q[4] = R(recover_pressure<S>(r, m0, m1, m2, e, bx, by, bz, u, v, w, gamma));
  q[5] = R(bx);
  q[6] = R(by);
  q[7] = R(bz);
  bn_lower = R(bn);
}

// The flux through the lower face along `axis` of haloed cell (i, j, k), in the frame of
// that axis; conserved rows returned in physical order (2D: rho, mx, my, mz, E, Bz; 3D:
// rho, mx, my, mz, E), computed in the state's precision like the stage kernels.
// The fields at the lower x- and y-faces of haloed 2D cell offset o (as the stage kernel
// forms them: in the state's type, rounded to the arithmetic type R).
template <typename S, typename R>
__device__ __forceinline__ void lower_face_fields(const S* A, int64_t o, int64_t p0, const PatchDesc& P,
                                                  const double* b0, R& bxl, R& byl) {
  using M = CellMath<S, R>;
  const S dx = S(P.dx[0]), dy = S(P.dx[1]);
  const S idx = M::inv(dx), idy = M::inv(dy);
  bxl = R(M::div(A[o + 1] - A[o], dy, idy) + S(b0[0]));
  byl = R(-M::div(A[o + p0] - A[o], dx, idx) + S(b0[1]));
}

// J_z = dB_y/dx - dB_x/dy at haloed 2D node (i, j), the lower-left corner of cell (i, j),
// from the four faces around it (carafe/kernels/mhd_resistive/mhd_resistive_pyccel.py:21-30).
template <typename S, typename R>
__device__ R node_current(const S* src, const PatchDesc& P, int i, int j, const double* b0) {
  using M = Math<R>;
  const S* A = src + 6 * P.fstride;
  const int64_t p0 = P.pitch0, o = cell_offset(P, i, j, 0);
  const R dx = R(P.dx[0]), dy = R(P.dx[1]);
  const R idx = M::inv(dx), idy = M::inv(dy);
  R bx, by, bx_below, by_left, unused;
  lower_face_fields<S, R>(A, o, p0, P, b0, bx, by);
  lower_face_fields<S, R>(A, o - p0, p0, P, b0, unused, by_left);
  lower_face_fields<S, R>(A, o - 1, p0, P, b0, bx_below, unused);
  return M::div(by - by_left, dx, idx) - M::div(bx - bx_below, dy, idy);
}

// Temperature p / rho of haloed 2D cell (i, j).
template <typename S, typename R>
__device__ R cell_temperature(const S* src, const PatchDesc& P, int i, int j, const double* b0, double gamma) {
  using M = Math<R>;
  R q[8], unused;
  cell_primitive<S, R>(src, P, 2, i, j, 0, 0, b0, gamma, q, unused);
  return M::div(q[4], q[0], M::inv(q[0]));
}

// The field at the lower `axis`-face of haloed 3D cell (i, j, k): the curl of the edge
// potential plus the mean field, with the arithmetic of the 3D stage kernel.
template <typename S, typename R>
__device__ R face_field3(const S* src, const PatchDesc& P, int axis, int i, int j, int k, const double* b0) {
  using M = CellMath<S, R>;
  const int64_t fs = P.fstride, p0 = P.pitch0, p1 = P.pitch1;
  const int64_t o = cell_offset(P, i, j, k);
  const S* Ax = src + 5 * fs;
  const S* Ay = src + 6 * fs;
  const S* Az = src + 7 * fs;
  const S dx = S(P.dx[0]), dy = S(P.dx[1]), dz = S(P.dx[2]);
  const S idx = M::inv(dx), idy = M::inv(dy), idz = M::inv(dz);
  if (axis == 0) return R(M::div(Az[o + p1] - Az[o], dy, idy) - M::div(Ay[o + 1] - Ay[o], dz, idz) + S(b0[0]));
  if (axis == 1) return R(M::div(Ax[o + 1] - Ax[o], dz, idz) - M::div(Az[o + p0] - Az[o], dx, idx) + S(b0[1]));
  return R(M::div(Ay[o + p0] - Ay[o], dx, idx) - M::div(Ax[o + p1] - Ax[o], dy, idy) + S(b0[2]));
}

struct Cell3 {
  int v[3];
};

// J_c = d_a B_b - d_b B_a ((c, a, b) cyclic) on the 3D c-edge whose lower corner is haloed
// cell y (carafe/mhd3d.py:579-590).
template <typename S, typename R>
__device__ R edge_current3(const S* src, const PatchDesc& P, int c, Cell3 y, const double* b0) {
  using M = Math<R>;
  const int a = (c + 1) % 3, b = (c + 2) % 3;
  Cell3 ya = y, yb = y;
  --ya.v[a];
  --yb.v[b];
  const R da = R(P.dx[a]), db = R(P.dx[b]);
  return M::div(face_field3<S, R>(src, P, b, y.v[0], y.v[1], y.v[2], b0) -
                    face_field3<S, R>(src, P, b, ya.v[0], ya.v[1], ya.v[2], b0),
                da, M::inv(da)) -
         M::div(face_field3<S, R>(src, P, a, y.v[0], y.v[1], y.v[2], b0) -
                    face_field3<S, R>(src, P, a, yb.v[0], yb.v[1], yb.v[2], b0),
                db, M::inv(db));
}

// eta (J_b B_c - J_c B_b) on the lower s-face of haloed 3D cell x ((s, b, c) cyclic): J the
// mean of the face's two b- and two c-edges, B the mean of the four faces around it
// (carafe/mhd3d.py:590-600).
template <typename S, typename R>
__device__ R resistive_energy3(const S* src, const PatchDesc& P, int s, Cell3 x, const double* b0, R eta) {
  const int b = (s + 1) % 3, c = (s + 2) % 3;
  auto shifted = [&](int axis1, int d1, int axis2, int d2) {
    Cell3 y = x;
    y.v[axis1] += d1;
    y.v[axis2] += d2;
    return y;
  };
  auto field = [&](int axis, Cell3 y) { return face_field3<S, R>(src, P, axis, y.v[0], y.v[1], y.v[2], b0); };
  const R jb = R(0.5) * (edge_current3<S, R>(src, P, b, x, b0) + edge_current3<S, R>(src, P, b, shifted(c, 1, c, 0), b0));
  const R jc = R(0.5) * (edge_current3<S, R>(src, P, c, x, b0) + edge_current3<S, R>(src, P, c, shifted(b, 1, b, 0), b0));
  const R bc = R(0.5) * (R(0.5) * (field(c, shifted(s, -1, s, 0)) + field(c, x)) +
                         R(0.5) * (field(c, shifted(s, -1, c, 1)) + field(c, shifted(c, 1, c, 0))));
  const R bb = R(0.5) * (R(0.5) * (field(b, shifted(s, -1, s, 0)) + field(b, x)) +
                         R(0.5) * (field(b, shifted(s, -1, b, 1)) + field(b, shifted(b, 1, b, 0))));
  return eta * (jb * bc - jc * bb);
}

// The non-ideal coefficients of the face fluxes: resistivity and the parallel and
// perpendicular conductivities (2D only).
struct FacePhysics {
  double eta, kappa_par, kappa_perp;
};

template <typename S, typename R, int LIM, bool PHYS>
__device__ void face_flux(const S* src, const PatchDesc& P, int ndim, int axis, int i, int j, int k,
                          const double* b0, double gamma, const FacePhysics& phys, double (&out)[6]) {
  int comp[7], rows[6];
  int ncons;
  if (ndim == 2) {
    ncons = 6;
    if (axis == 0) {
      const int c[7] = {0, 1, 2, 3, 4, 6, 7};
      const int r[6] = {0, 1, 2, 3, 4, 6};
      for (int t = 0; t < 7; ++t) comp[t] = c[t];
      for (int t = 0; t < 6; ++t) rows[t] = r[t];
    } else {
      const int c[7] = {0, 2, 1, 3, 4, 5, 7};
      const int r[6] = {0, 2, 1, 3, 4, 6};
      for (int t = 0; t < 7; ++t) comp[t] = c[t];
      for (int t = 0; t < 6; ++t) rows[t] = r[t];
    }
  } else {
    ncons = 5;
    const int s = axis, b = (axis + 1) % 3, c = (axis + 2) % 3;
    comp[0] = 0;
    comp[1] = 1 + s;
    comp[2] = 1 + b;
    comp[3] = 1 + c;
    comp[4] = 4;
    comp[5] = 5 + b;
    comp[6] = 5 + c;
    rows[0] = 0;
    rows[1 + s] = 1;
    rows[1 + b] = 2;
    rows[1 + c] = 3;
    rows[4] = 4;
  }
  R qs[4][7];
  R bn = R(0);
#pragma unroll
  for (int st = 0; st < 4; ++st) {
    int ii = i, jj = j, kk = k;
    if (axis == 0) ii += st - 2;
    if (axis == 1) jj += st - 2;
    if (axis == 2) kk += st - 2;
    R q[8], bl;
    cell_primitive<S, R>(src, P, ndim, ii, jj, kk, axis, b0, gamma, q, bl);
    if (st == 2) bn = bl;  // the face is the lower face of the third cell
    for (int t = 0; t < 7; ++t) qs[st][t] = q[comp[t]];
  }
  R L[7], Rt[7], F[7];
  reconstruct<LIM>(qs[0], qs[1], qs[2], qs[3], L, Rt);
  hlld_flux(L, Rt, bn, R(gamma), R(1.0 / (gamma - 1.0)), F);
  if (PHYS && ndim == 2) {
    // the resistive and conductive terms, with the stage kernel's arithmetic: cells a | b
    // are qs[1] | qs[2] (haloed cells (i-1, j) | (i, j) on an x-face, (i, j-1) | (i, j) on a y-face)
    using M = Math<R>;
    const bool xface = axis == 0;
    const R dx = R(P.dx[0]), dy = R(P.dx[1]);
    const R idx = M::inv(dx), idy = M::inv(dy);
    const R ht = xface ? dy : dx, iht = xface ? idy : idx;
    R slope[2] = {R(0), R(0)};
    if (phys.kappa_par != 0.0 || phys.kappa_perp != 0.0) {
      for (int side = 0; side < 2; ++side) {
        const int ci = xface ? i - 1 + side : i, cj = xface ? j : j - 1 + side;
        const int ti = xface ? 0 : 1, tj = xface ? 1 : 0;  // step to the transverse neighbours
        const R t0 = cell_temperature<S, R>(src, P, ci - ti, cj - tj, b0, gamma);
        const R t2 = cell_temperature<S, R>(src, P, ci + ti, cj + tj, b0, gamma);
        const R t1 = M::div(qs[1 + side][4], qs[1 + side][0], M::inv(qs[1 + side][0]));
        slope[side] = limited_slope<2>(M::div(t2 - t1, ht, iht), M::div(t1 - t0, ht, iht));
      }
    }
    R jz_0 = R(0), jz_1 = R(0);
    if (phys.eta != 0.0) {
      jz_0 = node_current<S, R>(src, P, i, j, b0);
      jz_1 = xface ? node_current<S, R>(src, P, i, j + 1, b0) : node_current<S, R>(src, P, i + 1, j, b0);
    }
    const R t_a = M::div(qs[1][4], qs[1][0], M::inv(qs[1][0]));
    const R t_b = M::div(qs[2][4], qs[2][0], M::inv(qs[2][0]));
    nonideal_face_terms(xface, bn, t_a, t_b, slope[0], slope[1], qs[1][5], qs[2][5], qs[1][6], qs[2][6], jz_0, jz_1,
                        xface ? dx : dy, xface ? idx : idy, R(phys.eta), R(phys.kappa_par), R(phys.kappa_perp), F);
  }
  if (PHYS && ndim == 3 && phys.eta != 0.0) {
    F[4] += resistive_energy3<S, R>(src, P, axis, Cell3{{i, j, k}}, b0, R(phys.eta));
  }
  for (int t = 0; t < ncons; ++t) out[t] = double(F[rows[t]]);
}

// One warp per interface side: reg[slot] += mean of the fine faces over each coarse face -
// the coarse face (each op holds both sides, so no two warps share a slot). The coarse face
// and its 2 (2D) or 4 (3D) fine faces are evaluated by separate lanes (32 / K coarse faces
// per round), then one lane per coarse face combines them from shared memory, the fine
// faces summed in the order (a, b). Most interfaces are a few coarse faces long, so a warp
// (four ops per 128-thread block) keeps the lanes busy where a block per op would not.
constexpr int kFluxThreads = 128;
constexpr int kFluxWarps = kFluxThreads / 32;

template <typename S, typename R, int LIM, bool PHYS>
__global__ void __launch_bounds__(kFluxThreads) face_flux_ops_kernel(const S* __restrict__ pool,
                                                                     const PatchDesc* __restrict__ patches,
                                                                     const FaceFluxOp* __restrict__ ops, int nops,
                                                                     double b0x, double b0y, double b0z, double gamma,
                                                                     FacePhysics phys, double* __restrict__ reg) {
  __shared__ double g_all[kFluxWarps][32][6];
  const int warp = threadIdx.x / 32, t = threadIdx.x % 32;
  const int index = blockIdx.x * kFluxWarps + warp;
  if (index >= nops) return;  // a whole warp: no block-wide barrier follows
  double(*g)[6] = g_all[warp];
  const FaceFluxOp op = ops[index];
  const PatchDesc C = patches[op.coarse];
  const PatchDesc F = patches[op.fine];
  const double b0[3] = {b0x, b0y, b0z};
  const int ncons = op.ndim == 2 ? 6 : 5;
  const int fine_b = op.ndim == 3 ? 2 : 1;
  const int K = 1 + 2 * fine_b;  // evaluations per coarse face
  const int per = 32 / K;        // coarse faces per round
  const int e = t % K;
  for (int s0 = 0; s0 < op.len; s0 += per) {
    const int s = s0 + t / K;
    if (t < per * K && s < op.len) {
      const int s1 = s / op.width, s2 = s % op.width;
      int idx[3] = {0, 0, 0};
      double out[6] = {0, 0, 0, 0, 0, 0};
      if (e == 0) {
        idx[op.axis] = op.coarse_plane;
        idx[op.t1] = op.coarse_t0[0] + s1;
        if (op.ndim == 3) idx[op.t2] = op.coarse_t0[1] + s2;
        face_flux<S, R, LIM, PHYS>(pool + C.off, C, op.ndim, op.axis, idx[0], idx[1], idx[2], b0, gamma, phys, out);
      } else {
        const int a = (e - 1) / fine_b, b = (e - 1) % fine_b;
        idx[op.axis] = op.fine_plane;
        idx[op.t1] = op.fine_t0[0] + 2 * s1 + a;
        if (op.ndim == 3) idx[op.t2] = op.fine_t0[1] + 2 * s2 + b;
        face_flux<S, R, LIM, PHYS>(pool + F.off, F, op.ndim, op.axis, idx[0], idx[1], idx[2], b0, gamma, phys, out);
      }
#pragma unroll
      for (int q = 0; q < 6; ++q) g[t][q] = out[q];
    }
    __syncwarp();
    if (t < per && s0 + t < op.len) {
      const int s = s0 + t;
      double fine[6] = {0, 0, 0, 0, 0, 0};
      for (int k = 1; k < K; ++k)
        for (int q = 0; q < ncons; ++q) fine[q] += g[t * K + k][q];
      const double count = double(K - 1);
      for (int q = 0; q < ncons; ++q) reg[op.reg_off + int64_t(q) * op.len + s] += fine[q] / count - g[t * K][q];
    }
    __syncwarp();
  }
}

// One block of 128 threads per op (ops.cuh reflux_op), no atomics: the ops of one launch
// must touch disjoint cells.
template <typename S>
__global__ void reflux_apply_kernel(S* __restrict__ pool, const PatchDesc* __restrict__ patches,
                                    const RefluxOp* __restrict__ ops, double* __restrict__ reg,
                                    const double* __restrict__ dt) {
  reflux_op<S, 128>(pool, patches, ops[blockIdx.x], reg, dt);
}

// 2D ideal MHD with the fine faces' fluxes as the fine patches' stage kernel formed them
// (its boundary-face output `bflux`: float64 rows (side, conserved row, face along the side)
// at each patch's PatchDesc.bflux, x-faces then y-faces): one thread per coarse face of all
// ops (op.first: the op's first face in that flat numbering), which recomputes the coarse
// face and sums the two fine faces in the order of face_flux_ops_kernel, so the register
// gets the same values as there.
constexpr int kStagedThreads = 128;

template <typename S, typename R, int LIM>
__global__ void __launch_bounds__(kStagedThreads) face_flux_staged_kernel(
    const S* __restrict__ pool, const PatchDesc* __restrict__ patches, const FaceFluxOp* __restrict__ ops, int nops,
    int nfaces, double b0x, double b0y, double b0z, double gamma, const double* __restrict__ bflux,
    double* __restrict__ reg) {
  const int face = blockIdx.x * kStagedThreads + threadIdx.x;
  if (face >= nfaces) return;
  // the op holding this face: the last one whose first face is not after it
  int lo = 0, hi = nops - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ops[mid].first <= face) lo = mid; else hi = mid - 1;
  }
  const FaceFluxOp op = ops[lo];
  const int s = face - op.first;
  if (s < 0 || s >= op.len || op.ndim != 2) return;
  const PatchDesc C = patches[op.coarse];
  const PatchDesc F = patches[op.fine];
  const double b0[3] = {b0x, b0y, b0z};
  int idx[3] = {0, 0, 0};
  idx[op.axis] = op.coarse_plane;
  idx[op.t1] = op.coarse_t0[0] + s;
  double coarse[6] = {0, 0, 0, 0, 0, 0};
  face_flux<S, R, LIM, false>(pool + C.off, C, 2, op.axis, idx[0], idx[1], idx[2], b0, gamma,
                              FacePhysics{0.0, 0.0, 0.0}, coarse);
  const int along = op.axis == 0 ? F.n[1] : F.n[0];
  const int side = op.fine_plane == kHalo ? 0 : 1;
  const double* rows = bflux + F.bflux + (op.axis == 0 ? 0 : 2 * 6 * F.n[1]);
  const int f0 = op.fine_t0[0] + 2 * s - kHalo;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const double* row = rows + (side * 6 + q) * along;
    double fine = 0.0;
    fine += row[f0];
    fine += row[f0 + 1];
    reg[op.reg_off + int64_t(q) * op.len + s] += fine / 2.0 - coarse[q];
  }
}

template <typename S, typename R>
void launch_face_flux_staged(const S* pool, const PatchDesc* patches, const FaceFluxOp* ops, int nops, int nfaces,
                             const double* b0, double gamma, int limiter, const double* bflux, double* reg,
                             cudaStream_t stream) {
  if (nfaces <= 0) return;
  const int grid = (nfaces + kStagedThreads - 1) / kStagedThreads;
  switch (limiter) {
    case 0: face_flux_staged_kernel<S, R, 0><<<grid, kStagedThreads, 0, stream>>>(pool, patches, ops, nops, nfaces, b0[0], b0[1], b0[2], gamma, bflux, reg); break;
    case 1: face_flux_staged_kernel<S, R, 1><<<grid, kStagedThreads, 0, stream>>>(pool, patches, ops, nops, nfaces, b0[0], b0[1], b0[2], gamma, bflux, reg); break;
    case 2: face_flux_staged_kernel<S, R, 2><<<grid, kStagedThreads, 0, stream>>>(pool, patches, ops, nops, nfaces, b0[0], b0[1], b0[2], gamma, bflux, reg); break;
    default: face_flux_staged_kernel<S, R, 3><<<grid, kStagedThreads, 0, stream>>>(pool, patches, ops, nops, nfaces, b0[0], b0[1], b0[2], gamma, bflux, reg); break;
  }
}

template <typename S, typename R, bool PHYS>
void launch_face_flux_kernel(const S* pool, const PatchDesc* patches, const FaceFluxOp* ops, int nops,
                             const double* b0, double gamma, int limiter, const FacePhysics& phys, double* reg,
                             cudaStream_t stream) {
  switch (limiter) {
    case 0: face_flux_ops_kernel<S, R, 0, PHYS><<<(nops + kFluxWarps - 1) / kFluxWarps, kFluxThreads, 0, stream>>>(pool, patches, ops, nops, b0[0], b0[1], b0[2], gamma, phys, reg); break;
    case 1: face_flux_ops_kernel<S, R, 1, PHYS><<<(nops + kFluxWarps - 1) / kFluxWarps, kFluxThreads, 0, stream>>>(pool, patches, ops, nops, b0[0], b0[1], b0[2], gamma, phys, reg); break;
    case 2: face_flux_ops_kernel<S, R, 2, PHYS><<<(nops + kFluxWarps - 1) / kFluxWarps, kFluxThreads, 0, stream>>>(pool, patches, ops, nops, b0[0], b0[1], b0[2], gamma, phys, reg); break;
    default: face_flux_ops_kernel<S, R, 3, PHYS><<<(nops + kFluxWarps - 1) / kFluxWarps, kFluxThreads, 0, stream>>>(pool, patches, ops, nops, b0[0], b0[1], b0[2], gamma, phys, reg); break;
  }
}

// physics: null for ideal MHD, else {eta, kappa_par, kappa_perp} (3D interfaces take eta only).
// R: the arithmetic of the recomputed faces (the stage kernels' R for the state's type S).
// bflux: the stage kernel's boundary-face fluxes of the patches (2D ideal MHD: the fine
// faces are read there instead of recomputed, one thread per coarse face of the `nfaces`
// the ops hold), or null.
template <typename S, typename R>
int launch_face_flux_ops(const S* pool, const PatchDesc* patches, const FaceFluxOp* ops, int nops, int nfaces,
                         const double* b0, double gamma, int limiter, const double* physics, const double* bflux,
                         double* reg, cudaStream_t stream) {
  if (nops <= 0) return kOk;
  if (bflux)
    launch_face_flux_staged<S, R>(pool, patches, ops, nops, nfaces, b0, gamma, limiter, bflux, reg, stream);
  else if (physics && (physics[0] != 0.0 || physics[1] != 0.0 || physics[2] != 0.0))
    launch_face_flux_kernel<S, R, true>(pool, patches, ops, nops, b0, gamma, limiter,
                                        FacePhysics{physics[0], physics[1], physics[2]}, reg, stream);
  else
    launch_face_flux_kernel<S, R, false>(pool, patches, ops, nops, b0, gamma, limiter, FacePhysics{0.0, 0.0, 0.0},
                                         reg, stream);
  return check_launch("face flux ops");
}

template <typename S>
int launch_reflux_apply(S* pool, const PatchDesc* patches, const RefluxOp* ops, int nops, double* reg,
                        const double* dt, cudaStream_t stream) {
  if (nops > 0) reflux_apply_kernel<S><<<nops, 128, 0, stream>>>(pool, patches, ops, reg, dt);
  return check_launch("reflux");
}

template int launch_face_flux_ops<float, float>(const float*, const PatchDesc*, const FaceFluxOp*, int, int,
                                                const double*, double, int, const double*, const double*, double*,
                                                cudaStream_t);
template int launch_face_flux_ops<double, double>(const double*, const PatchDesc*, const FaceFluxOp*, int, int,
                                                  const double*, double, int, const double*, const double*, double*,
                                                  cudaStream_t);
template int launch_face_flux_ops<double, float>(const double*, const PatchDesc*, const FaceFluxOp*, int, int,
                                                 const double*, double, int, const double*, const double*, double*,
                                                 cudaStream_t);
template int launch_reflux_apply<float>(float*, const PatchDesc*, const RefluxOp*, int, double*, const double*,
                                        cudaStream_t);
template int launch_reflux_apply<double>(double*, const PatchDesc*, const RefluxOp*, int, double*, const double*,
                                         cudaStream_t);

}  // namespace wb
