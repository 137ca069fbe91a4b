// The state transfer of a regrid on the device (patchwork's AMRHierarchy.regrid, as
// carafe/mhd.py:1043-1056 and carafe/mhd3d.py:803-816 call it: "the conserved fields keep
// their integrals, A is interpolated ... so the field stays divergence-free"). Level by
// level, coarse first, on the new hierarchy's pool:
//   * prolongation ops fill each new fine patch from the new coarser level: cells by
//     minmod-limited linear reconstruction (children c -/+ s/4 per axis, so the children's
//     mean is the coarse value: integrals kept, no new extrema), potentials linearly along
//     their node axes and constant along an edge's own axis (so the restriction that
//     follows gives back the coarse potential, hence the coarse field);
//   * kept-value ops copy, from the old hierarchy's pool, every point an old patch of the
//     same level held (periodic images included, so the duplicate node planes of a
//     periodic axis agree);
//   * positivity ops revisit every prolonged parent: where a child of the minmod
//     prolongation has a non-positive density or a pressure below a quarter of the parent's (conserved cells and a field
//     from the interpolated potential do not bound the pressure: the children's kinetic
//     and magnetic energies exceed the coarse ones at a strong front in low-beta gas, where
//     the reference's next step raises), the parent's children take its density,
//     momentum (and B_z) and an energy that keeps its pressure positive (below);
//   * the level's halos are filled (the engine's fill ops) before the next level reads
//     them.
// The same arithmetic as the host transfer (wellbalanced_b200/regrid.py), point by point.
#include "halo.cuh"
#include "layout.cuh"
#include "wb_internal.cuh"

namespace wb {

// One prolongation op: the fine points d .. d + n (haloed fine indices) of fields
// [field_lo, field_hi) from the coarse patch below.
struct ProlongOp {
  int32_t fine, coarse;
  int32_t field_lo, field_hi;
  int32_t node_mask;     // bit a: axis a is node-centred for these fields
  int32_t ndim;
  int32_t n[3];
  int32_t d[3];
  int32_t fine_lo[3];    // level index of the fine patch's first interior cell
  int32_t coarse_lo[3];  // level index of the coarse patch's first interior cell
  int32_t coarse_n[3];   // cells of the coarse level per axis
  int32_t periodic;      // bit a: axis a is periodic
};

constexpr int kTransferThreads = 128;

__device__ __forceinline__ int64_t point_offset(const PatchDesc& P, int i, int j, int k) {
  if (P.pitch1) return int64_t(i) * P.pitch0 + int64_t(j) * P.pitch1 + k;
  return int64_t(i) * P.pitch0 + j;
}

template <typename S>
__device__ __forceinline__ double minmod(double a, double b) {
  return a * b > 0.0 ? (fabs(a) < fabs(b) ? a : b) : 0.0;
}

template <typename S>
__global__ void __launch_bounds__(kTransferThreads) prolong_ops_kernel(S* __restrict__ pool,
                                                                      const PatchDesc* __restrict__ patches,
                                                                      const ProlongOp* __restrict__ ops) {
  const ProlongOp op = ops[blockIdx.x];
  const PatchDesc F = patches[op.fine];
  const PatchDesc C = patches[op.coarse];
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = threadIdx.x; t < count; t += kTransferThreads) {
    const unsigned line = t / n2;
    const int q[3] = {int(line / n1), int(line % n1), int(t - line * n2)};
    int fi[3], g[3];
    for (int a = 0; a < 3; ++a) {
      fi[a] = op.d[a] + q[a];
      g[a] = a < op.ndim ? fi[a] - kHalo + op.fine_lo[a] : 0;  // fine level index
    }
    // coarse haloed index of coarse level index c along axis a
    auto ch = [&](int a, int c) { return a < op.ndim ? c - op.coarse_lo[a] + kHalo : 0; };
    auto coarse_at = [&](int f, const int (&c)[3]) {
      return double(pool[C.off + f * C.fstride + point_offset(C, ch(0, c[0]), ch(1, c[1]), op.ndim == 3 ? ch(2, c[2]) : 0)]);
    };
    S* out = pool + F.off + point_offset(F, fi[0], fi[1], op.ndim == 3 ? fi[2] : 0);
    for (int f = op.field_lo; f < op.field_hi; ++f) {
      double value;
      if (op.node_mask == 0) {
        // cells: centre plus the minmod-limited slope of each axis times -1/4 or +1/4
        int c[3] = {g[0] >> 1, g[1] >> 1, op.ndim == 3 ? g[2] >> 1 : 0};
        const double centre = coarse_at(f, c);
        value = centre;
        for (int a = 0; a < op.ndim; ++a) {
          int lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[0], c[1], c[2]};
          const bool wraps = (op.periodic >> a) & 1;
          lo[a] = (!wraps && c[a] == 0) ? c[a] : c[a] - 1;  // the edge cell repeats outside a closed axis
          hi[a] = (!wraps && c[a] == op.coarse_n[a] - 1) ? c[a] : c[a] + 1;
          const double s = minmod<S>(centre - coarse_at(f, lo), coarse_at(f, hi) - centre);
          value = value + s * ((g[a] & 1) ? 0.25 : -0.25);
        }
      } else {
        // potentials: axis by axis (0 innermost), linear along node axes (coincident nodes
        // exact, midpoints the mean), constant along cell axes
        int base[3], two[3];
        for (int a = 0; a < 3; ++a) {
          const bool node = a < op.ndim && ((op.node_mask >> a) & 1);
          base[a] = a < op.ndim ? (node ? (g[a] >> 1) : (g[a] >> 1)) : 0;
          two[a] = node && (g[a] & 1);
        }
        double acc2[2];
        for (int k = 0; k <= two[2]; ++k) {
          double acc1[2];
          for (int j = 0; j <= two[1]; ++j) {
            double acc0[2];
            for (int i = 0; i <= two[0]; ++i) {
              const int c[3] = {base[0] + i, base[1] + j, base[2] + k};
              acc0[i] = coarse_at(f, c);
            }
            acc1[j] = two[0] ? 0.5 * (acc0[0] + acc0[1]) : acc0[0];
          }
          acc2[k] = two[1] ? 0.5 * (acc1[0] + acc1[1]) : acc1[0];
        }
        value = two[2] ? 0.5 * (acc2[0] + acc2[1]) : acc2[0];
      }
      out[f * F.fstride] = S(value);
    }
  }
}

// One positivity op: the parents n[0] x n[1] x n[2] (coarse haloed cells c0 ..) of the
// fine patch's children (haloed fine cells f0 .., two per axis).
struct PositivityOp {
  int32_t fine, coarse, ndim, pad;
  int32_t n[3];
  int32_t f0[3];
  int32_t c0[3];
};

// Arithmetic rounded operation by operation (no contraction into FMA), in the order of
// the host restatement, so that both pick the same parents and write the same bits.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// The cell-centred field of haloed cell x of patch P: the mean of its two faces per axis,
// each the curl of the potential plus the mean field (3D: edge potentials A_x, A_y, A_z
// in fields 5-7; 2D: the node potential A_z in field 6, B_z the cell field 5).
template <typename S>
__device__ void cell_field(const S* pool, const PatchDesc& P, int ndim, const int (&x)[3], const double (&b0)[3],
                           double (&b)[3]) {
  const S* base = pool + P.off;
  const int64_t fs = P.fstride;
  const double dx = P.dx[0], dy = P.dx[1];
  if (ndim == 2) {
    const int64_t o = point_offset(P, x[0], x[1], 0), p0 = P.pitch0;
    const S* A = base + 6 * fs;
    auto v = [&](int64_t q) { return double(A[q]); };
    const double bxl = dadd(ddiv(dsub(v(o + 1), v(o)), dy), b0[0]);
    const double bxh = dadd(ddiv(dsub(v(o + p0 + 1), v(o + p0)), dy), b0[0]);
    const double byl = dadd(-ddiv(dsub(v(o + p0), v(o)), dx), b0[1]);
    const double byh = dadd(-ddiv(dsub(v(o + p0 + 1), v(o + 1)), dx), b0[1]);
    b[0] = dmul(0.5, dadd(bxl, bxh));
    b[1] = dmul(0.5, dadd(byl, byh));
    b[2] = double(base[5 * fs + o]);
    return;
  }
  const double dz = P.dx[2];
  const int64_t p0 = P.pitch0, p1 = P.pitch1;
  const S* Ax = base + 5 * fs;
  const S* Ay = base + 6 * fs;
  const S* Az = base + 7 * fs;
  auto v = [](const S* A, int64_t q) { return double(A[q]); };
  auto fx = [&](int64_t c) {
    return dadd(dsub(ddiv(dsub(v(Az, c + p1), v(Az, c)), dy), ddiv(dsub(v(Ay, c + 1), v(Ay, c)), dz)), b0[0]);
  };
  auto fy = [&](int64_t c) {
    return dadd(dsub(ddiv(dsub(v(Ax, c + 1), v(Ax, c)), dz), ddiv(dsub(v(Az, c + p0), v(Az, c)), dx)), b0[1]);
  };
  auto fz = [&](int64_t c) {
    return dadd(dsub(ddiv(dsub(v(Ay, c + p0), v(Ay, c)), dx), ddiv(dsub(v(Ax, c + p1), v(Ax, c)), dy)), b0[2]);
  };
  const int64_t o = point_offset(P, x[0], x[1], x[2]);
  b[0] = dmul(0.5, dadd(fx(o), fx(o + p0)));
  b[1] = dmul(0.5, dadd(fy(o), fy(o + p1)));
  b[2] = dmul(0.5, dadd(fz(o), fz(o + 1)));
}

__device__ __forceinline__ double kinetic(double r, double m0, double m1, double m2) {
  return ddiv(dmul(0.5, dadd(dadd(dmul(m0, m0), dmul(m1, m1)), dmul(m2, m2))), r);
}

__device__ __forceinline__ double magnetic(const double (&b)[3]) {
  return dmul(0.5, dadd(dadd(dmul(b[0], b[0]), dmul(b[1], b[1])), dmul(b[2], b[2])));
}

// A child whose pressure falls below this fraction of its parent's counts as collapsed: at
// a front the prolonged children's pressures fall steeply before they turn negative, and a
// child left at a few percent of its neighbours' pressure turns negative in the next step.
constexpr double kPressureFraction = 0.25;

// One thread per parent. Children in the order of their offsets (last axis fastest).
// Where every child has a positive density and a pressure above kPressureFraction times
// the parent's (p = (gamma - 1)(E - K - M), M from the coarse potential) nothing changes. Else,
// with the parent's density rho, momentum m, energy E, kinetic energy K, magnetic energy
// M (its cell-centred field from the coarse potential) and pressure p, each child takes
// rho and m (and, in 2D, the parent's B_z) and, with M_i its own magnetic energy (its field
// from the fine potential) and M' the children's mean of M_i:
//   E_i = E + (M_i - M')                 where (gamma - 1)(E - K - M') > kPressureFraction p
//                                        (the energy's integral kept; every child at that
//                                        pressure),
//   E_i = p / (gamma - 1) + K + M_i      else (every child at the parent's pressure).
template <typename S>
__global__ void __launch_bounds__(kTransferThreads) positivity_ops_kernel(S* __restrict__ pool,
                                                                         const PatchDesc* __restrict__ patches,
                                                                         const PositivityOp* __restrict__ ops,
                                                                         double b0x, double b0y, double b0z,
                                                                         double gamma) {
  const PositivityOp op = ops[blockIdx.x];
  const PatchDesc F = patches[op.fine];
  const PatchDesc C = patches[op.coarse];
  const double b0[3] = {b0x, b0y, b0z};
  const double gm1 = gamma - 1.0;
  const int nchild = op.ndim == 3 ? 8 : 4;
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = threadIdx.x; t < count; t += kTransferThreads) {
    const unsigned line = t / n2;
    const int q[3] = {int(line / n1), int(line % n1), int(t - line * n2)};
    auto child = [&](int i, int (&x)[3]) {
      const int o[3] = {op.ndim == 3 ? (i >> 2) & 1 : (i >> 1) & 1, op.ndim == 3 ? (i >> 1) & 1 : i & 1,
                        op.ndim == 3 ? i & 1 : 0};
      for (int a = 0; a < 3; ++a) x[a] = a < op.ndim ? op.f0[a] + 2 * q[a] + o[a] : 0;
    };
    int xc[3];
    for (int a = 0; a < 3; ++a) xc[a] = a < op.ndim ? op.c0[a] + q[a] : 0;
    const int64_t oc = point_offset(C, xc[0], xc[1], xc[2]);
    const S* parent = pool + C.off + oc;
    const S rho = parent[0], m0 = parent[C.fstride], m1 = parent[2 * C.fstride], m2 = parent[3 * C.fstride];
    const double energy = double(parent[4 * C.fstride]);
    double bc[3];
    cell_field(pool, C, op.ndim, xc, b0, bc);
    const double k = kinetic(double(rho), double(m0), double(m1), double(m2));
    const double pc = dmul(gm1, dsub(dsub(energy, k), magnetic(bc)));
    if (!(double(rho) > 0.0 && pc > 0.0)) continue;  // the parent itself is not a valid state
    const double low = dmul(kPressureFraction, pc);
    bool bad = false;
    for (int i = 0; i < nchild; ++i) {
      int x[3];
      child(i, x);
      const int64_t o = point_offset(F, x[0], x[1], x[2]);
      const S* cell = pool + F.off + o;
      const double r = double(cell[0]);
      double b[3];
      cell_field(pool, F, op.ndim, x, b0, b);
      const double p = dmul(gm1, dsub(dsub(double(cell[4 * F.fstride]), kinetic(r, double(cell[F.fstride]),
                                                                                   double(cell[2 * F.fstride]),
                                                                                   double(cell[3 * F.fstride]))),
                                      magnetic(b)));
      if (!(r > 0.0 && p > low && isfinite(p))) bad = true;
    }
    if (!bad) continue;
    // the children's magnetic energies (2D: with the parent's B_z)
    double mag[8];
    double sum = 0.0;
    for (int i = 0; i < nchild; ++i) {
      int x[3];
      child(i, x);
      double b[3];
      cell_field(pool, F, op.ndim, x, b0, b);
      if (op.ndim == 2) b[2] = double(parent[5 * C.fstride]);
      mag[i] = magnetic(b);
      sum = dadd(sum, mag[i]);
    }
    const double mean = ddiv(sum, double(nchild));
    const bool keep = dmul(gm1, dsub(dsub(energy, k), mean)) > low;
    const double floor = dadd(ddiv(pc, gm1), k);
    for (int i = 0; i < nchild; ++i) {
      int x[3];
      child(i, x);
      S* cell = pool + F.off + point_offset(F, x[0], x[1], x[2]);
      cell[0] = rho;
      cell[F.fstride] = m0;
      cell[2 * F.fstride] = m1;
      cell[3 * F.fstride] = m2;
      cell[4 * F.fstride] = S(keep ? dadd(energy, dsub(mag[i], mean)) : dadd(floor, mag[i]));
      if (op.ndim == 2) cell[5 * F.fstride] = parent[5 * C.fstride];
    }
  }
}

// Kept values: dst[d + p] = old[s1 + p] over the box n, fields [field_lo, field_hi), from
// the old pool's patch src1 (CopyOp with unit weights and strides).
template <typename S>
__global__ void __launch_bounds__(kTransferThreads) kept_ops_kernel(S* __restrict__ pool,
                                                                   const PatchDesc* __restrict__ patches,
                                                                   const S* __restrict__ old_pool,
                                                                   const PatchDesc* __restrict__ old_patches,
                                                                   const CopyOp* __restrict__ ops) {
  const CopyOp op = ops[blockIdx.x];
  const PatchDesc D = patches[op.dst];
  const PatchDesc A = old_patches[op.src1];
  const unsigned n1 = unsigned(op.n[1]), n2 = unsigned(op.n[2]);
  const unsigned count = unsigned(op.n[0]) * n1 * n2;
  for (unsigned t = threadIdx.x; t < count; t += kTransferThreads) {
    const unsigned line = t / n2;
    const int p2 = int(t - line * n2), p1 = int(line % n1), p0 = int(line / n1);
    const int64_t od = point_offset(D, op.d[0] + p0, op.d[1] + p1, op.d[2] + p2);
    const int64_t os = point_offset(A, op.s1[0] + p0, op.s1[1] + p1, op.s1[2] + p2);
    for (int f = op.field_lo; f < op.field_hi; ++f) pool[D.off + f * D.fstride + od] = old_pool[A.off + f * A.fstride + os];
  }
}

}  // namespace wb

extern "C" {

int wb_prolong_ops(int precision, void* pool, const void* patches, const void* ops, int nops, void* stream) {
  using namespace wb;
  set_error("");
  if ((precision != 32 && precision != 64 && precision != 6432) || !pool || !patches || nops < 0 || (nops > 0 && !ops)) {
    set_error("prolong_ops: bad precision, op count or a NULL pointer");
    return kBadArgument;
  }
  if (nops == 0) return kOk;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == 32)
    prolong_ops_kernel<float><<<nops, kTransferThreads, 0, s>>>(static_cast<float*>(pool),
                                                                 static_cast<const PatchDesc*>(patches),
                                                                 static_cast<const ProlongOp*>(ops));
  else
    prolong_ops_kernel<double><<<nops, kTransferThreads, 0, s>>>(static_cast<double*>(pool),
                                                                  static_cast<const PatchDesc*>(patches),
                                                                  static_cast<const ProlongOp*>(ops));
  return check_launch("prolong_ops");
}

int wb_kept_ops(int precision, void* pool, const void* patches, const void* old_pool, const void* old_patches,
                const void* ops, int nops, void* stream) {
  using namespace wb;
  set_error("");
  if ((precision != 32 && precision != 64 && precision != 6432) || !pool || !patches || !old_pool || !old_patches ||
      nops < 0 || (nops > 0 && !ops)) {
    set_error("kept_ops: bad precision, op count or a NULL pointer");
    return kBadArgument;
  }
  if (nops == 0) return kOk;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == 32)
    kept_ops_kernel<float><<<nops, kTransferThreads, 0, s>>>(
        static_cast<float*>(pool), static_cast<const PatchDesc*>(patches), static_cast<const float*>(old_pool),
        static_cast<const PatchDesc*>(old_patches), static_cast<const CopyOp*>(ops));
  else
    kept_ops_kernel<double><<<nops, kTransferThreads, 0, s>>>(
        static_cast<double*>(pool), static_cast<const PatchDesc*>(patches), static_cast<const double*>(old_pool),
        static_cast<const PatchDesc*>(old_patches), static_cast<const CopyOp*>(ops));
  return check_launch("kept_ops");
}

int wb_positivity_ops(int precision, void* pool, const void* patches, const void* ops, int nops, double b0x,
                      double b0y, double b0z, double gamma, void* stream) {
  using namespace wb;
  set_error("");
  if ((precision != 32 && precision != 64 && precision != 6432) || !pool || !patches || nops < 0 || (nops > 0 && !ops)) {
    set_error("positivity_ops: bad precision, op count or a NULL pointer");
    return kBadArgument;
  }
  if (nops == 0) return kOk;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == 32)
    positivity_ops_kernel<float><<<nops, kTransferThreads, 0, s>>>(static_cast<float*>(pool),
                                                                    static_cast<const PatchDesc*>(patches),
                                                                    static_cast<const PositivityOp*>(ops), b0x, b0y,
                                                                    b0z, gamma);
  else
    positivity_ops_kernel<double><<<nops, kTransferThreads, 0, s>>>(static_cast<double*>(pool),
                                                                     static_cast<const PatchDesc*>(patches),
                                                                     static_cast<const PositivityOp*>(ops), b0x, b0y,
                                                                     b0z, gamma);
  return check_launch("positivity_ops");
}

}  // extern "C"
