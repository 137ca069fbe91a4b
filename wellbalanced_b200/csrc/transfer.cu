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

}  // extern "C"
