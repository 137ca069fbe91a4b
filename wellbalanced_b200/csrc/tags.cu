// The plain refinement tagger on the device: |J| times the cell size above a threshold,
// every cell of every patch of the tagged levels in one launch, written into the dense
// boolean arrays of the levels (carafe/mhd.py:1011-1041 in 2D, carafe/mhd3d.py:771-801
// in 3D). It replaces a per-patch loop of array operations and host copies: the host
// reads the levels' arrays once, for the clustering.
//
//   2D: J_z at the four nodes of a cell from the face fields (the curl of the nodal A_z
//       plus the mean field), averaged: 0.25 (J00 + J01 + J10 + J11) max(dx, dy);
//   3D: |curl B| of the cell-centred field (the mean of each cell's two faces), central
//       differences along each axis, times max(dx, dy, dz).
// All in float64 from the stored state (float32 or float64), with the reference's order of
// operations, so the tags are those of the reference's arithmetic on the same state.
#include "layout.cuh"
#include "wb_internal.cuh"

namespace wb {

constexpr int kTagThreads = 256;
constexpr unsigned kTagChunk = 2048;  // cells per work item (the rate kernels' chunks)

// Where a patch's cells go in the levels' arrays: tags[base + i s0 + j s1 + k] (s1 unused in
// 2D: tags[base + i s0 + j]).
struct TagPlace {
  int64_t base, s0, s1;
};

template <typename S>
__global__ void __launch_bounds__(kTagThreads) tags2d_kernel(const S* __restrict__ pool, const PatchDesc* patches,
                                                             const int* chunk_patch, const int* chunk_start,
                                                             const TagPlace* place, int levels, double b0x, double b0y,
                                                             double threshold, unsigned char* __restrict__ tags) {
  const int pi = chunk_patch[blockIdx.x];
  const PatchDesc P = patches[pi];
  if (P.level < 0 || P.level >= levels) return;
  const TagPlace T = place[pi];
  const int nx = P.n[0], ny = P.n[1];
  const S* A = pool + P.off + 6 * P.fstride;
  const int64_t p0 = P.pitch0;
  const double dx = P.dx[0], dy = P.dx[1], size = fmax(dx, dy);
  const unsigned total = unsigned(nx) * unsigned(ny);
  for (unsigned s = 0; s < kTagChunk / kTagThreads; ++s) {
    const unsigned t = unsigned(chunk_start[blockIdx.x]) + s * kTagThreads + threadIdx.x;
    if (t >= total) break;
    const int i = int(t / unsigned(ny)), j = int(t - unsigned(i) * unsigned(ny));
    // J_z at node (I, J) = (byf[I, J] - byf[I-1, J]) / dx - (bxf[I, J] - bxf[I, J-1]) / dy,
    // bxf[I, J] = (A[I, J+1] - A[I, J]) / dy + B0x, byf[I, J] = -(A[I+1, J] - A[I, J]) / dx + B0y
    auto bxf = [&](int I, int J) { return (double(A[I * p0 + J + 1]) - double(A[I * p0 + J])) / dy + b0x; };
    auto byf = [&](int I, int J) { return -((double(A[(I + 1) * p0 + J]) - double(A[I * p0 + J])) / dx) + b0y; };
    auto jz = [&](int I, int J) {
      return fabs((byf(I, J) - byf(I - 1, J)) / dx - (bxf(I, J) - bxf(I, J - 1)) / dy);
    };
    const int I = i + kHalo, J = j + kHalo;
    const double cell = 0.25 * (((jz(I, J) + jz(I, J + 1)) + jz(I + 1, J)) + jz(I + 1, J + 1));
    if (cell * size > threshold) tags[T.base + int64_t(i) * T.s0 + j] = 1;
  }
}

// The cell-centred field component a of haloed cell (I, J, K): the mean of its two
// a-faces, each the curl of the edge potential plus the mean field.
template <typename S>
__device__ __forceinline__ double cell_field3(const S* src, const PatchDesc& P, int a, int I, int J, int K,
                                              const double (&b0)[3]) {
  const int64_t fs = P.fstride, p0 = P.pitch0, p1 = P.pitch1;
  const int64_t step[3] = {p0, p1, 1};
  const int b = (a + 1) % 3, c = (a + 2) % 3;
  const S* Ab = src + (5 + b) * fs;
  const S* Ac = src + (5 + c) * fs;
  const double hb = P.dx[b], hc = P.dx[c];
  auto face = [&](int64_t o) {
    return (double(Ac[o + step[b]]) - double(Ac[o])) / hb - (double(Ab[o + step[c]]) - double(Ab[o])) / hc + b0[a];
  };
  const int64_t o = int64_t(I) * p0 + int64_t(J) * p1 + K;
  return 0.5 * (face(o) + face(o + step[a]));
}

template <typename S>
__global__ void __launch_bounds__(kTagThreads) tags3d_kernel(const S* __restrict__ pool, const PatchDesc* patches,
                                                             const int* chunk_patch, const int* chunk_start,
                                                             const TagPlace* place, int levels, double b0x, double b0y,
                                                             double b0z, double threshold,
                                                             unsigned char* __restrict__ tags) {
  const int pi = chunk_patch[blockIdx.x];
  const PatchDesc P = patches[pi];
  if (P.level < 0 || P.level >= levels) return;
  const TagPlace T = place[pi];
  const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
  const S* src = pool + P.off;
  const double b0[3] = {b0x, b0y, b0z};
  const double size = fmax(P.dx[0], fmax(P.dx[1], P.dx[2]));
  const unsigned total = unsigned(nx) * unsigned(ny) * unsigned(nz);
  for (unsigned s = 0; s < kTagChunk / kTagThreads; ++s) {
    const unsigned t = unsigned(chunk_start[blockIdx.x]) + s * kTagThreads + threadIdx.x;
    if (t >= total) break;
    const unsigned line = t / unsigned(nz);
    const int i = int(line / unsigned(ny)), j = int(line - unsigned(i) * unsigned(ny)), k = int(t - line * unsigned(nz));
    const int X[3] = {i + kHalo, j + kHalo, k + kHalo};
    double square = 0.0;
    for (int c = 0; c < 3; ++c) {
      const int a = (c + 1) % 3, b = (c + 2) % 3;
      // J_c = d_a B_b - d_b B_a, central differences (f[+1] - f[-1]) / (2 h)
      int lo[3] = {X[0], X[1], X[2]}, hi[3] = {X[0], X[1], X[2]};
      --lo[a], ++hi[a];
      const double dbb = (cell_field3(src, P, b, hi[0], hi[1], hi[2], b0) - cell_field3(src, P, b, lo[0], lo[1], lo[2], b0)) /
                         (2.0 * P.dx[a]);
      int lo2[3] = {X[0], X[1], X[2]}, hi2[3] = {X[0], X[1], X[2]};
      --lo2[b], ++hi2[b];
      const double dba = (cell_field3(src, P, a, hi2[0], hi2[1], hi2[2], b0) -
                          cell_field3(src, P, a, lo2[0], lo2[1], lo2[2], b0)) /
                         (2.0 * P.dx[b]);
      const double jc = dbb - dba;
      square = square + jc * jc;
    }
    if (sqrt(square) * size > threshold) tags[T.base + int64_t(i) * T.s0 + int64_t(j) * T.s1 + k] = 1;
  }
}

}  // namespace wb

extern "C" int wb_current_tags(int precision, int ndim, const void* pool, const void* patches, const int* chunk_patch,
                               const int* chunk_start, int nchunks, const void* place, int levels, double b0x,
                               double b0y, double b0z, double threshold, unsigned char* tags, void* stream) {
  using namespace wb;
  set_error("");
  if (precision != 32 && precision != 64 && precision != 6432) {
    set_error("current_tags: precision must be 32, 64 or 6432, got %d", precision);
    return kBadArgument;
  }
  if (!pool || !patches || !place || !tags || (nchunks > 0 && (!chunk_patch || !chunk_start)) || nchunks < 0 ||
      (ndim != 2 && ndim != 3) || levels < 0) {
    set_error("current_tags: bad ndim / levels / work list or a NULL pointer");
    return kBadArgument;
  }
  if (nchunks == 0 || levels == 0) return kOk;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const auto* P = static_cast<const PatchDesc*>(patches);
  const auto* T = static_cast<const TagPlace*>(place);
  if (precision == 32) {
    if (ndim == 2)
      tags2d_kernel<float><<<nchunks, kTagThreads, 0, s>>>(static_cast<const float*>(pool), P, chunk_patch,
                                                           chunk_start, T, levels, b0x, b0y, threshold, tags);
    else
      tags3d_kernel<float><<<nchunks, kTagThreads, 0, s>>>(static_cast<const float*>(pool), P, chunk_patch,
                                                           chunk_start, T, levels, b0x, b0y, b0z, threshold, tags);
  } else {
    if (ndim == 2)
      tags2d_kernel<double><<<nchunks, kTagThreads, 0, s>>>(static_cast<const double*>(pool), P, chunk_patch,
                                                            chunk_start, T, levels, b0x, b0y, threshold, tags);
    else
      tags3d_kernel<double><<<nchunks, kTagThreads, 0, s>>>(static_cast<const double*>(pool), P, chunk_patch,
                                                            chunk_start, T, levels, b0x, b0y, b0z, threshold, tags);
  }
  return check_launch("current_tags");
}
