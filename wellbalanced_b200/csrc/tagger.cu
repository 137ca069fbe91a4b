// Learned refinement tagger: stencil features of the 3D state and a small MLP
// (16 -> 64 -> 64 -> 1, ReLU) with bfloat16 weights and float32 accumulation, trained on
// the device. It predicts which cells the plain current tagger (|J| dx > threshold,
// carafe/mhd3d.py:771-801) will flag within the next steps, so a hierarchy can be regridded
// less often. There is no counterpart in the reference; the float64 NumPy restatement in
// oracle/mlp.py is the checker of the forward and backward passes.
//
// Model (the same in every kernel): x^ = bf16(x); z1 = bf16(W1) x^ + b1; h1 = relu(z1);
// z2 = bf16(W2) bf16(h1) + b2; h2 = relu(z2); z = bf16(W3) . h2 + b3. Gradients pass
// through the bf16 roundings unchanged. Parameters live in one float32 buffer:
// W1 [64][16] | b1 [64] | W2 [64][64] | b2 [64] | W3 [64] | b3 [1]  (5313 values).
#include <cuda_bf16.h>

#include <algorithm>

#include "layout.cuh"
#include "numerics.cuh"
#include "stage.cuh"
#include "wb_internal.cuh"

namespace wb {

constexpr int kFeat = 16, kHid = 64;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kFeat, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid, kParams = kOffB3 + 1;
static_assert(kParams == 5313, "parameter layout");

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// ---- features ------------------------------------------------------------------------------------
// (log rho, log p, |B|) of haloed cell (i, j, k) of a 3D patch (cell B = mean of its face fields
// from the curl of the edge potential, as the stage kernels form it).
template <typename S>
__device__ __forceinline__ void cell_quantities(const S* src, const PatchDesc& P, int i, int j, int k,
                                                const double* b0, double gamma, float (&q)[3]) {
  using M = Math<S>;
  const int64_t p0 = P.pitch0, p1 = P.pitch1, fs = P.fstride;
  const int64_t o = int64_t(i) * p0 + int64_t(j) * p1 + k;
  const S* Ax = src + 5 * fs;
  const S* Ay = src + 6 * fs;
  const S* Az = src + 7 * fs;
  const S dx = S(P.dx[0]), dy = S(P.dx[1]), dz = S(P.dx[2]);
  const S idx = M::inv(dx), idy = M::inv(dy), idz = M::inv(dz);
  auto fx = [&](int64_t c) { return M::div(Az[c + p1] - Az[c], dy, idy) - M::div(Ay[c + 1] - Ay[c], dz, idz) + S(b0[0]); };
  auto fy = [&](int64_t c) { return M::div(Ax[c + 1] - Ax[c], dz, idz) - M::div(Az[c + p0] - Az[c], dx, idx) + S(b0[1]); };
  auto fz = [&](int64_t c) { return M::div(Ay[c + p0] - Ay[c], dx, idx) - M::div(Ax[c + p1] - Ax[c], dy, idy) + S(b0[2]); };
  const S bx = S(0.5) * (fx(o) + fx(o + p0));
  const S by = S(0.5) * (fy(o) + fy(o + p1));
  const S bz = S(0.5) * (fz(o) + fz(o + 1));
  const S r = src[o];
  const S m0 = src[fs + o], m1 = src[2 * fs + o], m2 = src[3 * fs + o], e = src[4 * fs + o];
  const S ir = M::inv(r);
  const S p = recover_pressure<S>(r, m0, m1, m2, e, bx, by, bz, m0 * ir, m1 * ir, m2 * ir, gamma);
  q[0] = logf(fmaxf(float(r), 1e-30f));
  q[1] = logf(fmaxf(float(p), 1e-30f));
  q[2] = sqrtf(float(bx * bx + by * by + bz * bz));
}

// One thread per interior cell (work list of the rate kernels: up to 2048 cells per chunk).
// Features of a cell from its 3 x 3 x 3 neighbourhood, for each of (log rho, log p, |B|):
// the value, the three central differences (half the difference of the two neighbours
// along an axis) and the largest deviation over the 26 neighbours; feature 15 is zero.
// Output row t of a patch's block is its cell (i, j, k) in (i, j, k) order, normalised
// as (f - mean) * inv_std.
template <typename S>
__global__ void __launch_bounds__(256) tag_features3d_kernel(const S* __restrict__ pool, const PatchDesc* patches,
                                                             const int* chunk_patch, const int* chunk_start,
                                                             const int64_t* row_start, double b0x, double b0y,
                                                             double b0z, double gamma, const float* mean,
                                                             const float* inv_std, float* __restrict__ out) {
  const int pi = chunk_patch[blockIdx.x];
  const PatchDesc P = patches[pi];
  const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
  const S* src = pool + P.off;
  const double b0[3] = {b0x, b0y, b0z};
  const unsigned total = unsigned(nx) * unsigned(ny) * unsigned(nz);
  const unsigned start = unsigned(chunk_start[blockIdx.x]);
  for (int s = 0; s < 8; ++s) {
    const unsigned t = start + unsigned(s) * blockDim.x + threadIdx.x;
    if (t >= total) break;
    const unsigned line = t / unsigned(nz);
    const unsigned plane = line / unsigned(ny);
    const int i = int(plane) + kHalo, j = int(line - plane * unsigned(ny)) + kHalo,
              k = int(t - line * unsigned(nz)) + kHalo;
    float q[3][3][3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) cell_quantities<S>(src, P, i + a - 1, j + b - 1, k + c - 1, b0, gamma, q[a][b][c]);
    float f[kFeat];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const float c0 = q[1][1][1][v];
      float dev = 0.0f;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
          for (int c = 0; c < 3; ++c) dev = fmaxf(dev, fabsf(q[a][b][c][v] - c0));
      f[v] = c0;
      f[3 + 3 * v + 0] = 0.5f * (q[2][1][1][v] - q[0][1][1][v]);
      f[3 + 3 * v + 1] = 0.5f * (q[1][2][1][v] - q[1][0][1][v]);
      f[3 + 3 * v + 2] = 0.5f * (q[1][1][2][v] - q[1][1][0][v]);
      f[12 + v] = dev;
    }
    f[15] = 0.0f;
    float* row = out + (row_start[pi] + int64_t(t)) * kFeat;
#pragma unroll
    for (int c = 0; c < kFeat; ++c) row[c] = (f[c] - mean[c]) * inv_std[c];
  }
}

// ---- forward on the tensor cores --------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// D = A (16 x 16, row) * B (16 x 8, col) + D; bf16 inputs, float32 accumulation.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Padded row pitches (in bf16) of the weights in shared memory: rows 16 B apart modulo 128 B,
// so the 8 rows a fragment load touches fall in different banks.
constexpr int kPitch1 = kFeat + 8, kPitch2 = kHid + 8;

// Each warp takes 16 rows at a time: layer 1 as 8 mma (one per 8 outputs), layer 2 as
// 32 mma with the layer-1 accumulators re-packed in registers as its A fragments
// (the accumulator layout of m16n8 matches the A layout of the next k-tile), layer 3 as
// a dot product reduced over the four threads that hold a row.
__global__ void __launch_bounds__(256) mlp_forward_kernel(const float* __restrict__ X, int64_t n,
                                                          const float* __restrict__ params,
                                                          float* __restrict__ logits) {
  __shared__ __align__(16) __nv_bfloat16 sW1[kHid * kPitch1];
  __shared__ __align__(16) __nv_bfloat16 sW2[kHid * kPitch2];
  __shared__ float sB1[kHid], sB2[kHid], sW3[kHid];
  for (int t = threadIdx.x; t < kHid * kFeat; t += blockDim.x)
    sW1[(t / kFeat) * kPitch1 + t % kFeat] = __float2bfloat16_rn(params[kOffW1 + t]);
  for (int t = threadIdx.x; t < kHid * kHid; t += blockDim.x)
    sW2[(t / kHid) * kPitch2 + t % kHid] = __float2bfloat16_rn(params[kOffW2 + t]);
  for (int t = threadIdx.x; t < kHid; t += blockDim.x) {
    sB1[t] = params[kOffB1 + t];
    sB2[t] = params[kOffB2 + t];
    sW3[t] = bf16r(params[kOffW3 + t]);
  }
  __syncthreads();
  const float b3 = params[kOffB3];
  const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t tile = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); tile * 16 < n; tile += warps) {
    const int64_t r0 = tile * 16 + g, r1 = r0 + 8;
    auto x = [&](int64_t r, int c) { return r < n ? X[r * kFeat + c] : 0.0f; };
    uint32_t a[4];
    a[0] = pack_bf16(x(r0, 2 * tg), x(r0, 2 * tg + 1));
    a[1] = pack_bf16(x(r1, 2 * tg), x(r1, 2 * tg + 1));
    a[2] = pack_bf16(x(r0, 2 * tg + 8), x(r0, 2 * tg + 9));
    a[3] = pack_bf16(x(r1, 2 * tg + 8), x(r1, 2 * tg + 9));
    float h1[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int col = nt * 8 + 2 * tg;
      h1[nt][0] = h1[nt][2] = sB1[col];
      h1[nt][1] = h1[nt][3] = sB1[col + 1];
      const __nv_bfloat16* w = sW1 + (nt * 8 + g) * kPitch1 + 2 * tg;
      mma_bf16(h1[nt], a, *reinterpret_cast<const uint32_t*>(w), *reinterpret_cast<const uint32_t*>(w + 8));
#pragma unroll
      for (int e = 0; e < 4; ++e) h1[nt][e] = fmaxf(h1[nt][e], 0.0f);
    }
    float h2[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int col = nt * 8 + 2 * tg;
      h2[nt][0] = h2[nt][2] = sB2[col];
      h2[nt][1] = h2[nt][3] = sB2[col + 1];
    }
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      uint32_t a2[4];
      a2[0] = pack_bf16(h1[2 * kk][0], h1[2 * kk][1]);
      a2[1] = pack_bf16(h1[2 * kk][2], h1[2 * kk][3]);
      a2[2] = pack_bf16(h1[2 * kk + 1][0], h1[2 * kk + 1][1]);
      a2[3] = pack_bf16(h1[2 * kk + 1][2], h1[2 * kk + 1][3]);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const __nv_bfloat16* w = sW2 + (nt * 8 + g) * kPitch2 + kk * 16 + 2 * tg;
        mma_bf16(h2[nt], a2, *reinterpret_cast<const uint32_t*>(w), *reinterpret_cast<const uint32_t*>(w + 8));
      }
    }
    float z0 = 0.0f, z1 = 0.0f;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int col = nt * 8 + 2 * tg;
      z0 += fmaxf(h2[nt][0], 0.0f) * sW3[col] + fmaxf(h2[nt][1], 0.0f) * sW3[col + 1];
      z1 += fmaxf(h2[nt][2], 0.0f) * sW3[col] + fmaxf(h2[nt][3], 0.0f) * sW3[col + 1];
    }
    z0 += __shfl_xor_sync(0xffffffffu, z0, 1);
    z0 += __shfl_xor_sync(0xffffffffu, z0, 2);
    z1 += __shfl_xor_sync(0xffffffffu, z1, 1);
    z1 += __shfl_xor_sync(0xffffffffu, z1, 2);
    if (tg == 0) {
      if (r0 < n) logits[r0] = z0 + b3;
      if (r1 < n) logits[r1] = z1 + b3;
    }
  }
}

// ---- backward on the CUDA cores -----------------------------------------------------------------------
// 256 threads, 64 samples per round, 4 threads per sample (16 hidden units each). A round
// recomputes the forward pass in float32, forms dL/dz = w (sigmoid(z) - y) of the weighted
// binary cross-entropy (w = pos_weight for y = 1), back-propagates, and parks x^, bf16(h1),
// h2 and the deltas in shared memory; then every thread accumulates its share of the weight
// gradients over the round's samples. Each block adds its sums to `grads` (float32,
// parameter layout) once; `loss` (float64) gets the summed loss.
constexpr int kRound = 64;
constexpr size_t kBackwardSmem =
    sizeof(float) * (kHid * kFeat + kHid * (kHid + 1) + 3 * kHid + kRound * (kFeat + 1) + 4 * kRound * (kHid + 1) + kRound);

__global__ void __launch_bounds__(256) mlp_backward_kernel(const float* __restrict__ X, const float* __restrict__ y,
                                                           int64_t n, const float* __restrict__ params,
                                                           float pos_weight, float* __restrict__ grads,
                                                           double* __restrict__ loss) {
  extern __shared__ __align__(16) float smem[];
  float* sW1 = smem;                         // [64][16] bf16-rounded, [out][in]
  float* sW2 = sW1 + kHid * kFeat;           // [64][65]
  float* sB1 = sW2 + kHid * (kHid + 1);      // [64]
  float* sB2 = sB1 + kHid;                   // [64]
  float* sW3 = sB2 + kHid;                   // [64]
  float* sX = sW3 + kHid;                    // [round][17]
  float* sH1 = sX + kRound * (kFeat + 1);    // [round][65] bf16(h1)
  float* sH2 = sH1 + kRound * (kHid + 1);    // [round][65]
  float* sD1 = sH2 + kRound * (kHid + 1);    // [round][65]
  float* sD2 = sD1 + kRound * (kHid + 1);    // [round][65]
  float* sD3 = sD2 + kRound * (kHid + 1);    // [round]
  __shared__ double sLoss[8];
  for (int t = threadIdx.x; t < kHid * kFeat; t += blockDim.x) sW1[t] = bf16r(params[kOffW1 + t]);
  for (int t = threadIdx.x; t < kHid * kHid; t += blockDim.x)
    sW2[(t / kHid) * (kHid + 1) + t % kHid] = bf16r(params[kOffW2 + t]);
  for (int t = threadIdx.x; t < kHid; t += blockDim.x) {
    sB1[t] = params[kOffB1 + t];
    sB2[t] = params[kOffB2 + t];
    sW3[t] = bf16r(params[kOffW3 + t]);
  }
  __syncthreads();
  const float b3 = params[kOffB3];
  const int tid = threadIdx.x, s = tid >> 2, part = tid & 3;  // sample of the round, quarter of the units
  // gradient shares: W2 entries tid*16 .. +15 (row tid/4, columns (tid%4)*16 ..), W1 entries tid*4 .. +3
  float gw2[16], gw1[4], gw3 = 0.0f, gb1 = 0.0f, gb2 = 0.0f, gb3 = 0.0f;
#pragma unroll
  for (int e = 0; e < 16; ++e) gw2[e] = 0.0f;
#pragma unroll
  for (int e = 0; e < 4; ++e) gw1[e] = 0.0f;
  double my_loss = 0.0;
  for (int64_t base = int64_t(blockIdx.x) * kRound; base < n; base += int64_t(gridDim.x) * kRound) {
    const int64_t r = base + s;
    const bool live = r < n;
    // forward -----------------------------------------------------------------------------
    if (part == 0) {
#pragma unroll
      for (int c = 0; c < kFeat; ++c) sX[(s) * (kFeat + 1) + (c)] = live ? bf16r(X[r * kFeat + c]) : 0.0f;
    }
    __syncthreads();
    float z1[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int j = part * 16 + u;
      float acc = sB1[j];
#pragma unroll
      for (int c = 0; c < kFeat; ++c) acc = fmaf(sW1[j * kFeat + c], sX[(s) * (kFeat + 1) + (c)], acc);
      z1[u] = acc;
      sH1[(s) * (kHid + 1) + (j)] = bf16r(fmaxf(acc, 0.0f));
    }
    __syncthreads();
    float z2[16], z = 0.0f;
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int j = part * 16 + u;
      float acc = sB2[j];
      for (int c = 0; c < kHid; ++c) acc = fmaf(sW2[j * (kHid + 1) + c], sH1[(s) * (kHid + 1) + (c)], acc);
      z2[u] = acc;
      const float h = fmaxf(acc, 0.0f);
      sH2[(s) * (kHid + 1) + (j)] = h;
      z = fmaf(h, sW3[j], z);
    }
    z += __shfl_xor_sync(0xffffffffu, z, 1);
    z += __shfl_xor_sync(0xffffffffu, z, 2);
    z += b3;
    // loss and output delta -------------------------------------------------------------------
    const float target = live ? y[r] : 0.0f;
    const float w = target > 0.5f ? pos_weight : 1.0f;
    const float prob = 1.0f / (1.0f + __expf(-z));
    const float d3 = live ? w * (prob - target) : 0.0f;
    if (part == 0) {
      sD3[s] = d3;
      // softplus(z) - y z, evaluated without overflow
      const float sp = fmaxf(z, 0.0f) + log1pf(__expf(-fabsf(z)));
      my_loss += live ? double(w) * double(sp - target * z) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int j = part * 16 + u;
      sD2[(s) * (kHid + 1) + (j)] = z2[u] > 0.0f ? d3 * sW3[j] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int i = part * 16 + u;
      float acc = 0.0f;
      for (int j = 0; j < kHid; ++j) acc = fmaf(sW2[j * (kHid + 1) + i], sD2[(s) * (kHid + 1) + (j)], acc);
      sD1[(s) * (kHid + 1) + (i)] = z1[u] > 0.0f ? acc : 0.0f;
    }
    __syncthreads();
    // weight-gradient shares over the round's samples ---------------------------------------------
    {
      const int j2 = tid >> 2, i2 = (tid & 3) * 16;
      for (int q = 0; q < kRound; ++q) {
        const float d = sD2[(q) * (kHid + 1) + (j2)];
#pragma unroll
        for (int e = 0; e < 16; ++e) gw2[e] = fmaf(d, sH1[(q) * (kHid + 1) + (i2 + e)], gw2[e]);
      }
      const int j1 = tid >> 2, i1 = (tid & 3) * 4;
      for (int q = 0; q < kRound; ++q) {
        const float d = sD1[(q) * (kHid + 1) + (j1)];
#pragma unroll
        for (int e = 0; e < 4; ++e) gw1[e] = fmaf(d, sX[(q) * (kFeat + 1) + (i1 + e)], gw1[e]);
      }
      if (tid < kHid) {
        for (int q = 0; q < kRound; ++q) {
          gw3 = fmaf(sD3[q], sH2[(q) * (kHid + 1) + (tid)], gw3);
          gb2 += sD2[(q) * (kHid + 1) + (tid)];
          gb1 += sD1[(q) * (kHid + 1) + (tid)];
        }
      }
      if (tid == 0)
        for (int q = 0; q < kRound; ++q) gb3 += sD3[q];
    }
    __syncthreads();
  }
  const int j2 = tid >> 2, i2 = (tid & 3) * 16;
#pragma unroll
  for (int e = 0; e < 16; ++e) atomicAdd(&grads[kOffW2 + j2 * kHid + i2 + e], gw2[e]);
  const int j1 = tid >> 2, i1 = (tid & 3) * 4;
#pragma unroll
  for (int e = 0; e < 4; ++e) atomicAdd(&grads[kOffW1 + j1 * kFeat + i1 + e], gw1[e]);
  if (tid < kHid) {
    atomicAdd(&grads[kOffW3 + tid], gw3);
    atomicAdd(&grads[kOffB2 + tid], gb2);
    atomicAdd(&grads[kOffB1 + tid], gb1);
  }
  if (tid == 0) atomicAdd(&grads[kOffB3], gb3);
  // block sum of the loss (one value per sample-owning thread)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_loss += __shfl_xor_sync(0xffffffffu, my_loss, o);
  if ((tid & 31) == 0) sLoss[tid >> 5] = my_loss;
  __syncthreads();
  if (tid == 0) {
    double total = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) total += sLoss[w];
    atomicAdd(loss, total);
  }
}

// Adam on the float32 parameters with gradients scaled by `scale` (1 / batch size); the
// gradients are cleared for the next accumulation.
__global__ void mlp_adam_kernel(float* params, float* grads, float* m, float* v, int count, float lr, float beta1,
                                float beta2, float eps, float bias1, float bias2, float scale) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const float g = grads[t] * scale;
  const float mt = beta1 * m[t] + (1.0f - beta1) * g;
  const float vt = beta2 * v[t] + (1.0f - beta2) * g * g;
  m[t] = mt;
  v[t] = vt;
  params[t] -= lr * (mt / bias1) / (sqrtf(vt / bias2) + eps);
  grads[t] = 0.0f;
}

}  // namespace wb

// ---- C ABI ---------------------------------------------------------------------------------------
using namespace wb;

extern "C" int wb_tag_features(int precision, const void* pool, const void* patches, const int* chunk_patch,
                               const int* chunk_start, int nchunks, const int64_t* row_start, double b0x, double b0y,
                               double b0z, double gamma, const float* mean, const float* inv_std, float* out,
                               void* stream) {
  set_error("");
  if (!pool || !patches || !row_start || !mean || !inv_std || !out || (nchunks > 0 && (!chunk_patch || !chunk_start))) {
    set_error("tag_features: null pointer");
    return kBadArgument;
  }
  if (nchunks <= 0) return kOk;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == 32)
    tag_features3d_kernel<float><<<nchunks, 256, 0, s>>>(static_cast<const float*>(pool),
                                                         static_cast<const PatchDesc*>(patches), chunk_patch,
                                                         chunk_start, row_start, b0x, b0y, b0z, gamma, mean,
                                                         inv_std, out);
  else if (precision == 64 || precision == kMath32State64)  // a float64 state
    tag_features3d_kernel<double><<<nchunks, 256, 0, s>>>(static_cast<const double*>(pool),
                                                          static_cast<const PatchDesc*>(patches), chunk_patch,
                                                          chunk_start, row_start, b0x, b0y, b0z, gamma, mean,
                                                          inv_std, out);
  else {
    set_error("tag_features: precision is 32, 64 or %d, not %d", kMath32State64, precision);
    return kBadArgument;
  }
  return check_launch("tag_features");
}

extern "C" int wb_mlp_forward(const float* features, int64_t n, const float* params, float* logits, void* stream) {
  set_error("");
  if (!features || !params || !logits || n < 0) {
    set_error("mlp_forward: null pointer or negative row count");
    return kBadArgument;
  }
  if (n == 0) return kOk;
  const int64_t tiles = (n + 15) / 16;
  const int blocks = int(std::min<int64_t>((tiles + 7) / 8, 148 * 8));
  mlp_forward_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(features, n, params, logits);
  return check_launch("mlp_forward");
}

extern "C" int wb_mlp_backward(const float* features, const float* targets, int64_t n, const float* params,
                               float pos_weight, float* grads, double* loss, void* stream) {
  set_error("");
  if (!features || !targets || !params || !grads || !loss || n < 0) {
    set_error("mlp_backward: null pointer or negative row count");
    return kBadArgument;
  }
  if (n == 0) return kOk;
  const int blocks = int(std::min<int64_t>((n + kRound - 1) / kRound, 148 * 2));
  cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kBackwardSmem));
  mlp_backward_kernel<<<blocks, 256, kBackwardSmem, static_cast<cudaStream_t>(stream)>>>(
      features, targets, n, params, pos_weight, grads, loss);
  return check_launch("mlp_backward");
}

extern "C" int wb_mlp_adam(float* params, float* grads, float* m, float* v, int count, float lr, float beta1,
                           float beta2, float eps, int step, float scale, void* stream) {
  set_error("");
  if (!params || !grads || !m || !v || count != kParams || step < 1) {
    set_error("mlp_adam: null pointer, parameter count other than %d, or step < 1", kParams);
    return kBadArgument;
  }
  const float bias1 = 1.0f - powf(beta1, float(step)), bias2 = 1.0f - powf(beta2, float(step));
  mlp_adam_kernel<<<(count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      params, grads, m, v, count, lr, beta1, beta2, eps, bias1, bias2, scale);
  return check_launch("mlp_adam");
}
