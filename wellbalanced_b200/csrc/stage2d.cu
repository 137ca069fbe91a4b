// Fused 2D stage kernel: one RK stage of every tile of every patch in one launch.
//
// Per tile (TX x TY cells of a patch, a halo of two), all in shared memory:
//   1. load the conserved cells and A_z nodes, form the face fields (curl of A_z), the
//      cell field, the primitive variables (pressure recovery in float64), the cell E_z
//      and count bad cells (mhd_primitive_pyccel.py:23-87);
//   2. MUSCL + HLLD on every x- and y-face the tile needs (mhd_sweep_pyccel.py:254-319);
//   3. CT-contact E_z at the tile's nodes (ct_contact_pyccel.py:26-61), walls, and the
//      stage update of the cells (U -= dt div F, FluxRegister.update) and of A_z
//      (A -= dt E_z), with the Heun combine in stage 2 (carafe/mhd.py:889-927, 965-994).
// The primitive variables and fluxes never reach HBM; each stage reads its input state
// (and, in stage 2, the start state at the cell itself) and writes the new state once.
#include <type_traits>

#include "layout.cuh"
#include "numerics.cuh"
#include "stage.cuh"
#include "wb_internal.cuh"

namespace wb {

// Tile shapes (TX x TY cells) the 2D stage kernel is built for, per (state type S,
// arithmetic type R); the first of each is the default and the only one with the
// non-ideal terms. The others are candidates of the autotuner (more tiles for small
// patches, less halo overhead for large ones).
template <typename S, typename R = S>
struct Tile2D;

template <>
struct Tile2D<float, float> {
  static constexpr int TX = 16, TY = 32;
  static constexpr int kShapes = 4;
  static constexpr int kShape[kShapes][2] = {{16, 32}, {8, 32}, {16, 16}, {32, 16}};
};
template <>
struct Tile2D<double, double> {
  static constexpr int TX = 8, TY = 32;
  static constexpr int kShapes = 3;
  static constexpr int kShape[kShapes][2] = {{8, 32}, {8, 16}, {16, 16}};
};
// float64 state, float32 arithmetic: the float32 shapes (shared memory holds float32)
template <>
struct Tile2D<double, float> {
  static constexpr int TX = 16, TY = 32;
  static constexpr int kShapes = 3;
  static constexpr int kShape[kShapes][2] = {{16, 32}, {8, 32}, {16, 16}};
};

template <typename S>
__device__ __forceinline__ bool bad_cell(S r, S u, S v, S w, S p, S bx, S by, S bz) {
  if (!(r > S(0) && p > S(0))) return true;
  return !(isfinite(r) && isfinite(u) && isfinite(v) && isfinite(w) && isfinite(p) && isfinite(bx) &&
           isfinite(by) && isfinite(bz));
}

// J_z at interior node (ni, nj) of the tile from the face fields in shared memory:
// dB_y/dx - dB_x/dy (carafe/kernels/mhd_resistive/mhd_resistive_pyccel.py:21-67).
template <typename S, int CY>
__device__ __forceinline__ S node_current(const S* sBx, const S* sBy, int ni, int nj, S dx, S idx, S dy, S idy) {
  using M = Math<S>;
  return M::div(sBy[(ni + 2) * CY + nj + 2] - sBy[(ni + 1) * CY + nj + 2], dx, idx) -
         M::div(sBx[(ni + 2) * CY + nj + 2] - sBx[(ni + 2) * CY + nj + 1], dy, idy);
}

// Temperature p / rho of local cell t.
template <typename S, int NC>
__device__ __forceinline__ S temperature(const S* sP, int t) {
  using M = Math<S>;
  const S r = sP[t];
  return M::div(sP[4 * NC + t], r, M::inv(r));
}

// PHYS: the resistive and Braginskii-conductive face terms and gravity sources of the
// reference (carafe/mhd.py:844-927) in the same kernel; false for ideal MHD.
constexpr int kThreads2D = 256;  // threads of a stage2d CTA

// CTAs per SM the launch bounds hold the registers to: three 256-thread CTAs of float32
// (80 registers a thread, 63 KB of shared memory each), two of float64 and of the float64
// state with float32 arithmetic (its stage input and Heun base are held in float64).
template <typename S, typename R = S>
struct Occupancy2D {
  static constexpr int kBlocks = sizeof(S) == 4 ? 3 : 2;
};

// S: the state's type (loads, the conserved and potential updates, the Heun combine);
// R: the arithmetic of the reconstruction, HLLD and CT (float32 or float64). With a
// float64 state and float32 arithmetic (S = double, R = float) the primitive variables
// and face fields are formed in float64 from the float64 state (face fields from float64
// differences of the potential; pressure in float64) and rounded to float32 for the face
// work; the flux differences, the updates U -= dt div F and A -= dt E and the Heun combine
// are float64.
template <typename S, typename R, int LIM, bool PHYS, int TX, int TY>
__global__ void __launch_bounds__(kThreads2D, (Occupancy2D<S, R>::kBlocks)) stage2d_kernel(const StageArgs<S> a) {
  using M = Math<R>;
  // phase 1 (cells -> primitive variables) in the state's type; a float64 state with
  // float32 arithmetic takes float32-seeded float64 reciprocals there
  using W = S;
  using MW = typename std::conditional<std::is_same<S, R>::value, Math<S>, MathRefined>::type;
  constexpr bool kMixed = !std::is_same<S, R>::value;
  constexpr int CX = TX + 4, CY = TY + 4, NC = CX * CY;
  constexpr int FX = TX + 1, FY = TY + 1, NF = FX * FY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sP = reinterpret_cast<R*>(smem_raw);  // [8][NC] primitive variables
  R* sBx = sP + 8 * NC;                     // [NC] x-face field at each cell's lower x-face
  R* sBy = sBx + NC;                        // [NC] y-face field at each cell's lower y-face
  R* sE = sBy + NC;                         // [NC] cell E_z
  R* sFx = sE + NC;                         // [7][NF] x-face fluxes, face (fi, fj) at fi*FY + fj+1
  R* sFy = sFx + 7 * NF;                    // [7][NF] y-face fluxes, face (fi, fj) at (fi+1)*FY + fj

  const Tile tile = a.tiles[blockIdx.x];
  const PatchDesc P = a.patches[tile.patch];
  const int nx = P.n[0], ny = P.n[1];
  const int64_t pitch = P.pitch0, fs = P.fstride;
  const S* __restrict__ src = a.src + P.off;
  const R dx = R(P.dx[0]), dy = R(P.dx[1]);
  const R idx = M::inv(dx), idy = M::inv(dy);
  const R gamma = R(a.gamma), inv_gm1 = R(a.inv_gm1);
  const int x0 = tile.x0, y0 = tile.y0;
  const int own_nx = nx + ((P.flags & kOwnLast0) ? 1 : 0);
  const int own_ny = ny + ((P.flags & kOwnLast1) ? 1 : 0);

  // stage 2: fetch the Heun base state of the tile's cells and nodes into L2 now (each row
  // of the tile spans at most two 128-byte lines), so that phase 3 reads it from there
  if (a.base) {
    const S* bs = a.base + P.off;
    const int rows = min(TX, own_nx - x0);
    for (int t = threadIdx.x; t < 7 * rows * 2; t += blockDim.x) {
      const int f = t / (rows * 2), row = (t / 2) % rows, half = t & 1;
      const int col = min(y0 + 2 + half * (TY - 1), ny + 4);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(bs + f * fs + int64_t(x0 + row + 2) * pitch + col));
    }
  }

  // 1. cells and nodes -> primitive variables -------------------------------------
  unsigned bad = 0;
  {
    const W wdx = W(P.dx[0]), wdy = W(P.dx[1]);
    const W widx = MW::inv(wdx), widy = MW::inv(wdy);
    const W b0x = W(a.b0[0]), b0y = W(a.b0[1]);
    for (int t = threadIdx.x; t < NC; t += blockDim.x) {
      const int li = t / CY, lj = t - (t / CY) * CY;
      const int gi = x0 + li, gj = y0 + lj;  // haloed indices
      W r = W(1), m0 = W(0), m1 = W(0), m2 = W(0), e = W(1), bz = W(0);
      W bxl = W(0), bxh = W(0), byl = W(0), byh = W(0);
      const bool valid = gi < nx + 4 && gj < ny + 4;
      if (valid) {
        const int64_t c = int64_t(gi) * pitch + gj;
        r = src[c];
        m0 = src[fs + c];
        m1 = src[2 * fs + c];
        m2 = src[3 * fs + c];
        e = src[4 * fs + c];
        bz = src[5 * fs + c];
        const S* A = src + 6 * fs;
        const W a00 = A[c], a01 = A[c + 1], a10 = A[c + pitch], a11 = A[c + pitch + 1];
        bxl = MW::div(a01 - a00, wdy, widy) + b0x;
        bxh = MW::div(a11 - a10, wdy, widy) + b0x;
        byl = -MW::div(a10 - a00, wdx, widx) + b0y;
        byh = -MW::div(a11 - a01, wdx, widx) + b0y;
      }
      const W ir = MW::inv(r);
      const W u = MW::div(m0, r, ir), v = MW::div(m1, r, ir), w = MW::div(m2, r, ir);
      const W bx = W(0.5) * (bxl + bxh), by = W(0.5) * (byl + byh);
      W p = recover_pressure<W>(r, m0, m1, m2, e, bx, by, bz, u, v, w, a.gamma);
      if (!valid) p = W(1);
      sP[t] = R(r);
      sP[NC + t] = R(u);
      sP[2 * NC + t] = R(v);
      sP[3 * NC + t] = R(w);
      sP[4 * NC + t] = R(p);
      sP[5 * NC + t] = R(bx);
      sP[6 * NC + t] = R(by);
      sP[7 * NC + t] = R(bz);
      sBx[t] = R(bxl);
      sBy[t] = R(byl);
      sE[t] = R(bx * v - by * u);
      // the tile's own cells
      const int ci = li - 2, cj = lj - 2;
      if (valid && ci >= 0 && ci < TX && cj >= 0 && cj < TY && x0 + ci < nx && y0 + cj < ny &&
          bad_cell(r, u, v, w, p, bx, by, bz))
        ++bad;
    }
  }
  if (bad) atomicAdd(a.bad, (unsigned long long)bad);
  __syncthreads();

  // 2. x- and y-faces: MUSCL + HLLD -------------------------------------------------
  for (int t = threadIdx.x; t < 2 * NF; t += blockDim.x) {
    const bool xface = t < NF;
    const int u = xface ? t : t - NF;
    int fi, fj, base, step;
    R bn;
    int comp[7];
    if (xface) {
      fi = u / FY;           // face fi: between cells fi-1 and fi (tile-relative)
      fj = u % FY - 1;       // row fj in [-1, TY)
      base = fi * CY + (fj + 2);  // local cell fi-2 -> li = fi
      step = CY;
      bn = sBx[(fi + 2) * CY + fj + 2];
      comp[0] = 0; comp[1] = 1; comp[2] = 2; comp[3] = 3; comp[4] = 4; comp[5] = 6; comp[6] = 7;
    } else {
      fi = u / FY - 1;       // column fi in [-1, TX)
      fj = u % FY;           // face fj: between cells fj-1 and fj
      base = (fi + 2) * CY + fj;
      step = 1;
      bn = sBy[(fi + 2) * CY + fj + 2];
      comp[0] = 0; comp[1] = 2; comp[2] = 1; comp[3] = 3; comp[4] = 4; comp[5] = 5; comp[6] = 7;
    }
    R q0[7], q1[7], q2[7], q3[7];
#pragma unroll
    for (int c = 0; c < 7; ++c) {
      const R* row = sP + comp[c] * NC + base;
      q0[c] = row[0];
      q1[c] = row[step];
      q2[c] = row[2 * step];
      q3[c] = row[3 * step];
    }
    R L[7], Rt[7], F[7];
    reconstruct<LIM>(q0, q1, q2, q3, L, Rt);
    hlld_flux(L, Rt, bn, gamma, inv_gm1, F);
    if (PHYS) {
      // the cells beside the face (local indices) and the step to their transverse neighbours
      const int ca = base + step, cb = base + 2 * step, across = xface ? 1 : CY;
      const R ht = xface ? dy : dx, iht = xface ? idy : idx;  // spacing across the face's normal
      R slope_a = R(0), slope_b = R(0);
      if (a.kappa_par != 0.0 || a.kappa_perp != 0.0) {
        // MC-limited transverse temperature slopes of the two cells
#pragma unroll
        for (int side = 0; side < 2; ++side) {
          const int c = side == 0 ? ca : cb;
          const R t0 = temperature<R, NC>(sP, c - across), t1 = temperature<R, NC>(sP, c),
                  t2 = temperature<R, NC>(sP, c + across);
          (side == 0 ? slope_a : slope_b) = limited_slope<2>(M::div(t2 - t1, ht, iht), M::div(t1 - t0, ht, iht));
        }
      }
      R jz_0 = R(0), jz_1 = R(0);
      if (a.eta != 0.0) {
        jz_0 = node_current<R, CY>(sBx, sBy, fi, fj, dx, idx, dy, idy);
        jz_1 = xface ? node_current<R, CY>(sBx, sBy, fi, fj + 1, dx, idx, dy, idy)
                     : node_current<R, CY>(sBx, sBy, fi + 1, fj, dx, idx, dy, idy);
      }
      const int bt_row = xface ? 6 : 5;  // the in-plane tangential field
      nonideal_face_terms(xface, bn, temperature<R, NC>(sP, ca), temperature<R, NC>(sP, cb), slope_a, slope_b,
                          sP[bt_row * NC + ca], sP[bt_row * NC + cb], sP[7 * NC + ca], sP[7 * NC + cb], jz_0, jz_1,
                          xface ? dx : dy, xface ? idx : idy, R(a.eta), R(a.kappa_par), R(a.kappa_perp), F);
    }
    // walls: nothing but the pressure crosses (carafe/mhd.py:874-886)
    bool wall;
    if (xface) {
      const int g = x0 + fi;
      wall = ((P.flags & kWallLo0) && g == 0) || ((P.flags & kWallHi0) && g == nx);
    } else {
      const int g = y0 + fj;
      wall = ((P.flags & kWallLo1) && g == 0) || ((P.flags & kWallHi1) && g == ny);
    }
    if (wall) {
      F[0] = R(0);
      F[2] = R(0);
      F[3] = R(0);
      F[4] = R(0);
      F[6] = R(0);
    }
    R* out = xface ? sFx + fi * FY + (fj + 1) : sFy + (fi + 1) * FY + fj;
#pragma unroll
    for (int c = 0; c < 7; ++c) out[c * NF] = F[c];
  }
  // the global values phase 3 reads (each of the thread's cells and nodes: the stage's
  // input and, in stage 2, the Heun base), loaded before the barrier so that their
  // latency overlaps the wait
  const S dt = S(a.dt[P.instance]);
  // the inverse spacings of the float64 flux differences (mixed precision only)
  const S sidx = kMixed ? S(1) / S(P.dx[0]) : S(0), sidy = kMixed ? S(1) / S(P.dx[1]) : S(0);
  const S* __restrict__ base_state = a.base ? a.base + P.off : nullptr;
  S* __restrict__ dst = a.dst + P.off;
  constexpr int NIT = (TX * TY + kThreads2D - 1) / kThreads2D;  // phase-3 rounds of the threads
  S in_cell[NIT][6], in_node[NIT], base_cell[NIT][6], base_node[NIT];
#pragma unroll
  for (int it = 0; it < NIT; ++it) {
    const int t = threadIdx.x + kThreads2D * it;
    const int ni = t / TY, nj = t % TY;
    const int gx = x0 + ni, gy = y0 + nj;
    const bool node_ok = t < TX * TY && gx < own_nx && gy < own_ny;
    const bool cell_ok = t < TX * TY && gx < nx && gy < ny;
    const int64_t cell = int64_t(gx + 2) * pitch + (gy + 2);
    in_node[it] = node_ok ? src[6 * fs + cell] : S(0);
    base_node[it] = node_ok && base_state ? base_state[6 * fs + cell] : S(0);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      in_cell[it][q] = cell_ok ? src[q * fs + cell] : S(0);
      base_cell[it][q] = cell_ok && base_state ? base_state[q * fs + cell] : S(0);
    }
  }
  __syncthreads();

  // 3. CT-contact E_z at the nodes, A_z and the cells ---------------------------------
#pragma unroll
  for (int it = 0; it < NIT; ++it) {
    const int t = threadIdx.x + kThreads2D * it;
    if (t >= TX * TY) break;
    const int ni = t / TY, nj = t % TY;
    const int gx = x0 + ni, gy = y0 + nj;  // interior node / cell indices
    if (gx < own_nx && gy < own_ny) {
      R ez = ct_node(sFx[5 * NF + ni * FY + nj], sFx[5 * NF + ni * FY + nj + 1], sFx[ni * FY + nj],
                     sFx[ni * FY + nj + 1], sFy[5 * NF + ni * FY + nj], sFy[5 * NF + (ni + 1) * FY + nj],
                     sFy[ni * FY + nj], sFy[(ni + 1) * FY + nj], sE[(ni + 1) * CY + nj + 1],
                     sE[(ni + 2) * CY + nj + 1], sE[(ni + 1) * CY + nj + 2], sE[(ni + 2) * CY + nj + 2]);
      if (PHYS && a.eta != 0.0) ez += R(a.eta) * node_current<R, CY>(sBx, sBy, ni, nj, dx, idx, dy, idy);
      const bool wall = ((P.flags & kWallLo0) && gx == 0) || ((P.flags & kWallHi0) && gx == nx) ||
                        ((P.flags & kWallLo1) && gy == 0) || ((P.flags & kWallHi1) && gy == ny);
      if (wall) ez = R(0);
      const int64_t node = 6 * fs + int64_t(gx + 2) * pitch + (gy + 2);
      S value = in_node[it] - dt * S(ez);
      if (base_state) value = (value + base_node[it]) * S(0.5);
      dst[node] = value;
    }
    if (gx < nx && gy < ny && ni < TX && nj < TY) {
      const int64_t cell = int64_t(gx + 2) * pitch + (gy + 2);
      const int xrow[6] = {0, 1, 2, 3, 4, 6};
      const int yrow[6] = {0, 2, 1, 3, 4, 6};
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        S div;
        if constexpr (kMixed) {
          // float64 flux differences of the float32 fluxes
          div = (S(sFx[xrow[q] * NF + (ni + 1) * FY + nj + 1]) - S(sFx[xrow[q] * NF + ni * FY + nj + 1])) * sidx +
                (S(sFy[yrow[q] * NF + (ni + 1) * FY + nj + 1]) - S(sFy[yrow[q] * NF + (ni + 1) * FY + nj])) * sidy;
        } else {
          div = M::div(sFx[xrow[q] * NF + (ni + 1) * FY + nj + 1] - sFx[xrow[q] * NF + ni * FY + nj + 1], dx, idx) +
                M::div(sFy[yrow[q] * NF + (ni + 1) * FY + nj + 1] - sFy[yrow[q] * NF + (ni + 1) * FY + nj], dy, idy);
        }
        S value = in_cell[it][q] - dt * div;
        if (PHYS) {
          // gravity: rho g on the momentum, m . g on the energy, from the stage's input
          const S gx = S(a.gravity[0]), gy = S(a.gravity[1]);
          if (q == 1) value += dt * (in_cell[it][0] * gx);
          if (q == 2) value += dt * (in_cell[it][0] * gy);
          if (q == 4) value += dt * (in_cell[it][1] * gx + in_cell[it][2] * gy);
        }
        if (base_state) value = (value + base_cell[it][q]) * S(0.5);
        dst[q * fs + cell] = value;
      }
      if (a.bflux && P.bflux >= 0) {
        // boundary-face fluxes of the patch for the flux register, float64
        double* bf = a.bflux + P.bflux;
        if (gx == 0 || gx == nx - 1) {
          const int side = gx == 0 ? 0 : 1;
          const int fi = gx == 0 ? ni : ni + 1;
          for (int q = 0; q < 6; ++q)
            bf[(side * 6 + q) * ny + gy] = double(sFx[xrow[q] * NF + fi * FY + nj + 1]);
        }
        if (gy == 0 || gy == ny - 1) {
          const int side = gy == 0 ? 0 : 1;
          const int fj = gy == 0 ? nj : nj + 1;
          double* by = bf + 2 * 6 * ny;
          for (int q = 0; q < 6; ++q)
            by[(side * 6 + q) * nx + gx] = double(sFy[yrow[q] * NF + (ni + 1) * FY + fj]);
        }
      }
    }
  }
}

template <typename S, typename R, int LIM, bool PHYS, int TX, int TY>
void launch_shape(const StageArgs<S>& args, int ntiles, cudaStream_t stream) {
  constexpr int NC = (TX + 4) * (TY + 4), NF = (TX + 1) * (TY + 1);
  const size_t smem = sizeof(R) * (11 * NC + 14 * NF);
  cudaFuncSetAttribute(stage2d_kernel<S, R, LIM, PHYS, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       int(smem));
  stage2d_kernel<S, R, LIM, PHYS, TX, TY><<<ntiles, kThreads2D, smem, stream>>>(args);
}

// One limiter: the default shape (ideal or non-ideal) or one of the other shapes (ideal).
template <typename S, typename R, int LIM>
int launch_limiter(const StageArgs<S>& args, int ntiles, bool phys, int shape, cudaStream_t stream) {
  using T = Tile2D<S, R>;
  if (shape == 0) {
    if (phys)
      launch_shape<S, R, LIM, true, T::kShape[0][0], T::kShape[0][1]>(args, ntiles, stream);
    else
      launch_shape<S, R, LIM, false, T::kShape[0][0], T::kShape[0][1]>(args, ntiles, stream);
    return kOk;
  }
  if (phys) {
    set_error("stage2d: the non-ideal terms run on the default %dx%d tiles", T::TX, T::TY);
    return kBadArgument;
  }
  switch (shape) {
    case 1: launch_shape<S, R, LIM, false, T::kShape[1][0], T::kShape[1][1]>(args, ntiles, stream); break;
    case 2: launch_shape<S, R, LIM, false, T::kShape[2][0], T::kShape[2][1]>(args, ntiles, stream); break;
    default:
      if constexpr (T::kShapes > 3)
        launch_shape<S, R, LIM, false, T::kShape[3][0], T::kShape[3][1]>(args, ntiles, stream);
      break;
  }
  return kOk;
}

template <typename S, typename R>
int launch_stage2d(const StageArgs<S>& args, int ntiles, int limiter, int tx, int ty, cudaStream_t stream) {
  if (ntiles <= 0) return kOk;
  using T = Tile2D<S, R>;
  int shape = -1;
  for (int i = 0; i < T::kShapes; ++i)
    if (T::kShape[i][0] == tx && T::kShape[i][1] == ty) shape = i;
  if (shape < 0) {
    set_error("stage2d: no %dx%d tile shape for this precision", tx, ty);
    return kBadArgument;
  }
  const bool phys = args.eta != 0.0 || args.kappa_par != 0.0 || args.kappa_perp != 0.0 || args.gravity[0] != 0.0 ||
                    args.gravity[1] != 0.0;
  int status;
  switch (limiter) {
    case 0: status = launch_limiter<S, R, 0>(args, ntiles, phys, shape, stream); break;
    case 1: status = launch_limiter<S, R, 1>(args, ntiles, phys, shape, stream); break;
    case 2: status = launch_limiter<S, R, 2>(args, ntiles, phys, shape, stream); break;
    case 3: status = launch_limiter<S, R, 3>(args, ntiles, phys, shape, stream); break;
    default:
      set_error("limiter code %d is not one of 0..3", limiter);
      return kBadArgument;
  }
  if (status != kOk) return status;
  return check_launch("stage2d");
}

template int launch_stage2d<float, float>(const StageArgs<float>&, int, int, int, int, cudaStream_t);
template int launch_stage2d<double, double>(const StageArgs<double>&, int, int, int, int, cudaStream_t);
template int launch_stage2d<double, float>(const StageArgs<double>&, int, int, int, int, cudaStream_t);

template <typename T>
static int copy_shapes(int* shapes, int max) {
  for (int i = 0; i < T::kShapes && i < max; ++i) {
    shapes[2 * i] = T::kShape[i][0];
    shapes[2 * i + 1] = T::kShape[i][1];
  }
  return T::kShapes;
}

int tile_shapes_2d(int mode, int* shapes, int max) {
  if (mode == kMath32State64) return copy_shapes<Tile2D<double, float>>(shapes, max);
  return mode ? copy_shapes<Tile2D<double>>(shapes, max) : copy_shapes<Tile2D<float>>(shapes, max);
}

void tile_shape_2d(int mode, int* tx, int* ty) {
  if (mode == kMath32State64) {
    *tx = Tile2D<double, float>::TX, *ty = Tile2D<double, float>::TY;
    return;
  }
  *tx = mode ? Tile2D<double>::TX : Tile2D<float>::TX;
  *ty = mode ? Tile2D<double>::TY : Tile2D<float>::TY;
}

}  // namespace wb
