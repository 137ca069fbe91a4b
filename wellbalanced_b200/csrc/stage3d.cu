// Fused 3D stage kernel: one RK stage of the 3D step over a work list of tiles.
//
// A tile is TY x TZ columns (y, z) of a patch, marched along x over `lx` cell planes.
// TY TZ + TY + TZ threads (288 for the default 16 x 16 tile), each with fixed roles per
// plane (two barriers per plane):
//   * one x-face column (j, k) of the L-shaped set the tile needs — its thread keeps
//     the four cell planes of the x-stencil of that column in registers;
//   * one y-face and one z-face of the current plane;
//   * (the first TY TZ) one cell column and the three edges at its lower corner.
// Per plane p the kernel
//   A: loads cell plane p+1 (conserved cells; face fields as the curl of the edge
//      potential, carafe/mhd3d.py:361-386), forms the primitive variables (pressure in
//      float64 for a float32 state) and the cell electric fields, counts bad cells
//      (carafe/mhd3d.py:475-509);
//   B1: MUSCL + HLLD on the y- and z-faces of plane p (loaded one plane earlier), in the
//      same barrier interval as A, so the uneven load rounds of A overlap face work;
//   B2 (after a barrier): the x-face p, whose stencil reaches plane p+1; each face in
//      the cyclic frame of its axis (carafe/mhd3d.py:511-528, mhd_sweep_pyccel.py:254-319);
//   C: CT-contact edge fields (carafe/mhd3d.py:530-559; ct_contact_pyccel.py:36-61):
//      E_x on the x-edges of cell plane p, E_y and E_z on node plane p; updates A there
//      (A -= dt E) and the cells of plane p-1 (U -= dt div F), with the Heun combine in
//      stage 2 (carafe/mhd3d.py:635-671, 726-754).
// Primitive variables, fluxes and edge fields stay on chip; each stage reads the state
// once (plus halo overlap between tiles) and writes it once.
// PHYS adds the reference's resistivity and gravity (carafe/mhd3d.py:561-600, 639-671):
// the face fields are kept for three planes (p-1, p, p+1), so that B2 forms J = curl B
// on the edges around its faces, adds eta (J x B) to the energy flux of its x-, y- and
// z-faces and hands eta J of its column's three edges to C (E += eta J); C adds rho g and
// m . g to the cells.
#include <type_traits>

#include "layout.cuh"
#include "numerics.cuh"
#include "stage.cuh"
#include "wb_internal.cuh"

namespace wb {

// Tile shapes (TY x TZ columns) the kernel is built for, the default first (the only one
// with the non-ideal terms); the others are candidates of the autotuner: a 8 x 16 tile
// needs half the shared memory, so twice the CTAs share an SM, at more halo work per cell;
// a 16 x 32 tile (float32 only: 191 KB) has less halo work per cell and one CTA per SM.
// R is the arithmetic type (shared memory holds R): float32 arithmetic on a float64
// state takes the float32 shapes.
template <typename S, typename R = S>
struct Tile3D {
  static constexpr int TY = 16, TZ = 16;
  static constexpr int kShapes = 2;
  static constexpr int kShape[3][2] = {{16, 16}, {8, 16}, {16, 16}};
};

template <>
struct Tile3D<float, float> {
  static constexpr int TY = 16, TZ = 16;
  static constexpr int kShapes = 3;
  static constexpr int kShape[3][2] = {{16, 16}, {8, 16}, {16, 32}};
};

template <>
struct Tile3D<double, float> {
  static constexpr int TY = 16, TZ = 16;
  static constexpr int kShapes = 3;
  static constexpr int kShape[3][2] = {{16, 16}, {8, 16}, {16, 32}};
};

template <int TY, int TZ>
__host__ __device__ constexpr int threads3d() {
  return TY * TZ + TY + TZ;
}

// Shared memory of a tile shape: primitive variables (2 planes), face fields (2 or 3),
// cell E (4 planes), y/z face fluxes (3 planes), x-face fluxes.
template <typename S, bool PHYS, int TY, int TZ>
__host__ __device__ constexpr size_t smem3d() {
  return sizeof(S) * (2 * 8 * (TY + 4) * (TZ + 4) + (PHYS ? 3 : 2) * 3 * (TY + 4) * (TZ + 4) +
                      4 * 3 * (TY + 1) * (TZ + 1) + 3 * 2 * 7 * (TY + 1) * (TZ + 1) + 3 * (TY + 1) * (TZ + 1));
}

// Hint that a global value will be read soon: fetch its line into L2.
__device__ __forceinline__ void prefetch_l2(const void* ptr) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

template <typename S>
__device__ __forceinline__ bool bad3(S r, S u, S v, S w, S p, S bx, S by, S bz) {
  if (!(r > S(0) && p > S(0))) return true;
  return !(isfinite(r) && isfinite(u) && isfinite(v) && isfinite(w) && isfinite(p) && isfinite(bx) &&
           isfinite(by) && isfinite(bz));
}

// CTAs per SM the shared memory allows (228 KB per SM, 1 KB reserved per CTA), at most 4:
// the register cap of the launch bounds follows from it.
template <typename S, bool PHYS, int TY, int TZ>
struct Occupancy3D {
  static constexpr int kFit = int(233472 / (smem3d<S, PHYS, TY, TZ>() + 1024));
  static constexpr int kBlocks = kFit < 1 ? 1 : (kFit > 4 ? 4 : kFit);
};

// Planes of face fields kept in shared memory: two, or three with the resistive terms.
template <bool PHYS>
__host__ __device__ constexpr int face_slots() {
  return PHYS ? 3 : 2;
}

template <bool PHYS>
__device__ __forceinline__ int face_slot(int plane) {
  return PHYS ? (plane + 6) % 3 : (plane + 4) & 1;  // plane >= -3
}

// The y- and z-face of a B1 thread from the primitive plane P (rows of NR values): the
// y-stencil starts at ry with stride sy, the z-stencil at rz with stride 1; fluxes to
// outy[c G], outz[c G].
template <int LIM, typename R>
__device__ __forceinline__ void yz_faces(const R* P, int NR, int ry, int sy, int rz, R bny, R bnz, R gamma,
                                         R inv_gm1, R* outy, R* outz, int G) {
  constexpr int yrow[7] = {0, 2, 3, 1, 4, 7, 5};
  constexpr int zrow[7] = {0, 3, 1, 2, 4, 5, 6};
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int* rows = side == 0 ? yrow : zrow;
    const int r0 = side == 0 ? ry : rz, st = side == 0 ? sy : 1;
    R a0[7], a1[7], a2[7], a3[7];
#pragma unroll
    for (int c = 0; c < 7; ++c) {
      const R* row = P + rows[c] * NR + r0;
      a0[c] = row[0];
      a1[c] = row[st];
      a2[c] = row[2 * st];
      a3[c] = row[3 * st];
    }
    R L[7], Rt[7], F[7];
    reconstruct<LIM>(a0, a1, a2, a3, L, Rt);
    hlld_flux(L, Rt, side == 0 ? bny : bnz, gamma, inv_gm1, F);
    R* out = side == 0 ? outy : outz;
#pragma unroll
    for (int c = 0; c < 7; ++c) out[c * G] = F[c];
  }
}

// S: the state's type (loads, the conserved and potential updates, the Heun combine);
// R: the arithmetic of the reconstruction, HLLD and CT. With a float64 state and float32
// arithmetic (S = double, R = float) phase A forms the primitive variables and face fields
// in float64 from the float64 state (face fields from float64 differences of the edge
// potential, pressure in float64) and rounds them to float32 for the face work; phase C
// takes float64 flux differences and updates U, A and the Heun combine in float64.
template <typename S, typename R, int LIM, bool PHYS, int TY, int TZ>
__global__ void __launch_bounds__(threads3d<TY, TZ>(), (Occupancy3D<R, PHYS, TY, TZ>::kBlocks))
    stage3d_kernel(const StageArgs<S> a) {
  using M = Math<R>;
  using W = S;  // phase A's arithmetic: the state's type
  using MW = typename std::conditional<std::is_same<S, R>::value, Math<S>, MathRefined>::type;
  constexpr bool kMixed = !std::is_same<S, R>::value;
  constexpr int RZ = TZ + 4, NR = (TY + 4) * (TZ + 4);  // plane region j, k in [-2, T+2)
  constexpr int GZ = TZ + 1, G = (TY + 1) * (TZ + 1);    // face / column grids
  constexpr int NCORE = TY * TZ;
  constexpr int NB = face_slots<PHYS>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sP = reinterpret_cast<R*>(smem_raw);  // [2 slots][8][NR] primitive variables
  R* sBn = sP + 2 * 8 * NR;                 // [NB slots][3][NR] field at each cell's lower faces
  R* sEc = sBn + NB * 3 * NR;               // [4 slots][3][G] cell E_x, E_y, E_z
  R* sYZ = sEc + 4 * 3 * G;                 // [3 slots][2 dirs][7][G] y- and z-face fluxes
  R* sX = sYZ + 3 * 2 * 7 * G;              // [3][G] x-face mass, B_y and B_z fluxes

  const Tile tile = a.tiles[blockIdx.x];
  const PatchDesc P = a.patches[tile.patch];
  const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
  const int64_t p0 = P.pitch0, p1 = P.pitch1, fs = P.fstride;
  const S* __restrict__ src = a.src + P.off;
  const R dx = R(P.dx[0]), dy = R(P.dx[1]), dz = R(P.dx[2]);
  const R idx = M::inv(dx), idy = M::inv(dy), idz = M::inv(dz);
  const R gamma = R(a.gamma), inv_gm1 = R(a.inv_gm1);
  const int x0 = tile.x0, y0 = tile.y0, z0 = tile.z0;
  const int own_nx = nx + ((P.flags & kOwnLast0) ? 1 : 0);
  const int own_ny = ny + ((P.flags & kOwnLast1) ? 1 : 0);
  const int own_nz = nz + ((P.flags & kOwnLast2) ? 1 : 0);
  const int xe = min(x0 + a.lx, nx);      // cell planes [x0, xe)
  const int xn = min(x0 + a.lx, own_nx);  // node planes [x0, xn)
  const int tid = threadIdx.x;

  // roles ------------------------------------------------------------------------------
  int cj, ck;  // x-face column
  int yj, yk;  // y-face (face index yj, cell yk)
  int zj, zk;  // z-face (cell zj, face index zk)
  if (tid < NCORE) {
    cj = yj = zj = tid / TZ;
    ck = yk = zk = tid % TZ;
  } else {
    // the rim: x-columns (-1, k) and (j, -1), y-faces (TY, k) and (j, -1), z-faces
    // (j, TZ) and (-1, k)
    const int u = tid - NCORE;
    if (u < TZ) {
      cj = -1, ck = u;
      yj = TY, yk = u;
    } else {
      cj = u - TZ, ck = -1;
      yj = u - TZ, yk = -1;
    }
    if (u < TY) {
      zj = u, zk = TZ;
    } else {
      zj = -1, zk = u - TY;
    }
  }
  const int col_r = (cj + 2) * RZ + (ck + 2);  // column's position in the plane region
  const int col_g = (cj + 1) * GZ + (ck + 1);  // column's index in the face grid
  const int y_g = yj * GZ + (yk + 1);
  const int z_g = (zj + 1) * GZ + zk;

  // the x-stencil of the column: plane p-1 in registers (x-frame rows; planes p and p+1
  // are read from the primitive slots), and the limited x-slope of plane p-1
  R qm[7];
  R slope[7];
#pragma unroll
  for (int c = 0; c < 7; ++c) qm[c] = R(1);
#pragma unroll
  for (int c = 0; c < 7; ++c) slope[c] = R(0);
  R fprev[5] = {R(0), R(0), R(0), R(0), R(0)};
  R fnow[5] = {R(0), R(0), R(0), R(0), R(0)};
  R ejx = R(0), ejy = R(0), ejz = R(0);  // eta J on the column's edges (PHYS)
  // PHYS: the field at the lower `axis`-face of cell (plane, j, k) of the tile, and the
  // current J_c = d_a B_b - d_b B_a ((c, a, b) cyclic) on the c-edge whose lower corner
  // is that cell (carafe/mhd3d.py:579-590); planes p-1 .. p+1 are held during B2
  auto face = [&](int plane, int axis, int j, int k) -> R {
    return sBn[(face_slot<PHYS>(plane) * 3 + axis) * NR + (j + 2) * RZ + (k + 2)];
  };
  auto jx_at = [&](int plane, int j, int k) -> R {
    return M::div(face(plane, 2, j, k) - face(plane, 2, j - 1, k), dy, idy) -
           M::div(face(plane, 1, j, k) - face(plane, 1, j, k - 1), dz, idz);
  };
  auto jy_at = [&](int plane, int j, int k) -> R {
    return M::div(face(plane, 0, j, k) - face(plane, 0, j, k - 1), dz, idz) -
           M::div(face(plane, 2, j, k) - face(plane - 1, 2, j, k), dx, idx);
  };
  auto jz_at = [&](int plane, int j, int k) -> R {
    return M::div(face(plane, 1, j, k) - face(plane - 1, 1, j, k), dx, idx) -
           M::div(face(plane, 0, j, k) - face(plane, 0, j - 1, k), dy, idy);
  };
  const S dt = S(a.dt[P.instance]);
  const S* __restrict__ base_state = a.base ? a.base + P.off : nullptr;
  S* __restrict__ dst = a.dst + P.off;
  unsigned bad = 0;
  // phase A's spacings and mean field in the state's type
  const W wdx = W(P.dx[0]), wdy = W(P.dx[1]), wdz = W(P.dx[2]);
  const W widx = MW::inv(wdx), widy = MW::inv(wdy), widz = MW::inv(wdz);
  const W b0x = W(a.b0[0]), b0y = W(a.b0[1]), b0z = W(a.b0[2]);
  // the inverse spacings of the float64 flux differences (mixed precision only)
  const S sidx = kMixed ? S(1) / S(P.dx[0]) : S(0), sidy = kMixed ? S(1) / S(P.dx[1]) : S(0),
          sidz = kMixed ? S(1) / S(P.dx[2]) : S(0);

  for (int p = x0 - 3; p <= xe; ++p) {
    // prefetch into L2 what phase C of the next plane reads from global memory: the
    // cells and edges of its column in the input state (read two planes ago, usually
    // still cached) and in the Heun base state (not read before)
    if (tid < NCORE && p + 1 >= x0 && p < xe) {
      const int gj = y0 + cj, gk = z0 + ck;
      const int64_t o = int64_t(p + kHalo) * p0 + int64_t(gj + kHalo) * p1 + (gk + kHalo);
      if (base_state) {
#pragma unroll
        for (int f = 0; f < 8; ++f) prefetch_l2(base_state + f * fs + o);
      }
    }
    // A: load cell plane c = p + 1 ------------------------------------------------------
    {
      const int c = p + 1;
      const int slot = (c + 4) & 1;
      const int slot4 = (c + 8) & 3;
      R* P8 = sP + slot * 8 * NR;
      R* B3 = sBn + (PHYS ? face_slot<PHYS>(c) : slot) * 3 * NR;
      R* E3 = sEc + slot4 * 3 * G;
      const int I = c + kHalo;
      for (int r = tid; r < NR; r += threads3d<TY, TZ>()) {
        const int j = r / RZ - 2, k = r % RZ - 2;
        const int J = y0 + j + kHalo, K = z0 + k + kHalo;
        W rho = W(1), m0 = W(0), m1 = W(0), m2 = W(0), e = W(1);
        W bxl = W(0), bxh = W(0), byl = W(0), byh = W(0), bzl = W(0), bzh = W(0);
        const bool valid = J < ny + 4 && K < nz + 4 && I < nx + 4;
        if (valid) {
          const int64_t o = int64_t(I) * p0 + int64_t(J) * p1 + K;
          rho = src[o];
          m0 = src[fs + o];
          m1 = src[2 * fs + o];
          m2 = src[3 * fs + o];
          e = src[4 * fs + o];
          const S* Ax = src + 5 * fs;
          const S* Ay = src + 6 * fs;
          const S* Az = src + 7 * fs;
          // x-faces at nodes I and I+1: dA_z/dy - dA_y/dz + B0x
          bxl = MW::div(Az[o + p1] - Az[o], wdy, widy) - MW::div(Ay[o + 1] - Ay[o], wdz, widz) + b0x;
          bxh = MW::div(Az[o + p0 + p1] - Az[o + p0], wdy, widy) - MW::div(Ay[o + p0 + 1] - Ay[o + p0], wdz, widz) + b0x;
          // y-faces at nodes J and J+1: dA_x/dz - dA_z/dx + B0y
          byl = MW::div(Ax[o + 1] - Ax[o], wdz, widz) - MW::div(Az[o + p0] - Az[o], wdx, widx) + b0y;
          byh = MW::div(Ax[o + p1 + 1] - Ax[o + p1], wdz, widz) - MW::div(Az[o + p1 + p0] - Az[o + p1], wdx, widx) + b0y;
          // z-faces at nodes K and K+1: dA_y/dx - dA_x/dy + B0z
          bzl = MW::div(Ay[o + p0] - Ay[o], wdx, widx) - MW::div(Ax[o + p1] - Ax[o], wdy, widy) + b0z;
          bzh = MW::div(Ay[o + p0 + 1] - Ay[o + 1], wdx, widx) - MW::div(Ax[o + p1 + 1] - Ax[o + 1], wdy, widy) + b0z;
        }
        const W irho = MW::inv(rho);
        const W u = MW::div(m0, rho, irho), v = MW::div(m1, rho, irho), w = MW::div(m2, rho, irho);
        const W bx = W(0.5) * (bxl + bxh), by = W(0.5) * (byl + byh), bz = W(0.5) * (bzl + bzh);
        W pr = recover_pressure<W>(rho, m0, m1, m2, e, bx, by, bz, u, v, w, a.gamma);
        if (!valid) pr = W(1);
        P8[r] = R(rho);
        P8[NR + r] = R(u);
        P8[2 * NR + r] = R(v);
        P8[3 * NR + r] = R(w);
        P8[4 * NR + r] = R(pr);
        P8[5 * NR + r] = R(bx);
        P8[6 * NR + r] = R(by);
        P8[7 * NR + r] = R(bz);
        B3[r] = R(bxl);
        B3[NR + r] = R(byl);
        B3[2 * NR + r] = R(bzl);
        if (j >= -1 && j < TY && k >= -1 && k < TZ) {
          const int g = (j + 1) * GZ + (k + 1);
          E3[g] = R(by * w - bz * v);          // E_x
          E3[G + g] = R(bz * u - bx * w);      // E_y
          E3[2 * G + g] = R(bx * v - by * u);  // E_z
        }
        if (valid && c >= x0 && c < xe && j >= 0 && j < TY && k >= 0 && k < TZ && y0 + j < ny &&
            z0 + k < nz && bad3(rho, u, v, w, pr, bx, by, bz))
          ++bad;
      }
    }
    // B1: y- and z-faces of plane p (plane p was loaded before the previous barrier), in
    // the same barrier interval as the loads of plane p + 1 ------------------------------
    {
      const int slot = (p + 4) & 1, slot3 = (p + 6) % 3;
      const R* Pp = sP + slot * 8 * NR;
      const R* Bp = sBn + (PHYS ? face_slot<PHYS>(p) : slot) * 3 * NR;
      const bool need_yz = p >= x0 - 1 && (p < xe || xn > xe);
      if (need_yz) {
        R* Y7 = sYZ + (slot3 * 2 + 0) * 7 * G;
        R* Z7 = sYZ + (slot3 * 2 + 1) * 7 * G;
        // the y-face between cells (yj-1, yk) and (yj, yk), frame (y, z, x), and the z-face
        // between cells (zj, zk-1) and (zj, zk), frame (z, x, y)
        yz_faces<LIM>(Pp, NR, (yj - 2 + 2) * RZ + (yk + 2), RZ, (zj + 2) * RZ + (zk - 2 + 2),
                      Bp[NR + (yj + 2) * RZ + (yk + 2)], Bp[2 * NR + (zj + 2) * RZ + (zk + 2)], gamma, inv_gm1,
                      Y7 + y_g, Z7 + z_g, G);
      }
    }
    __syncthreads();

    // B2: x-face of plane p (needs plane p + 1 for its stencil) --------------------------
    {
      const R* Pc = sP + ((p + 4) & 1) * 8 * NR;      // plane p
      const R* Pn = sP + ((p + 1 + 4) & 1) * 8 * NR;  // plane p + 1
      constexpr int xrow[7] = {0, 1, 2, 3, 4, 6, 7};
      // plane x0 - 3 (the first p) was never loaded: its column reads as 1 like qm, and the
      // slopes formed before plane x0 - 1 are never used
      const bool loaded = p >= x0 - 2;
      R q1[7], q2[7];
#pragma unroll
      for (int cc = 0; cc < 7; ++cc) {
        q1[cc] = loaded ? Pc[xrow[cc] * NR + col_r] : R(1);
        q2[cc] = Pn[xrow[cc] * NR + col_r];
      }
      // the slope of plane p, kept for face p + 1: each cell's x-slope is formed once
      R now[7];
      if constexpr (std::is_same<R, float>::value) {
        float back[7], fwd[7];
#pragma unroll
        for (int cc = 0; cc < 7; ++cc) {
          back[cc] = q1[cc] - qm[cc];
          fwd[cc] = q2[cc] - q1[cc];
        }
        limited_slopes7<LIM>(back, fwd, now);
      } else {
#pragma unroll
        for (int cc = 0; cc < 7; ++cc) now[cc] = limited_slope<LIM>(q1[cc] - qm[cc], q2[cc] - q1[cc]);
      }
      const R* Bp = sBn + (PHYS ? face_slot<PHYS>(p) : ((p + 4) & 1)) * 3 * NR;
      if (p >= x0) {
        R L[7], Rt[7], F[7];
        reconstruct_sloped(qm, q1, slope, now, L, Rt);
        hlld_flux(L, Rt, Bp[col_r], gamma, inv_gm1, F);
        if (PHYS && a.eta != 0.0 && tid < NCORE) {
          // eta (J_y B_z - J_z B_y) on the x-face: J of its two y- and two z-edges, B of
          // the four y- and z-faces around it (carafe/mhd3d.py:590-600)
          const R eta = R(a.eta);
          const R jb = R(0.5) * (jy_at(p, cj, ck) + jy_at(p, cj, ck + 1));
          const R jc = R(0.5) * (jz_at(p, cj, ck) + jz_at(p, cj + 1, ck));
          const R bc = R(0.5) * (R(0.5) * (face(p - 1, 2, cj, ck) + face(p, 2, cj, ck)) +
                                 R(0.5) * (face(p - 1, 2, cj, ck + 1) + face(p, 2, cj, ck + 1)));
          const R bb = R(0.5) * (R(0.5) * (face(p - 1, 1, cj, ck) + face(p, 1, cj, ck)) +
                                 R(0.5) * (face(p - 1, 1, cj + 1, ck) + face(p, 1, cj + 1, ck)));
          F[4] += eta * (jb * bc - jc * bb);
        }
        // x-face walls: none in 3D (the reference's MHD3D has periodic and outflow faces)
        sX[col_g] = F[0];
        sX[G + col_g] = F[5];
        sX[2 * G + col_g] = F[6];
#pragma unroll
        for (int cc = 0; cc < 5; ++cc) fnow[cc] = F[cc];
      }
#pragma unroll
      for (int cc = 0; cc < 7; ++cc) {
        slope[cc] = now[cc];
        qm[cc] = q1[cc];
      }
      if (PHYS && a.eta != 0.0 && p >= x0) {
        const R eta = R(a.eta);
        if (p < xe) {
          // eta (J_z B_x - J_x B_z) on the y-face (cell p, node yj, cell yk) and
          // eta (J_x B_y - J_y B_x) on the z-face (cell p, cell zj, node zk), added to the
          // energy fluxes this thread formed in B1 (read by C one plane later)
          const int sl3 = (p + 6) % 3;
          if (yk >= 0) {
            const R jb = R(0.5) * (jz_at(p, yj, yk) + jz_at(p + 1, yj, yk));
            const R jc = R(0.5) * (jx_at(p, yj, yk) + jx_at(p, yj, yk + 1));
            const R bc = R(0.5) * (R(0.5) * (face(p, 0, yj - 1, yk) + face(p, 0, yj, yk)) +
                                   R(0.5) * (face(p + 1, 0, yj - 1, yk) + face(p + 1, 0, yj, yk)));
            const R bb = R(0.5) * (R(0.5) * (face(p, 2, yj - 1, yk) + face(p, 2, yj, yk)) +
                                   R(0.5) * (face(p, 2, yj - 1, yk + 1) + face(p, 2, yj, yk + 1)));
            sYZ[(sl3 * 2 + 0) * 7 * G + 4 * G + y_g] += eta * (jb * bc - jc * bb);
          }
          if (zj >= 0) {
            const R jb = R(0.5) * (jx_at(p, zj, zk) + jx_at(p, zj + 1, zk));
            const R jc = R(0.5) * (jy_at(p, zj, zk) + jy_at(p + 1, zj, zk));
            const R bc = R(0.5) * (R(0.5) * (face(p, 1, zj, zk - 1) + face(p, 1, zj, zk)) +
                                   R(0.5) * (face(p, 1, zj + 1, zk - 1) + face(p, 1, zj + 1, zk)));
            const R bb = R(0.5) * (R(0.5) * (face(p, 0, zj, zk - 1) + face(p, 0, zj, zk)) +
                                   R(0.5) * (face(p + 1, 0, zj, zk - 1) + face(p + 1, 0, zj, zk)));
            sYZ[(sl3 * 2 + 1) * 7 * G + 4 * G + z_g] += eta * (jb * bc - jc * bb);
          }
        }
        if (tid < NCORE) {
          // eta J on the column's x-edge (cell plane p) and y- and z-edges (node plane p)
          ejx = eta * jx_at(p, cj, ck);
          ejy = eta * jy_at(p, cj, ck);
          ejz = eta * jz_at(p, cj, ck);
        }
      }
    }
    // the global values phase C reads (the conserved values of the column's cell in plane
    // p - 1 and the potentials of its edges in plane p, with their Heun base values in
    // stage 2), loaded before the barrier so that their latency overlaps the wait
    const int gj_c = y0 + cj, gk_c = z0 + ck;
    const bool core_c = p >= x0 && tid < NCORE;
    const bool do_cell = core_c && p - 1 >= x0 && p - 1 < xe && gj_c < ny && gk_c < nz;
    const bool do_ex = core_c && p < xe && gj_c < own_ny && gk_c < own_nz;
    const bool do_ey = core_c && p < xn && gj_c < ny && gk_c < own_nz;
    const bool do_ez = core_c && p < xn && gj_c < own_ny && gk_c < nz;
    const int64_t o_cell = int64_t(p - 1 + kHalo) * p0 + int64_t(gj_c + kHalo) * p1 + (gk_c + kHalo);
    const int64_t o_edge = o_cell + p0;
    S cv[5], cb[5], ev[3], eb[3];
#pragma unroll
    for (int qf = 0; qf < 5; ++qf) {
      cv[qf] = do_cell ? src[qf * fs + o_cell] : S(0);
      cb[qf] = do_cell && base_state ? base_state[qf * fs + o_cell] : S(0);
    }
    {
      const bool ok[3] = {do_ex, do_ey, do_ez};
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        ev[e] = ok[e] ? src[(5 + e) * fs + o_edge] : S(0);
        eb[e] = ok[e] && base_state ? base_state[(5 + e) * fs + o_edge] : S(0);
      }
    }
    __syncthreads();

    // C: edges and cells ----------------------------------------------------------------
    if (core_c) {
      const int j = cj, k = ck;
      const int gj = gj_c, gk = gk_c;
      const int sc = (p + 6) % 3, sp = (p + 5) % 3;  // flux slots of planes p and p-1
      const R* Yc = sYZ + (sc * 2 + 0) * 7 * G;
      const R* Zc = sYZ + (sc * 2 + 1) * 7 * G;
      const R* Yp = sYZ + (sp * 2 + 0) * 7 * G;
      const R* Zp = sYZ + (sp * 2 + 1) * 7 * G;
      const R* Ec = sEc + ((p + 8) & 3) * 3 * G;
      const R* Ep = sEc + ((p + 7) & 3) * 3 * G;
      auto yi = [&](int fj, int kk) { return fj * GZ + (kk + 1); };
      auto zi = [&](int jj, int fk) { return (jj + 1) * GZ + fk; };
      auto gi = [&](int jj, int kk) { return (jj + 1) * GZ + (kk + 1); };
      // cells of plane p-1
      if (do_cell) {
        const int64_t o = o_cell;
        const int yrow[5] = {0, 3, 1, 2, 4};  // y-sweep rows of (rho, m_x, m_y, m_z, E)
        const int zrow[5] = {0, 2, 3, 1, 4};  // z-sweep rows
#pragma unroll
        for (int qf = 0; qf < 5; ++qf) {
          S div;
          if constexpr (kMixed) {
            // float64 flux differences of the float32 fluxes
            div = (S(fnow[qf]) - S(fprev[qf])) * sidx +
                  (S(Yp[yrow[qf] * G + yi(j + 1, k)]) - S(Yp[yrow[qf] * G + yi(j, k)])) * sidy +
                  (S(Zp[zrow[qf] * G + zi(j, k + 1)]) - S(Zp[zrow[qf] * G + zi(j, k)])) * sidz;
          } else {
            div = M::div(fnow[qf] - fprev[qf], dx, idx) +
                  M::div(Yp[yrow[qf] * G + yi(j + 1, k)] - Yp[yrow[qf] * G + yi(j, k)], dy, idy) +
                  M::div(Zp[zrow[qf] * G + zi(j, k + 1)] - Zp[zrow[qf] * G + zi(j, k)], dz, idz);
          }
          S value = cv[qf] - dt * div;
          if (PHYS) {
            // gravity: rho g on the momentum, m . g on the energy, from the stage's input
            const S g0 = S(a.gravity[0]), g1 = S(a.gravity[1]), g2 = S(a.gravity[2]);
            if (qf >= 1 && qf <= 3) value += dt * (S(a.gravity[qf - 1]) * cv[0]);
            if (qf == 4) value += dt * (cv[1] * g0 + cv[2] * g1 + cv[3] * g2);
          }
          if (base_state) value = (value + cb[qf]) * S(0.5);
          dst[qf * fs + o] = value;
        }
      }
      // E_x on the x-edges of cell plane p: (a, b) = (y, z)
      if (do_ex) {
        R ex = ct_node(Yc[5 * G + yi(j, k - 1)], Yc[5 * G + yi(j, k)], Yc[yi(j, k - 1)], Yc[yi(j, k)],
                             Zc[6 * G + zi(j - 1, k)], Zc[6 * G + zi(j, k)], Zc[zi(j - 1, k)], Zc[zi(j, k)],
                             Ec[gi(j - 1, k - 1)], Ec[gi(j, k - 1)], Ec[gi(j - 1, k)], Ec[gi(j, k)]);
        if (PHYS) ex += ejx;
        const int64_t o = 5 * fs + o_edge;
        S value = ev[0] - dt * S(ex);
        if (base_state) value = (value + eb[0]) * S(0.5);
        dst[o] = value;
      }
      {
        // E_y on the y-edges of node plane p: (a, b) = (z, x)
        if (do_ey) {
          R ey = ct_node(Zp[5 * G + zi(j, k)], Zc[5 * G + zi(j, k)], Zp[zi(j, k)], Zc[zi(j, k)],
                               sX[2 * G + gi(j, k - 1)], sX[2 * G + gi(j, k)], sX[gi(j, k - 1)], sX[gi(j, k)],
                               Ep[G + gi(j, k - 1)], Ep[G + gi(j, k)], Ec[G + gi(j, k - 1)], Ec[G + gi(j, k)]);
          if (PHYS) ey += ejy;
          const int64_t o = 6 * fs + o_edge;
          S value = ev[1] - dt * S(ey);
          if (base_state) value = (value + eb[1]) * S(0.5);
          dst[o] = value;
        }
        // E_z on the z-edges of node plane p: (a, b) = (x, y)
        if (do_ez) {
          R ez = ct_node(sX[G + gi(j - 1, k)], sX[G + gi(j, k)], sX[gi(j - 1, k)], sX[gi(j, k)],
                               Yp[6 * G + yi(j, k)], Yc[6 * G + yi(j, k)], Yp[yi(j, k)], Yc[yi(j, k)],
                               Ep[2 * G + gi(j - 1, k)], Ec[2 * G + gi(j - 1, k)], Ep[2 * G + gi(j, k)],
                               Ec[2 * G + gi(j, k)]);
          if (PHYS) ez += ejz;
          const int64_t o = 7 * fs + o_edge;
          S value = ev[2] - dt * S(ez);
          if (base_state) value = (value + eb[2]) * S(0.5);
          dst[o] = value;
        }
      }
#pragma unroll
      for (int cc = 0; cc < 5; ++cc) fprev[cc] = fnow[cc];
    }
    // no barrier here: phase A of the next plane writes only the primitive, face-field and
    // cell-E slots of plane p + 2 (the E ring has 4 slots, phase C reads those of p and
    // p - 1), and phase B of the next plane, which overwrites the faces read above, comes
    // after the next barrier
  }
  if (bad) atomicAdd(a.bad, (unsigned long long)bad);
}

template <typename S, typename R, int LIM, bool PHYS, int TY, int TZ>
void launch_shape3d(const StageArgs<S>& args, int ntiles, cudaStream_t stream) {
  constexpr size_t smem = smem3d<R, PHYS, TY, TZ>();
  cudaFuncSetAttribute(stage3d_kernel<S, R, LIM, PHYS, TY, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       int(smem));
  stage3d_kernel<S, R, LIM, PHYS, TY, TZ><<<ntiles, threads3d<TY, TZ>(), smem, stream>>>(args);
}

template <typename S, typename R, int LIM>
int launch_limiter3d(const StageArgs<S>& args, int ntiles, bool phys, int shape, cudaStream_t stream) {
  using T = Tile3D<S, R>;
  if (shape == 0) {
    if (phys)
      launch_shape3d<S, R, LIM, true, T::kShape[0][0], T::kShape[0][1]>(args, ntiles, stream);
    else
      launch_shape3d<S, R, LIM, false, T::kShape[0][0], T::kShape[0][1]>(args, ntiles, stream);
    return kOk;
  }
  if (phys) {
    set_error("stage3d: the non-ideal terms run on the default %dx%d tiles", T::TY, T::TZ);
    return kBadArgument;
  }
  if (shape == 1)
    launch_shape3d<S, R, LIM, false, T::kShape[1][0], T::kShape[1][1]>(args, ntiles, stream);
  else if constexpr (T::kShapes > 2)
    launch_shape3d<S, R, LIM, false, T::kShape[2][0], T::kShape[2][1]>(args, ntiles, stream);
  return kOk;
}

template <typename S, typename R>
int launch_stage3d(const StageArgs<S>& args, int ntiles, int limiter, int ty, int tz, cudaStream_t stream) {
  if (ntiles <= 0) return kOk;
  if (args.lx <= 0) {
    set_error("stage3d: lx must be positive");
    return kBadArgument;
  }
  using T = Tile3D<S, R>;
  int shape = -1;
  for (int i = 0; i < T::kShapes; ++i)
    if (T::kShape[i][0] == ty && T::kShape[i][1] == tz) shape = i;
  if (shape < 0) {
    set_error("stage3d: no %dx%d tile shape", ty, tz);
    return kBadArgument;
  }
  const bool phys = args.eta != 0.0 || args.gravity[0] != 0.0 || args.gravity[1] != 0.0 || args.gravity[2] != 0.0;
  int status;
  switch (limiter) {
    case 0: status = launch_limiter3d<S, R, 0>(args, ntiles, phys, shape, stream); break;
    case 1: status = launch_limiter3d<S, R, 1>(args, ntiles, phys, shape, stream); break;
    case 2: status = launch_limiter3d<S, R, 2>(args, ntiles, phys, shape, stream); break;
    case 3: status = launch_limiter3d<S, R, 3>(args, ntiles, phys, shape, stream); break;
    default:
      set_error("limiter code %d is not one of 0..3", limiter);
      return kBadArgument;
  }
  if (status != kOk) return status;
  return check_launch("stage3d");
}

template int launch_stage3d<float, float>(const StageArgs<float>&, int, int, int, int, cudaStream_t);
template int launch_stage3d<double, double>(const StageArgs<double>&, int, int, int, int, cudaStream_t);
template int launch_stage3d<double, float>(const StageArgs<double>&, int, int, int, int, cudaStream_t);

template <typename T>
static int copy_shapes3d(int* shapes, int max) {
  for (int i = 0; i < T::kShapes && i < max; ++i) {
    shapes[2 * i] = T::kShape[i][0];
    shapes[2 * i + 1] = T::kShape[i][1];
  }
  return T::kShapes;
}

int tile_shapes_3d(int mode, int* shapes, int max) {
  if (mode == kMath32State64) return copy_shapes3d<Tile3D<double, float>>(shapes, max);
  return mode ? copy_shapes3d<Tile3D<double>>(shapes, max) : copy_shapes3d<Tile3D<float>>(shapes, max);
}

void tile_shape_3d(int mode, int* ty, int* tz) {
  if (mode == kMath32State64) {
    *ty = Tile3D<double, float>::TY, *tz = Tile3D<double, float>::TZ;
    return;
  }
  *ty = mode ? Tile3D<double>::TY : Tile3D<float>::TY;
  *tz = mode ? Tile3D<double>::TZ : Tile3D<float>::TZ;
}

}  // namespace wb
