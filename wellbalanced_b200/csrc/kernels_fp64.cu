// Per-kernel float64 CUDA versions of the reference's six MHD block kernels.
//
// Same arguments, shapes and out-parameter convention as carafe/kernels/<name>
// (Pyccel / NumPy versions), one thread per output element, C-contiguous float64
// device arrays. These are the drop-in for `carafe.kernels.<name>.kernel` and the
// building blocks of the plain float64 GPU step (the reference's dataflow, each
// intermediate in HBM).
#include "numerics.cuh"
#include "wb_internal.cuh"

namespace wb {

// mhd_primitive (carafe/kernels/mhd_primitive/mhd_primitive_pyccel.py:23-87)
__global__ void primitive_fp64_kernel(const double* __restrict__ rho, const double* __restrict__ mx,
                                      const double* __restrict__ my, const double* __restrict__ mz,
                                      const double* __restrict__ energy,
                                      const double* __restrict__ bz, const double* __restrict__ az,
                                      int X, int Y, double dx, double dy, double b0x, double b0y,
                                      double gamma, double* __restrict__ prim,
                                      double* __restrict__ bxf, double* __restrict__ byf,
                                      double* __restrict__ ecc, unsigned long long* bad) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nodes = int64_t(X + 1) * (Y + 1);
  if (t >= nodes) return;
  const int i = int(t / (Y + 1));
  const int j = int(t % (Y + 1));
  const int A = Y + 1;  // row pitch of az
  if (j < Y) bxf[int64_t(i) * Y + j] = (az[int64_t(i) * A + j + 1] - az[int64_t(i) * A + j]) / dy + b0x;
  if (i < X) byf[int64_t(i) * (Y + 1) + j] = -(az[int64_t(i + 1) * A + j] - az[int64_t(i) * A + j]) / dx + b0y;
  if (i >= X || j >= Y) return;
  const int64_t c = int64_t(i) * Y + j;
  const double bx_lo = (az[int64_t(i) * A + j + 1] - az[int64_t(i) * A + j]) / dy + b0x;
  const double bx_hi = (az[int64_t(i + 1) * A + j + 1] - az[int64_t(i + 1) * A + j]) / dy + b0x;
  const double by_lo = -(az[int64_t(i + 1) * A + j] - az[int64_t(i) * A + j]) / dx + b0y;
  const double by_hi = -(az[int64_t(i + 1) * A + j + 1] - az[int64_t(i) * A + j + 1]) / dx + b0y;
  const double r = rho[c];
  const double u = mx[c] / r;
  const double v = my[c] / r;
  const double w = mz[c] / r;
  const double bx = 0.5 * (bx_lo + bx_hi);
  const double by = 0.5 * (by_lo + by_hi);
  const double b = bz[c];
  const double p =
      (gamma - 1.0) * (energy[c] - 0.5 * r * (u * u + v * v + w * w) - 0.5 * (bx * bx + by * by + b * b));
  const int64_t plane = int64_t(X) * Y;
  prim[c] = r;
  prim[plane + c] = u;
  prim[2 * plane + c] = v;
  prim[3 * plane + c] = w;
  prim[4 * plane + c] = p;
  prim[5 * plane + c] = bx;
  prim[6 * plane + c] = by;
  prim[7 * plane + c] = b;
  ecc[c] = bx * v - by * u;
  const double big = 1.7976931348623157e308;
  bool ok = r > 0.0 && p > 0.0;
  if (ok) {
    ok = fabs(r) <= big && fabs(u) <= big && fabs(v) <= big && fabs(w) <= big && fabs(p) <= big &&
         fabs(bx) <= big && fabs(by) <= big && fabs(b) <= big;
  }
  if (!ok) atomicAdd(bad, 1ull);
}

// mhd_sweep (mhd_sweep_pyccel.py:254-319): one thread per face of one line.
template <int LIM>
__global__ void sweep_fp64_kernel(const double* __restrict__ prim, const double* __restrict__ bn,
                                  int axis, double gamma, int X, int Y, double* __restrict__ flux) {
  const int n = axis == 0 ? X : Y;
  const int lines = axis == 0 ? Y : X;
  const int faces = n - 3;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= int64_t(faces) * lines) return;
  // axis 0: consecutive threads take consecutive lines (coalesced along y)
  int k, line;
  if (axis == 0) {
    k = int(t / lines);
    line = int(t % lines);
  } else {
    line = int(t / faces);
    k = int(t % faces);
  }
  const int comp[7] = {0, 1 + axis, 2 - axis, 3, 4, 6 - axis, 7};
  const int64_t plane = int64_t(X) * Y;
  double q[4][7];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int64_t cell = axis == 0 ? int64_t(k + s) * Y + line : int64_t(line) * Y + (k + s);
#pragma unroll
    for (int c = 0; c < 7; ++c) q[s][c] = prim[comp[c] * plane + cell];
  }
  double L[7], Rt[7], F[7];
  reconstruct<LIM>(q[0], q[1], q[2], q[3], L, Rt);
  const double normal = axis == 0 ? bn[int64_t(k + 2) * Y + line] : bn[int64_t(line) * (Y + 1) + k + 2];
  hlld_flux(L, Rt, normal, gamma, 1.0 / (gamma - 1.0), F);
  const int64_t fplane = int64_t(faces) * lines;
  const int64_t out = axis == 0 ? int64_t(k) * Y + line : int64_t(line) * faces + k;
#pragma unroll
  for (int c = 0; c < 7; ++c) flux[c * fplane + out] = F[c];
}

// ct_contact (ct_contact_pyccel.py:26-61): one thread per node.
__global__ void ct_fp64_kernel(const double* __restrict__ fx_by, const double* __restrict__ gy_bx,
                               const double* __restrict__ fx_rho, const double* __restrict__ gy_rho,
                               const double* __restrict__ ecc, int X, int Y, int na, int nb,
                               double* __restrict__ ez) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= int64_t(na) * nb) return;
  const int a = int(t / nb), b = int(t % nb);
  const int i = a + 2, j = b + 2;
  const int FY = Y - 3;  // row pitch of gy_*
  ez[t] = ct_node(fx_by[int64_t(i - 2) * Y + j - 1], fx_by[int64_t(i - 2) * Y + j],
                  fx_rho[int64_t(i - 2) * Y + j - 1], fx_rho[int64_t(i - 2) * Y + j],
                  gy_bx[int64_t(i - 1) * FY + j - 2], gy_bx[int64_t(i) * FY + j - 2],
                  gy_rho[int64_t(i - 1) * FY + j - 2], gy_rho[int64_t(i) * FY + j - 2],
                  ecc[int64_t(i - 1) * Y + j - 1], ecc[int64_t(i) * Y + j - 1],
                  ecc[int64_t(i - 1) * Y + j], ecc[int64_t(i) * Y + j]);
}

// ct_contact over a stack of planes (the per-plane calls of carafe/mhd3d.py:544-557 in one
// launch): plane q of every array starts at q times its plane size.
__global__ void ct_fp64_planes_kernel(const double* __restrict__ fx_by, const double* __restrict__ gy_bx,
                                      const double* __restrict__ fx_rho, const double* __restrict__ gy_rho,
                                      const double* __restrict__ ecc, int X, int Y, int na, int nb,
                                      double* __restrict__ ez) {
  const int64_t q = blockIdx.y;
  const int64_t fxs = int64_t(X - 3) * Y, gys = int64_t(X) * (Y - 3), es = int64_t(X) * Y, os = int64_t(na) * nb;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= os) return;
  const int a = int(t / nb), b = int(t % nb);
  const int i = a + 2, j = b + 2;
  const int FY = Y - 3;
  const double* fb = fx_by + q * fxs;
  const double* fr = fx_rho + q * fxs;
  const double* gb = gy_bx + q * gys;
  const double* gr = gy_rho + q * gys;
  const double* ec = ecc + q * es;
  ez[q * os + t] = ct_node(fb[int64_t(i - 2) * Y + j - 1], fb[int64_t(i - 2) * Y + j], fr[int64_t(i - 2) * Y + j - 1],
                           fr[int64_t(i - 2) * Y + j], gb[int64_t(i - 1) * FY + j - 2], gb[int64_t(i) * FY + j - 2],
                           gr[int64_t(i - 1) * FY + j - 2], gr[int64_t(i) * FY + j - 2], ec[int64_t(i - 1) * Y + j - 1],
                           ec[int64_t(i) * Y + j - 1], ec[int64_t(i - 1) * Y + j], ec[int64_t(i) * Y + j]);
}

// mhd_rate (mhd_rate_pyccel.py:30-83): max rate and min density over the block's own
// cells, reduced with order-preserving integer keys (exact, order independent).
__global__ void rate_fp64_kernel(const double* __restrict__ rho, const double* __restrict__ mx,
                                 const double* __restrict__ my, const double* __restrict__ mz,
                                 const double* __restrict__ energy, const double* __restrict__ bz,
                                 const double* __restrict__ az, int X, int Y, int halo, double dx,
                                 double dy, double b0x, double b0y, double gamma,
                                 unsigned long long* keys) {
  const int nx = X - 2 * halo, ny = Y - 2 * halo;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double rate = 0.0;
  double smallest = __longlong_as_double(0x7ff0000000000000ll);  // +inf
  if (t < int64_t(nx) * ny) {
    const int i = int(t / ny) + halo, j = int(t % ny) + halo;
    const int A = Y + 1;
    const int64_t c = int64_t(i) * Y + j;
    const double r = rho[c];
    const double u = mx[c] / r, v = my[c] / r, w = mz[c] / r;
    const double bx = 0.5 * ((az[int64_t(i) * A + j + 1] - az[int64_t(i) * A + j]) / dy + b0x +
                             ((az[int64_t(i + 1) * A + j + 1] - az[int64_t(i + 1) * A + j]) / dy + b0x));
    const double by = 0.5 * (-(az[int64_t(i + 1) * A + j] - az[int64_t(i) * A + j]) / dx + b0y +
                             (-(az[int64_t(i + 1) * A + j + 1] - az[int64_t(i) * A + j + 1]) / dx + b0y));
    const double bzc = bz[c];
    const double p =
        (gamma - 1.0) * (energy[c] - 0.5 * r * (u * u + v * v + w * w) - 0.5 * (bx * bx + by * by + bzc * bzc));
    rate = (fabs(u) + fast_speed(r, p, bx, by, bzc, gamma)) / dx +
           (fabs(v) + fast_speed(r, p, by, bx, bzc, gamma)) / dy;
    smallest = r;
  }
  block_reduce_keys(rate, smallest, keys);
}

__global__ void rate_finish_kernel(unsigned long long* keys, double* out) {
  out[0] = key_to_double(keys[0]);
  out[1] = key_to_double(keys[1]);
}

// mhd_resistive (mhd_resistive_pyccel.py:21-67)
__device__ __forceinline__ double jz_node(const double* bxf, const double* byf, int X, int Y,
                                          int i, int j, double dx, double dy) {
  // J_z at node (i, j) of the haloed block, i, j >= 1
  return (byf[int64_t(i) * (Y + 1) + j] - byf[int64_t(i - 1) * (Y + 1) + j]) / dx -
         (bxf[int64_t(i) * Y + j] - bxf[int64_t(i) * Y + j - 1]) / dy;
}

__global__ void resistive_fp64_kernel(const double* __restrict__ prim, const double* __restrict__ bxf,
                                      const double* __restrict__ byf, int X, int Y, double dx,
                                      double dy, double eta, double* __restrict__ fx,
                                      double* __restrict__ fy, double* __restrict__ ez) {
  const int h = 2, nx = X - 2 * h, ny = Y - 2 * h;
  const int64_t plane = int64_t(X) * Y;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t n_xf = int64_t(nx + 1) * ny, n_yf = int64_t(nx) * (ny + 1), n_node = int64_t(nx + 1) * (ny + 1);
  if (t < n_xf) {
    const int f = int(t / ny), b = int(t % ny);
    const int i = h + f, j = h + b;
    const double jy = -(prim[7 * plane + int64_t(i) * Y + j] - prim[7 * plane + int64_t(i - 1) * Y + j]) / dx;
    const double bz_x = 0.5 * (prim[7 * plane + int64_t(i) * Y + j] + prim[7 * plane + int64_t(i - 1) * Y + j]);
    const double by_x = 0.5 * (prim[6 * plane + int64_t(i) * Y + j] + prim[6 * plane + int64_t(i - 1) * Y + j]);
    const double jz_x = 0.5 * (jz_node(bxf, byf, X, Y, i, j, dx, dy) + jz_node(bxf, byf, X, Y, i, j + 1, dx, dy));
    const int64_t fp = int64_t(X - 3) * Y;
    const int64_t o = int64_t(f) * Y + j;
    fx[6 * fp + o] = fx[6 * fp + o] + eta * jy;
    fx[4 * fp + o] = fx[4 * fp + o] + eta * (jy * bz_x - jz_x * by_x);
    return;
  }
  const int64_t t2 = t - n_xf;
  if (t2 < n_yf) {
    const int a = int(t2 / (ny + 1)), f = int(t2 % (ny + 1));
    const int i = h + a, j = h + f;
    const double jx = (prim[7 * plane + int64_t(i) * Y + j] - prim[7 * plane + int64_t(i) * Y + j - 1]) / dy;
    const double bz_y = 0.5 * (prim[7 * plane + int64_t(i) * Y + j] + prim[7 * plane + int64_t(i) * Y + j - 1]);
    const double bx_y = 0.5 * (prim[5 * plane + int64_t(i) * Y + j] + prim[5 * plane + int64_t(i) * Y + j - 1]);
    const double jz_y = 0.5 * (jz_node(bxf, byf, X, Y, i, j, dx, dy) + jz_node(bxf, byf, X, Y, i + 1, j, dx, dy));
    const int FY = Y - 3;
    const int64_t fp = int64_t(X) * FY;
    const int64_t o = int64_t(i) * FY + f;
    fy[6 * fp + o] = fy[6 * fp + o] + -eta * jx;
    fy[4 * fp + o] = fy[4 * fp + o] + eta * (jz_y * bx_y - jx * bz_y);
    return;
  }
  const int64_t t3 = t2 - n_yf;
  if (t3 < n_node) {
    const int a = int(t3 / (ny + 1)), b = int(t3 % (ny + 1));
    const int64_t o = int64_t(a) * (Y - 3) + b;
    ez[o] = ez[o] + eta * jz_node(bxf, byf, X, Y, h + a, h + b, dx, dy);
  }
}

// mhd_conductive (mhd_conductive_pyccel.py:38-100)
__device__ __forceinline__ double mc2(double a, double b) { return limited_slope<2>(a, b); }

__device__ __forceinline__ double temperature(const double* prim, int64_t plane, int Y, int i, int j) {
  return prim[4 * plane + int64_t(i) * Y + j] / prim[int64_t(i) * Y + j];
}

__global__ void conductive_fp64_kernel(const double* __restrict__ prim, const double* __restrict__ bxf,
                                       const double* __restrict__ byf, int X, int Y, double dx,
                                       double dy, double kpar, double kperp,
                                       double* __restrict__ fx, double* __restrict__ fy) {
  const int64_t plane = int64_t(X) * Y;
  const double tiny = 2.2250738585072014e-308;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t n_xf = int64_t(X - 3) * Y, n_yf = int64_t(X) * (Y - 3);
  if (t < n_xf) {
    const int k = int(t / Y), j = int(t % Y);
    // the limited gradient along y of cells k + 1 and k + 2 (zero in the first/last row)
    double across[2];
    for (int s = 0; s < 2; ++s) {
      const int i = k + 1 + s;
      across[s] = 0.0;
      if (j >= 1 && j <= Y - 2) {
        const double tc = temperature(prim, plane, Y, i, j);
        across[s] = mc2((temperature(prim, plane, Y, i, j + 1) - tc) / dy,
                        (tc - temperature(prim, plane, Y, i, j - 1)) / dy);
      }
    }
    const double bn = bxf[int64_t(k + 2) * Y + j];
    const double bt = 0.5 * (prim[6 * plane + int64_t(k + 1) * Y + j] + prim[6 * plane + int64_t(k + 2) * Y + j]);
    const double bzf = 0.5 * (prim[7 * plane + int64_t(k + 1) * Y + j] + prim[7 * plane + int64_t(k + 2) * Y + j]);
    const double magnitude = fmax(sqrt(bn * bn + bt * bt + bzf * bzf), tiny);
    const double b_n = bn / magnitude, b_t = bt / magnitude;
    const double normal = (temperature(prim, plane, Y, k + 2, j) - temperature(prim, plane, Y, k + 1, j)) / dx;
    const double transverse = mc2(across[0], across[1]);
    const int64_t o = 4 * int64_t(X - 3) * Y + int64_t(k) * Y + j;
    fx[o] = fx[o] - (kpar * b_n * (b_n * normal + b_t * transverse) + kperp * normal);
    return;
  }
  const int64_t t2 = t - n_xf;
  if (t2 < n_yf) {
    const int i = int(t2 / (Y - 3)), k = int(t2 % (Y - 3));
    double across[2];
    for (int s = 0; s < 2; ++s) {
      const int j = k + 1 + s;
      across[s] = 0.0;
      if (i >= 1 && i <= X - 2) {
        const double tc = temperature(prim, plane, Y, i, j);
        across[s] = mc2((temperature(prim, plane, Y, i + 1, j) - tc) / dx,
                        (tc - temperature(prim, plane, Y, i - 1, j)) / dx);
      }
    }
    const double bn = byf[int64_t(i) * (Y + 1) + k + 2];
    const double bt = 0.5 * (prim[5 * plane + int64_t(i) * Y + k + 1] + prim[5 * plane + int64_t(i) * Y + k + 2]);
    const double bzf = 0.5 * (prim[7 * plane + int64_t(i) * Y + k + 1] + prim[7 * plane + int64_t(i) * Y + k + 2]);
    const double magnitude = fmax(sqrt(bn * bn + bt * bt + bzf * bzf), tiny);
    const double b_n = bn / magnitude, b_t = bt / magnitude;
    const double normal = (temperature(prim, plane, Y, i, k + 2) - temperature(prim, plane, Y, i, k + 1)) / dy;
    const double transverse = mc2(across[0], across[1]);
    const int64_t o = 4 * int64_t(X) * (Y - 3) + int64_t(i) * (Y - 3) + k;
    fy[o] = fy[o] - (kpar * b_n * (b_n * normal + b_t * transverse) + kperp * normal);
  }
}

// ---------------------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------------------
static inline unsigned blocks_for(int64_t n, int threads) { return unsigned((n + threads - 1) / threads); }

int launch_primitive_fp64(const double* rho, const double* mx, const double* my, const double* mz,
                          const double* energy, const double* bz, const double* az, int X, int Y,
                          double dx, double dy, double b0x, double b0y, double gamma, double* prim,
                          double* bxf, double* byf, double* ecc, unsigned long long* bad,
                          cudaStream_t stream) {
  const int64_t n = int64_t(X + 1) * (Y + 1);
  if (n > 0)
    primitive_fp64_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(rho, mx, my, mz, energy, bz, az, X, Y, dx, dy,
                                                                 b0x, b0y, gamma, prim, bxf, byf, ecc, bad);
  return check_launch("mhd_primitive");
}

int launch_sweep_fp64(const double* prim, const double* bn, int axis, int limiter, double gamma, int X,
                      int Y, double* flux, cudaStream_t stream) {
  const int n = axis == 0 ? X : Y;
  const int lines = axis == 0 ? Y : X;
  const int64_t total = int64_t(n - 3) * lines;
  if (total <= 0) return 0;
  const unsigned grid = blocks_for(total, 128);
  switch (limiter) {
    case 0: sweep_fp64_kernel<0><<<grid, 128, 0, stream>>>(prim, bn, axis, gamma, X, Y, flux); break;
    case 1: sweep_fp64_kernel<1><<<grid, 128, 0, stream>>>(prim, bn, axis, gamma, X, Y, flux); break;
    case 2: sweep_fp64_kernel<2><<<grid, 128, 0, stream>>>(prim, bn, axis, gamma, X, Y, flux); break;
    default: sweep_fp64_kernel<3><<<grid, 128, 0, stream>>>(prim, bn, axis, gamma, X, Y, flux); break;
  }
  return check_launch("mhd_sweep");
}

int launch_ct_fp64(const double* fx_by, const double* gy_bx, const double* fx_rho, const double* gy_rho,
                   const double* ecc, int X, int Y, int na, int nb, double* ez, cudaStream_t stream) {
  const int64_t n = int64_t(na) * nb;
  if (n > 0) ct_fp64_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(fx_by, gy_bx, fx_rho, gy_rho, ecc, X, Y, na, nb, ez);
  return check_launch("ct_contact");
}

int launch_ct_planes_fp64(const double* fx_by, const double* gy_bx, const double* fx_rho, const double* gy_rho,
                          const double* ecc, int X, int Y, int na, int nb, int planes, double* ez,
                          cudaStream_t stream) {
  const int64_t n = int64_t(na) * nb;
  if (n > 0 && planes > 0)
    ct_fp64_planes_kernel<<<dim3(blocks_for(n, 256), planes), 256, 0, stream>>>(fx_by, gy_bx, fx_rho, gy_rho, ecc, X, Y,
                                                                                na, nb, ez);
  return check_launch("ct_contact_planes");
}

int launch_rate_fp64(const double* rho, const double* mx, const double* my, const double* mz,
                     const double* energy, const double* bz, const double* az, int X, int Y, int halo,
                     double dx, double dy, double b0x, double b0y, double gamma, double* out,
                     cudaStream_t stream) {
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(out);
  init_keys_kernel<<<1, 1, 0, stream>>>(keys);
  const int64_t n = int64_t(X - 2 * halo) * (Y - 2 * halo);
  if (n > 0)
    rate_fp64_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(rho, mx, my, mz, energy, bz, az, X, Y, halo, dx, dy,
                                                            b0x, b0y, gamma, keys);
  rate_finish_kernel<<<1, 1, 0, stream>>>(keys, out);
  return check_launch("mhd_rate");
}

int launch_resistive_fp64(const double* prim, const double* bxf, const double* byf, int X, int Y, double dx,
                          double dy, double eta, double* fx, double* fy, double* ez, cudaStream_t stream) {
  const int nx = X - 4, ny = Y - 4;
  const int64_t n = int64_t(nx + 1) * ny + int64_t(nx) * (ny + 1) + int64_t(nx + 1) * (ny + 1);
  if (n > 0) resistive_fp64_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(prim, bxf, byf, X, Y, dx, dy, eta, fx, fy, ez);
  return check_launch("mhd_resistive");
}

int launch_conductive_fp64(const double* prim, const double* bxf, const double* byf, int X, int Y,
                           double dx, double dy, double kpar, double kperp, double* fx, double* fy,
                           cudaStream_t stream) {
  const int64_t n = int64_t(X - 3) * Y + int64_t(X) * (Y - 3);
  if (n > 0) conductive_fp64_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(prim, bxf, byf, X, Y, dx, dy, kpar, kperp, fx, fy);
  return check_launch("mhd_conductive");
}

}  // namespace wb
