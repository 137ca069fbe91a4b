// Device numerics of the ideal-MHD face flux: PLM limiters, fast speed, HLLD.
//
// Restated from the reference kernels (carafe/kernels/mhd_sweep/mhd_sweep_pyccel.py):
//   limited_slope  :25-48    fast_speed :51-61
//   side_state     :64-98    star_state :101-145    hlld_face :148-251
// The HLLD here first picks the side of the contact the face lies on (S_M >= 0: the
// left fan, else the right) and evaluates the star / double-star state of that side
// only; the other side contributes its star density, tangential velocity and field,
// which the double-star average needs. The five-region selection and every formula
// are those of the reference (Miyoshi & Kusano 2005), so the float64 instantiation
// agrees with it to rounding.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace wb {

// Relative size below which the HLLD star denominator counts as zero (carafe/mhd.py:138).
constexpr double kDegenerate = 1.0e-12;

// abs / min / max as single instructions (abs modifiers, FMNMX / DMNMX); the operands
// here are never NaN in a valid state, where these agree with the reference's min / max.
__device__ __forceinline__ float rabs(float x) { return fabsf(x); }
__device__ __forceinline__ double rabs(double x) { return fabs(x); }
__device__ __forceinline__ float rmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double rmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float rmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double rmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float rcopysign(float m, float s) { return copysignf(m, s); }
__device__ __forceinline__ double rcopysign(double m, double s) { return copysign(m, s); }

// Arithmetic policy of the two precisions.
//  float64 keeps every division and square root of the reference, in its order, so the
//  float64 kernels agree with the reference to rounding (`div(a, b, inv_b)` is a / b and
//  the precomputed reciprocal is dead code the compiler drops).
//  float32 shares one approximate reciprocal (MUFU rcp, ~1 ulp) per denominator and takes
//  square roots as x * rsqrt(x): ~14 special-function ops per HLLD face instead of ~40
//  correctly rounded division / square-root sequences.
template <typename R>
struct Math;

template <>
struct Math<double> {
  static __device__ __forceinline__ double inv(double b) { return 1.0 / b; }
  static __device__ __forceinline__ double div(double a, double b, double) { return a / b; }
  static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
  // 1 / sqrt(x) as the reference writes it: 1 / sqrt(x)
  static __device__ __forceinline__ double over_sqrt(double a, double sq) { return a / sq; }
};

template <>
struct Math<float> {
  static __device__ __forceinline__ float inv(float b) { return __fdividef(1.0f, b); }
  static __device__ __forceinline__ float div(float a, float, float inv_b) { return a * inv_b; }
  static __device__ __forceinline__ float sqrt(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }
  static __device__ __forceinline__ float over_sqrt(float a, float sq) { return a * __fdividef(1.0f, sq); }
};

// float64 arithmetic seeded from the float32 special-function units: the reciprocal and
// the reciprocal square root of the float32 value refined by one Newton step in float64
// (relative error ~1e-13). Used by the float32 kernels where float32 is not enough (the
// near-degenerate HLLD star states below).
struct MathRefined {
  static __device__ __forceinline__ double inv(double b) {
    const double r = double(__fdividef(1.0f, float(b)));
    return r * (2.0 - b * r);
  }
  static __device__ __forceinline__ double div(double a, double, double inv_b) { return a * inv_b; }
  static __device__ __forceinline__ double sqrt(double x) {
    if (!(x > 0.0)) return 0.0;
    const double r0 = double(rsqrtf(float(x)));
    return x * (r0 * (1.5 - 0.5 * x * r0 * r0));
  }
  static __device__ __forceinline__ double over_sqrt(double a, double sq) { return a * inv(sq); }
};

__device__ __forceinline__ float rsqrt_(float x) { return Math<float>::sqrt(x); }
__device__ __forceinline__ double rsqrt_(double x) { return sqrt(x); }

// Limited PLM slope of a cell from its backward (a) and forward (b) differences.
// LIM: 0 minmod, 1 van Leer, 2 monotonized central, 3 none (central). Branch-free: where
// a * b > 0 the slope is, for MC, sign(a) min(|a + b| / 2, 2 min(|a|, |b|)) — the
// reference's central / bound / size selection (mhd_sweep_pyccel.py:25-48) when a and b
// share a sign — and zero elsewhere.
template <int LIM, typename R>
__device__ __forceinline__ R limited_slope(R a, R b) {
  if (LIM == 3) return R(0.5) * (a + b);
  const bool same = a * b > R(0);
  R slope;
  if (LIM == 0) {
    slope = rabs(a) < rabs(b) ? a : b;
  } else if (LIM == 1) {
    const R product = a * b;
    slope = Math<R>::div(R(2) * product, a + b, Math<R>::inv(a + b));
  } else {
    const R central = R(0.5) * (a + b);
    const R bound = R(2) * rmin(rabs(a), rabs(b));
    slope = rcopysign(rmin(rabs(central), bound), a);
  }
  return same ? slope : R(0);
}

// Runtime-limiter form (used by the per-kernel path, which takes the code as data).
template <typename R>
__device__ __forceinline__ R limited_slope_rt(R a, R b, int limiter) {
  switch (limiter) {
    case 0: return limited_slope<0>(a, b);
    case 1: return limited_slope<1>(a, b);
    case 2: return limited_slope<2>(a, b);
    default: return limited_slope<3>(a, b);
  }
}

// Fast magnetosonic speed along the normal; the discriminant is clipped at zero.
template <typename R, typename M = Math<R>>
__device__ __forceinline__ R fast_speed(R rho, R p, R bn, R bt1, R bt2, R gamma) {
  const R inv_rho = M::inv(rho);
  const R a2 = M::div(gamma * p, rho, inv_rho);
  const R b2 = M::div(bn * bn + bt1 * bt1 + bt2 * bt2, rho, inv_rho);
  const R disc = (a2 + b2) * (a2 + b2) - M::div(R(4) * a2 * bn * bn, rho, inv_rho);
  const R root = disc > R(0) ? M::sqrt(disc) : R(0);
  return M::sqrt(R(0.5) * (a2 + b2 + root));
}

// Conserved state U and physical flux F along the normal of a normal-frame primitive
// state w = (rho, vn, vt1, vt2, p, bt1, bt2); returns the total pressure.
template <typename R>
__device__ __forceinline__ R side_state(const R (&w)[7], R bn, R inv_gm1, R (&u)[7], R (&f)[7]) {
  const R rho = w[0], vn = w[1], vt1 = w[2], vt2 = w[3], p = w[4], bt1 = w[5], bt2 = w[6];
  const R magnetic = R(0.5) * (bn * bn + bt1 * bt1 + bt2 * bt2);
  const R energy = p * inv_gm1 + R(0.5) * rho * (vn * vn + vt1 * vt1 + vt2 * vt2) + magnetic;
  const R pt = p + magnetic;
  const R vb = vn * bn + vt1 * bt1 + vt2 * bt2;
  u[0] = rho;
  u[1] = rho * vn;
  u[2] = rho * vt1;
  u[3] = rho * vt2;
  u[4] = energy;
  u[5] = bt1;
  u[6] = bt2;
  f[0] = rho * vn;
  f[1] = rho * vn * vn + pt - bn * bn;
  f[2] = rho * vn * vt1 - bn * bt1;
  f[3] = rho * vn * vt2 - bn * bt2;
  f[4] = (energy + pt) * vn - bn * vb;
  f[5] = bt1 * vn - bn * vt1;
  f[6] = bt2 * vn - bn * vt2;
  return pt;
}

// Star tangential velocity and field of one side (star_state without the energy); `den`
// returns the star denominator d (s - s_M) - B_n^2.
template <typename R, typename M = Math<R>>
__device__ __forceinline__ void star_tangential(const R (&w)[7], R bn, R s, R d, R pt, R sm,
                                                R& rho_s, R& vt1, R& vt2, R& bt1, R& bt2, R& den) {
  const R vn = w[1];
  rho_s = M::div(d, s - sm, M::inv(s - sm));
  den = d * (s - sm) - bn * bn;
  vt1 = w[2];
  vt2 = w[3];
  bt1 = w[5];
  bt2 = w[6];
  const bool regular = rabs(den) >= R(kDegenerate) * (pt + bn * bn);
  const R inv_den = M::inv(den);
  const R scale = d * (s - vn) - bn * bn;
  const R v1 = w[2] - M::div(bn * w[5] * (sm - vn), den, inv_den);
  const R v2 = w[3] - M::div(bn * w[6] * (sm - vn), den, inv_den);
  const R b1 = M::div(w[5] * scale, den, inv_den);
  const R b2 = M::div(w[6] * scale, den, inv_den);
  vt1 = regular ? v1 : vt1;
  vt2 = regular ? v2 : vt2;
  bt1 = regular ? b1 : bt1;
  bt2 = regular ? b2 : bt2;
}

// The wave speeds, S_M, p_T* and both sides' star density, tangential velocity and field.
template <typename R>
struct HlldFront {
  R sl, sr, ptl, ptr, dl, dr, sm, pts;
  R rsl, vtl1, vtl2, btl1, btl2, den_l;
  R rsr, vtr1, vtr2, btr1, btr2, den_r;
};

template <typename R, typename M>
__device__ __forceinline__ void hlld_front(const R (&L)[7], const R (&Rt)[7], R bn, R gamma, HlldFront<R>& o) {
  const R rl = L[0], vl = L[1], rr = Rt[0], vr = Rt[1];
  const R cf = rmax(fast_speed<R, M>(rl, L[4], bn, L[5], L[6], gamma),
                    fast_speed<R, M>(rr, Rt[4], bn, Rt[5], Rt[6], gamma));
  o.sl = rmin(vl, vr) - cf;
  o.sr = rmax(vl, vr) + cf;
  const R bn2 = bn * bn;
  o.ptl = L[4] + R(0.5) * (bn2 + L[5] * L[5] + L[6] * L[6]);
  o.ptr = Rt[4] + R(0.5) * (bn2 + Rt[5] * Rt[5] + Rt[6] * Rt[6]);
  o.dl = (o.sl - vl) * rl;
  o.dr = (o.sr - vr) * rr;
  const R inv_dd = M::inv(o.dr - o.dl);
  o.sm = M::div(o.dr * vr - o.dl * vl - o.ptr + o.ptl, o.dr - o.dl, inv_dd);
  o.pts = M::div(o.dr * o.ptl - o.dl * o.ptr + o.dl * o.dr * (vr - vl), o.dr - o.dl, inv_dd);
  star_tangential<R, M>(L, bn, o.sl, o.dl, o.ptl, o.sm, o.rsl, o.vtl1, o.vtl2, o.btl1, o.btl2, o.den_l);
  star_tangential<R, M>(Rt, bn, o.sr, o.dr, o.ptr, o.sm, o.rsr, o.vtr1, o.vtr2, o.btr1, o.btr2, o.den_r);
}

// Relative size of the star denominator below which a float32 evaluation is redone in
// float64: the float32 fast speeds carry relative errors ~1e-7, so d (s - s_M) - B_n^2 has
// absolute errors up to ~1e-6 (p_T + B_n^2) where it cancels (Alfven speed close to the
// fast speed, small tangential field); above 1e-3 the float32 value is good to ~0.1%.
constexpr float kNearDegenerate32 = 1.0e-3f;

template <typename R>
__device__ __forceinline__ void hlld_front_checked(const R (&L)[7], const R (&Rt)[7], R bn, R gamma,
                                                   HlldFront<R>& o) {
  hlld_front<R, Math<R>>(L, Rt, bn, gamma, o);
}

// HLLD flux through a face between normal-frame states L and Rt with normal field bn
// (float64; the float32 faces take the lane code of numerics_lanes.cuh). Straight-line code: the star / double-star flux of the side of the contact the face
// lies on is always formed and the supersonic and star-only cases are selected at the
// end (no divergent branches). Where a face is supersonic (S_L >= 0 or S_R < 0) the
// contact lies on the same side as the upwind state, so one side state serves both.
template <typename R>
__device__ __forceinline__ void hlld_flux(const R (&L)[7], const R (&Rt)[7], R bn, R gamma,
                                          R inv_gm1, R (&F)[7]) {
  using M = Math<R>;
  HlldFront<R> fr;
  hlld_front_checked<R>(L, Rt, bn, gamma, fr);
  const R sl = fr.sl, sr = fr.sr, ptl = fr.ptl, ptr = fr.ptr, sm = fr.sm, pts = fr.pts;
  const R rsl = fr.rsl, vtl1 = fr.vtl1, vtl2 = fr.vtl2, btl1 = fr.btl1, btl2 = fr.btl2;
  const R rsr = fr.rsr, vtr1 = fr.vtr1, vtr2 = fr.vtr2, btr1 = fr.btr1, btr2 = fr.btr2;
  const R sql = M::sqrt(rsl);
  const R sqr = M::sqrt(rsr);
  const R sign = bn > R(0) ? R(1) : (bn < R(0) ? R(-1) : R(0));
  const R inv_sum = M::inv(sql + sqr);
  const R vt2_1 = M::div(sql * vtl1 + sqr * vtr1 + (btr1 - btl1) * sign, sql + sqr, inv_sum);
  const R vt2_2 = M::div(sql * vtl2 + sqr * vtr2 + (btr2 - btl2) * sign, sql + sqr, inv_sum);
  const R bt2_1 = M::div(sql * btr1 + sqr * btl1 + sql * sqr * (vtr1 - vtl1) * sign, sql + sqr, inv_sum);
  const R bt2_2 = M::div(sql * btr2 + sqr * btl2 + sql * sqr * (vtr2 - vtl2) * sign, sql + sqr, inv_sum);
  const R vb2 = sm * bn + vt2_1 * bt2_1 + vt2_2 * bt2_2;
  // the side of the contact the face lies on (also the upwind side when supersonic)
  const bool left = sm >= R(0);
  R w[7];
#pragma unroll
  for (int c = 0; c < 7; ++c) w[c] = left ? L[c] : Rt[c];
  const R s = left ? sl : sr;
  const R pt = left ? ptl : ptr;
  const R rho_s = left ? rsl : rsr;
  const R vt1 = left ? vtl1 : vtr1;
  const R vt2 = left ? vtl2 : vtr2;
  const R bt1 = left ? btl1 : btr1;
  const R bt2 = left ? btl2 : btr2;
  const R sq = left ? sql : sqr;
  const R ss = left ? sm - M::over_sqrt(rabs(bn), sql) : sm + M::over_sqrt(rabs(bn), sqr);
  const bool twice = left ? !(ss >= R(0)) : ss >= R(0);
  const bool supersonic = sl >= R(0) || sr < R(0);
  const R sense = left ? R(-1) : R(1);
  R u[7], f[7];
  side_state(w, bn, inv_gm1, u, f);
  const R vn = w[1];
  const R vb = vn * bn + w[2] * w[5] + w[3] * w[6];
  const R vb_s = sm * bn + vt1 * bt1 + vt2 * bt2;
  const R energy_s = M::div((s - vn) * u[4] - pt * vn + pts * sm + bn * (vb - vb_s), s - sm, M::inv(s - sm));
  R us[7], ud[7];
  us[0] = rho_s;
  us[1] = rho_s * sm;
  us[2] = rho_s * vt1;
  us[3] = rho_s * vt2;
  us[4] = energy_s;
  us[5] = bt1;
  us[6] = bt2;
  ud[0] = rho_s;
  ud[1] = rho_s * sm;
  ud[2] = rho_s * vt2_1;
  ud[3] = rho_s * vt2_2;
  ud[4] = energy_s + sense * sq * (vb_s - vb2) * sign;
  ud[5] = bt2_1;
  ud[6] = bt2_2;
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    const R star = f[c] + s * (us[c] - u[c]);
    const R twice_star = star + ss * (ud[c] - us[c]);
    F[c] = supersonic ? f[c] : (twice ? twice_star : star);
  }
}

// Left/right states of a face from four consecutive cells q0..q3 (the face lies between
// q1 and q2), with the first-order fallback where a reconstructed density or pressure
// is not positive (mhd_sweep_pyccel.py:286-307).
template <int LIM, typename R>
__device__ __forceinline__ void reconstruct(const R (&q0)[7], const R (&q1)[7], const R (&q2)[7],
                                            const R (&q3)[7], R (&L)[7], R (&Rt)[7]) {
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    const R s1 = limited_slope<LIM>(q1[c] - q0[c], q2[c] - q1[c]);
    const R s2 = limited_slope<LIM>(q2[c] - q1[c], q3[c] - q2[c]);
    L[c] = q1[c] + R(0.5) * s1;
    Rt[c] = q2[c] - R(0.5) * s2;
  }
  const bool first_order = L[0] <= R(0) || L[4] <= R(0) || Rt[0] <= R(0) || Rt[4] <= R(0);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    L[c] = first_order ? q1[c] : L[c];
    Rt[c] = first_order ? q2[c] : Rt[c];
  }
}

// The same left/right states from the two cells beside the face (q1 | q2) and their
// limited slopes, already formed (s1 of q1, s2 of q2) -- for a caller that keeps each
// cell's slope for both of its faces.
template <typename R>
__device__ __forceinline__ void reconstruct_sloped(const R (&q1)[7], const R (&q2)[7], const R (&s1)[7],
                                                   const R (&s2)[7], R (&L)[7], R (&Rt)[7]) {
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    L[c] = q1[c] + R(0.5) * s1[c];
    Rt[c] = q2[c] - R(0.5) * s2[c];
  }
  const bool first_order = L[0] <= R(0) || L[4] <= R(0) || Rt[0] <= R(0) || Rt[4] <= R(0);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    L[c] = first_order ? q1[c] : L[c];
    Rt[c] = first_order ? q2[c] : Rt[c];
  }
}

// The resistive and Braginskii-conductive terms of a 2D face, added to its HLLD flux F
// (frame of the face; rows 4 energy, 6 B_z), in the reference's order: the heat flux
// q = kpar b_n (b_n dT/dn + b_t dT/dt) + kperp dT/dn is subtracted
// (carafe/kernels/mhd_conductive/mhd_conductive_pyccel.py:38-100), then eta J terms are
// added (mhd_resistive_pyccel.py:21-67). Inputs: the cells a | b beside the face, their
// temperatures and MC-limited transverse temperature slopes, their in-plane tangential
// field (B_y on an x-face, B_x on a y-face) and B_z, the normal face field bn, J_z at the
// face's two end nodes (lower first), the spacing along the normal.
template <typename S>
__device__ __forceinline__ void nonideal_face_terms(bool xface, S bn, S t_a, S t_b, S slope_a, S slope_b, S bt_a,
                                                    S bt_b, S bz_a, S bz_b, S jz_0, S jz_1, S hn, S ihn, S eta,
                                                    S kpar, S kperp, S (&F)[7]) {
  using M = Math<S>;
  if (kpar != S(0) || kperp != S(0)) {
    const S transverse = limited_slope<2>(slope_a, slope_b);
    const S bt = S(0.5) * (bt_a + bt_b);
    const S bzf = S(0.5) * (bz_a + bz_b);
    const S tiny = sizeof(S) == 4 ? S(1.17549435e-38f) : S(2.2250738585072014e-308);
    const S magnitude = rmax(rsqrt_(bn * bn + bt * bt + bzf * bzf), tiny);
    const S im = M::inv(magnitude);
    const S b_n = M::div(bn, magnitude, im), b_t = M::div(bt, magnitude, im);
    const S normal = M::div(t_b - t_a, hn, ihn);
    F[4] -= kpar * b_n * (b_n * normal + b_t * transverse) + kperp * normal;
  }
  if (eta != S(0)) {
    const S bz_f = S(0.5) * (bz_a + bz_b);
    const S bt_f = S(0.5) * (bt_a + bt_b);
    const S jz_f = S(0.5) * (jz_0 + jz_1);
    if (xface) {
      const S jy = -M::div(bz_b - bz_a, hn, ihn);  // J_y = -dB_z/dx
      F[6] += eta * jy;
      F[4] += eta * (jy * bz_f - jz_f * bt_f);
    } else {
      const S jx = M::div(bz_b - bz_a, hn, ihn);  // J_x = dB_z/dy
      F[6] += -eta * jx;
      F[4] += eta * (jz_f * bt_f - jx * bz_f);
    }
  }
}

// CT-contact upwind pick (ct_contact_pyccel.py:17-24).
template <typename R>
__device__ __forceinline__ R upwind(R mass, R positive, R negative) {
  const R mean = R(0.5) * (positive + negative);
  return mass > R(0) ? positive : (mass < R(0) ? negative : mean);
}

// E at a node from its four faces and four cells (ct_contact_pyccel.py:36-61):
//   fb_lo/fb_hi: a-face fluxes of B_b (= -E) below/above the node along b, with their
//                mass fluxes m_lo/m_hi;
//   gb_lo/gb_hi: b-face fluxes of B_a (= +E) left/right of the node along a, with
//                mass fluxes n_lo/n_hi;
//   e00, e10, e01, e11: the cell E of the cells (a-1,b-1), (a,b-1), (a-1,b), (a,b).
template <typename R>
__device__ __forceinline__ R ct_node(R fb_lo, R fb_hi, R m_lo, R m_hi, R gb_lo, R gb_hi, R n_lo,
                                     R n_hi, R e00, R e10, R e01, R e11) {
  const R dl2 = upwind(m_lo, gb_lo - e00, gb_hi - e10);
  const R dr2 = upwind(m_hi, gb_lo - e01, gb_hi - e11);
  const R dl1 = upwind(n_lo, -fb_lo - e00, -fb_hi - e01);
  const R dr1 = upwind(n_hi, -fb_lo - e10, -fb_hi - e11);
  return R(0.25) * (gb_hi + gb_lo - fb_hi - fb_lo + dl1 + dr1 + dl2 + dr2);
}

// Pressure recovery p = (gamma - 1)(E - rho u^2 / 2 - B^2 / 2) of a cell.
template <typename S>
__device__ __forceinline__ S recover_pressure(S r, S m0, S m1, S m2, S e, S bx, S by, S bz, S u, S v,
                                              S w, double gamma);

// float64: the reference's expression (mhd_primitive_pyccel.py:60-64)
template <>
__device__ __forceinline__ double recover_pressure<double>(double r, double, double, double, double e,
                                                           double bx, double by, double bz, double u,
                                                           double v, double w, double gamma) {
  return (gamma - 1.0) * (e - 0.5 * r * (u * u + v * v + w * w) - 0.5 * (bx * bx + by * by + bz * bz));
}

// float32 state: the same difference evaluated in float64 from the stored values, so
// the cancellation of low-beta cells costs no extra rounding.
template <>
__device__ __forceinline__ float recover_pressure<float>(float r, float m0, float m1, float m2, float e,
                                                         float bx, float by, float bz, float, float,
                                                         float, double gamma) {
  double inv_r = double(__fdividef(1.0f, r));
  inv_r = inv_r * (2.0 - double(r) * inv_r);
  const double kinetic = 0.5 * (double(m0) * m0 + double(m1) * m1 + double(m2) * m2) * inv_r;
  const double magnetic = 0.5 * (double(bx) * bx + double(by) * by + double(bz) * bz);
  return float((gamma - 1.0) * (double(e) - kinetic - magnetic));
}

}  // namespace wb

#include "numerics_lanes.cuh"
