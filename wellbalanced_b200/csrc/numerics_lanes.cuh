// The float32 face arithmetic (MUSCL slopes, HLLD) written over lane types: `L1` (one
// value) and `F2` (two values on the packed float32 instructions of sm_100). A face pairs
// what it computes twice: the left and right states' slopes and reconstruction, their fast
// speeds, total pressures and star states; the rest runs on one lane.
//
// Same formulas, region selection and near-degenerate fallback as the float64 templates of
// numerics.cuh (mhd_sweep_pyccel.py:25-48, 51-61, 64-98, 101-145, 148-251; Miyoshi & Kusano
// 2005); the multiply-adds are explicit and every float32 face of every kernel (stage
// kernels, refluxing) runs this code, so a face's flux has the same bits wherever it is
// formed.
#pragma once

#include "lanes.cuh"

namespace wb {

template <typename V>
__device__ __forceinline__ V lsqrt(V x) {  // x > 0 ? sqrt(x) : 0, as x rsqrt(x)
  return sel(x > V(0.0f), x * lrsqrt(x), V(0.0f));
}

template <int LIM, typename V>
__device__ __forceinline__ V limited_slope_l(V a, V b) {
  if (LIM == 3) return V(0.5f) * (a + b);
  const auto same = a * b > V(0.0f);
  V slope;
  if (LIM == 0) {
    slope = sel(labs(a) < labs(b), a, b);
  } else if (LIM == 1) {
    const V sum = a + b;
    slope = V(2.0f) * (a * b) * linv(sum);
  } else {
    const V central = V(0.5f) * (a + b);
    const V bound = V(2.0f) * lmin(labs(a), labs(b));
    slope = lcopysign(lmin(labs(central), bound), a);
  }
  return sel(same, slope, V(0.0f));
}

// Fast magnetosonic speed along the normal (the discriminant clipped at zero).
template <typename V>
__device__ __forceinline__ V fast_speed_l(V rho, V p, V bn, V bt1, V bt2, V gamma) {
  const V ir = linv(rho);
  const V a2 = gamma * p * ir;
  const V bn2 = bn * bn;
  const V b2 = fma(bt1, bt1, fma(bt2, bt2, bn2)) * ir;
  const V s = a2 + b2;
  const V disc = fma(V(-4.0f) * a2 * ir, bn2, s * s);
  return lsqrt(V(0.5f) * (s + lsqrt(disc)));
}

// Conserved state and normal flux of a normal-frame primitive state; returns p_T.
template <typename V>
__device__ __forceinline__ V side_state_l(const V (&w)[7], V bn, V nbn, V inv_gm1, V (&u)[7], V (&f)[7]) {
  const V rho = w[0], vn = w[1], vt1 = w[2], vt2 = w[3], p = w[4], bt1 = w[5], bt2 = w[6];
  const V magnetic = V(0.5f) * fma(bn, bn, fma(bt1, bt1, bt2 * bt2));
  const V kinetic2 = fma(vn, vn, fma(vt1, vt1, vt2 * vt2));
  const V energy = fma(p, inv_gm1, fma(V(0.5f) * rho, kinetic2, magnetic));
  const V pt = p + magnetic;
  const V vb = fma(vn, bn, fma(vt1, bt1, vt2 * bt2));
  const V mass = rho * vn;
  u[0] = rho;
  u[1] = mass;
  u[2] = rho * vt1;
  u[3] = rho * vt2;
  u[4] = energy;
  u[5] = bt1;
  u[6] = bt2;
  f[0] = mass;
  f[1] = fma(mass, vn, pt - bn * bn);
  f[2] = fma(mass, vt1, nbn * bt1);
  f[3] = fma(mass, vt2, nbn * bt2);
  f[4] = fma(energy + pt, vn, nbn * vb);
  f[5] = fma(bt1, vn, nbn * vt1);
  f[6] = fma(bt2, vn, nbn * vt2);
  return pt;
}

// The wave speeds, S_M, p_T* and both sides' star density, tangential velocity and field.
template <typename V>
struct HlldFrontL {
  V sl, sr, ptl, ptr, sm, pts;
  V rsl, vtl1, vtl2, btl1, btl2, den_l;
  V rsr, vtr1, vtr2, btr1, btr2, den_r;
};

// Star tangential velocity and field of one side; `den` returns d (s - s_M) - B_n^2.
template <typename V>
__device__ __forceinline__ void star_tangential_l(const V (&w)[7], V bn, V bn2, V s, V d, V pt, V sm, V& rho_s,
                                                  V& vt1, V& vt2, V& bt1, V& bt2, V& den) {
  const V vn = w[1];
  const V ssm = s - sm;
  rho_s = d * linv(ssm);
  den = fma(d, ssm, lneg(bn2));
  const auto regular = labs(den) >= V(float(kDegenerate)) * (pt + bn2);
  const V inv_den = linv(den);
  const V scale = fma(d, s - vn, lneg(bn2)) * inv_den;
  const V shift = bn * (vn - sm) * inv_den;
  vt1 = sel(regular, fma(shift, w[5], w[2]), w[2]);
  vt2 = sel(regular, fma(shift, w[6], w[3]), w[3]);
  bt1 = sel(regular, w[5] * scale, w[5]);
  bt2 = sel(regular, w[6] * scale, w[6]);
}

// The front half of one face with its left and right sides in the two lanes of F2 (fast
// speeds, total pressures, d = (S - v) rho and the star states of both sides in one packed
// evaluation each); S_M and p_T* on one lane. Where either side's star denominator is near
// zero (relative size below kNearDegenerate32) the front is redone in float64 from the
// float32 inputs.
__device__ __forceinline__ void hlld_front_lr(const float (&L)[7], const float (&Rt)[7], float bn, float gamma,
                                              HlldFrontL<L1>& o) {
  F2 w[7];
#pragma unroll
  for (int c = 0; c < 7; ++c) w[c] = F2(L[c], Rt[c]);
  const L1 vl = L[1], vr = Rt[1];
  const F2 cf2 = fast_speed_l<F2>(w[0], w[4], F2(bn), w[5], w[6], F2(gamma));
  const L1 cf = lmax(L1(cf2.v.x), L1(cf2.v.y));
  o.sl = lmin(vl, vr) - cf;
  o.sr = lmax(vl, vr) + cf;
  const L1 bn2 = L1(bn) * L1(bn);
  const F2 pt2 = fma(F2(0.5f), fma(w[5], w[5], fma(w[6], w[6], F2(bn2.v))), w[4]);
  o.ptl = pt2.v.x;
  o.ptr = pt2.v.y;
  const F2 s2(o.sl.v, o.sr.v);
  const F2 d2 = (s2 - w[1]) * w[0];
  const L1 dl = d2.v.x, dr = d2.v.y;
  const L1 ndl = lneg(dl);
  const L1 inv_dd = linv(dr - dl);
  o.sm = fma(dr, vr, fma(ndl, vl, o.ptl - o.ptr)) * inv_dd;
  o.pts = fma(dr, o.ptl, fma(ndl, o.ptr, dl * dr * (vr - vl))) * inv_dd;
  F2 rho_s, vt1, vt2, bt1, bt2, den;
  star_tangential_l<F2>(w, F2(bn), F2(bn2.v), s2, d2, pt2, F2(o.sm.v), rho_s, vt1, vt2, bt1, bt2, den);
  o.rsl = rho_s.v.x, o.rsr = rho_s.v.y;
  o.vtl1 = vt1.v.x, o.vtr1 = vt1.v.y;
  o.vtl2 = vt2.v.x, o.vtr2 = vt2.v.y;
  o.btl1 = bt1.v.x, o.btr1 = bt1.v.y;
  o.btl2 = bt2.v.x, o.btr2 = bt2.v.y;
  o.den_l = den.v.x, o.den_r = den.v.y;
  if (!any(labs(den) < F2(kNearDegenerate32) * (pt2 + F2(bn2.v)))) return;
  double Ld[7], Rd[7];
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    Ld[c] = L[c];
    Rd[c] = Rt[c];
  }
  HlldFront<double> d;
  hlld_front<double, MathRefined>(Ld, Rd, double(bn), double(gamma), d);
  o.sl = float(d.sl), o.sr = float(d.sr), o.ptl = float(d.ptl), o.ptr = float(d.ptr);
  o.sm = float(d.sm), o.pts = float(d.pts);
  o.rsl = float(d.rsl), o.vtl1 = float(d.vtl1), o.vtl2 = float(d.vtl2);
  o.btl1 = float(d.btl1), o.btl2 = float(d.btl2), o.den_l = float(d.den_l);
  o.rsr = float(d.rsr), o.vtr1 = float(d.vtr1), o.vtr2 = float(d.vtr2);
  o.btr1 = float(d.btr1), o.btr2 = float(d.btr2), o.den_r = float(d.den_r);
}

// The back half of the HLLD flux from its front (straight-line code: the star / double-star
// flux of the side of the contact the face lies on, selected at the end; as hlld_flux in
// numerics.cuh).
template <typename V>
__device__ __forceinline__ void hlld_tail_l(const V (&L)[7], const V (&Rt)[7], V bn, V inv_gm1,
                                            const HlldFrontL<V>& fr, V (&F)[7]) {
  const V sm = fr.sm;
  const V sql = lsqrt(fr.rsl);
  const V sqr = lsqrt(fr.rsr);
  const V sign = sel(bn > V(0.0f), V(1.0f), sel(bn < V(0.0f), V(-1.0f), V(0.0f)));
  const V inv_sum = linv(sql + sqr);
  const V vt2_1 = fma(sql, fr.vtl1, fma(sqr, fr.vtr1, (fr.btr1 - fr.btl1) * sign)) * inv_sum;
  const V vt2_2 = fma(sql, fr.vtl2, fma(sqr, fr.vtr2, (fr.btr2 - fr.btl2) * sign)) * inv_sum;
  const V cross = sql * sqr * sign;
  const V bt2_1 = fma(sql, fr.btr1, fma(sqr, fr.btl1, cross * (fr.vtr1 - fr.vtl1))) * inv_sum;
  const V bt2_2 = fma(sql, fr.btr2, fma(sqr, fr.btl2, cross * (fr.vtr2 - fr.vtl2))) * inv_sum;
  const V vb2 = fma(sm, bn, fma(vt2_1, bt2_1, vt2_2 * bt2_2));
  // the side of the contact the face lies on (also the upwind side when supersonic)
  const auto left = sm >= V(0.0f);
  V w[7];
#pragma unroll
  for (int c = 0; c < 7; ++c) w[c] = sel(left, L[c], Rt[c]);
  const V s = sel(left, fr.sl, fr.sr);
  const V pt = sel(left, fr.ptl, fr.ptr);
  const V rho_s = sel(left, fr.rsl, fr.rsr);
  const V vt1 = sel(left, fr.vtl1, fr.vtr1);
  const V vt2 = sel(left, fr.vtl2, fr.vtr2);
  const V bt1 = sel(left, fr.btl1, fr.btr1);
  const V bt2 = sel(left, fr.btl2, fr.btr2);
  const V sq = sel(left, sql, sqr);
  const V alfven = labs(bn) * linv(sq);
  const V ss = sel(left, sm - alfven, sm + alfven);
  const auto twice = left ^ (ss >= V(0.0f));
  const auto supersonic = fr.sl >= V(0.0f) | fr.sr < V(0.0f);
  const V sense = sel(left, V(-1.0f), V(1.0f));
  const V nbn = lneg(bn);
  V u[7], f[7];
  side_state_l(w, bn, nbn, inv_gm1, u, f);
  const V vn = w[1];
  const V vb = fma(vn, bn, fma(w[2], w[5], w[3] * w[6]));
  const V vb_s = fma(sm, bn, fma(vt1, bt1, vt2 * bt2));
  const V energy_s =
      fma(s - vn, u[4], fma(fr.pts, sm, fma(bn, vb - vb_s, lneg(pt) * vn))) * linv(s - sm);
  V us[7], ud[7];
  us[0] = rho_s;
  us[1] = rho_s * sm;
  us[2] = rho_s * vt1;
  us[3] = rho_s * vt2;
  us[4] = energy_s;
  us[5] = bt1;
  us[6] = bt2;
  ud[2] = rho_s * vt2_1;
  ud[3] = rho_s * vt2_2;
  ud[4] = fma(sense * sq * sign, vb_s - vb2, energy_s);
  ud[5] = bt2_1;
  ud[6] = bt2_2;
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    const V star = fma(s, us[c] - u[c], f[c]);
    // the double-star state differs from the star state in rows 2-6 only
    const V twice_star = c < 2 ? star : fma(ss, ud[c] - us[c], star);
    F[c] = sel(supersonic, f[c], sel(twice, twice_star, star));
  }
}

// ---- float32 entry points of the kernels: one face (L1) ------------------------------------
template <typename V, int N>
__device__ __forceinline__ void to_lanes(const float (&a)[N], V (&b)[N]) {
#pragma unroll
  for (int c = 0; c < N; ++c) b[c] = V(a[c]);
}

template <int N>
__device__ __forceinline__ void from_lanes(const L1 (&a)[N], float (&b)[N]) {
#pragma unroll
  for (int c = 0; c < N; ++c) b[c] = a[c].v;
}

// The float32 HLLD flux of one face: front on the packed lanes, back half on one lane.
__device__ __forceinline__ void hlld_flux(const float (&L)[7], const float (&Rt)[7], float bn, float gamma,
                                          float inv_gm1, float (&F)[7]) {
  HlldFrontL<L1> fr;
  hlld_front_lr(L, Rt, bn, gamma, fr);
  L1 l[7], r[7], f[7];
  to_lanes(L, l);
  to_lanes(Rt, r);
  hlld_tail_l<L1>(l, r, L1(bn), L1(inv_gm1), fr, f);
  from_lanes(f, F);
}

// One face's reconstruction with its left and right states in the two lanes of F2: the
// two limited slopes of each component in one packed evaluation (lane x: the cell below the
// face, lane y: the cell above), the states as one packed FMA. Lane by lane the same
// operations as the one-lane form.
template <int LIM>
__device__ __forceinline__ void reconstruct(const float (&q0)[7], const float (&q1)[7], const float (&q2)[7],
                                            const float (&q3)[7], float (&L)[7], float (&Rt)[7]) {
  const F2 half(0.5f, -0.5f);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    const F2 a01(q0[c], q1[c]), a12(q1[c], q2[c]), a23(q2[c], q3[c]);
    const F2 lr = fma(half, limited_slope_l<LIM>(a12 - a01, a23 - a12), a12);
    L[c] = lr.v.x;
    Rt[c] = lr.v.y;
  }
  const bool first_order = L[0] <= 0.0f || L[4] <= 0.0f || Rt[0] <= 0.0f || Rt[4] <= 0.0f;
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    L[c] = first_order ? q1[c] : L[c];
    Rt[c] = first_order ? q2[c] : Rt[c];
  }
}

__device__ __forceinline__ void reconstruct_sloped(const float (&q1)[7], const float (&q2)[7], const float (&s1)[7],
                                                   const float (&s2)[7], float (&L)[7], float (&Rt)[7]) {
  const F2 half(0.5f, -0.5f);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    const F2 lr = fma(half, F2(s1[c], s2[c]), F2(q1[c], q2[c]));
    L[c] = lr.v.x;
    Rt[c] = lr.v.y;
  }
  const bool first_order = L[0] <= 0.0f || L[4] <= 0.0f || Rt[0] <= 0.0f || Rt[4] <= 0.0f;
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    L[c] = first_order ? q1[c] : L[c];
    Rt[c] = first_order ? q2[c] : Rt[c];
  }
}

// Limited slopes of seven components from their backward (a) and forward (b) differences,
// two components per packed evaluation (lane by lane as limited_slope_l<L1>).
template <int LIM>
__device__ __forceinline__ void limited_slopes7(const float (&a)[7], const float (&b)[7], float (&out)[7]) {
#pragma unroll
  for (int c = 0; c < 6; c += 2) {
    const F2 s = limited_slope_l<LIM>(F2(a[c], a[c + 1]), F2(b[c], b[c + 1]));
    out[c] = s.v.x;
    out[c + 1] = s.v.y;
  }
  out[6] = limited_slope_l<LIM>(L1(a[6]), L1(b[6])).v;
}

template <int LIM>
__device__ __forceinline__ float limited_slope(float a, float b) {
  return limited_slope_l<LIM>(L1(a), L1(b)).v;
}

}  // namespace wb
