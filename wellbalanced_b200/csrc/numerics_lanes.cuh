// The float32 face arithmetic (MUSCL slopes, HLLD) written over lane types: `L1` (one
// face) and `F2` (two faces at once on the packed float32 instructions of sm_100).
//
// Same formulas, region selection and near-degenerate fallback as the float64 templates of
// numerics.cuh (mhd_sweep_pyccel.py:25-48, 51-61, 64-98, 101-145, 148-251; Miyoshi & Kusano
// 2005); the multiply-adds are explicit, so one face gets the same bits in either lane type.
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

template <typename V>
__device__ __forceinline__ void hlld_front_l(const V (&L)[7], const V (&Rt)[7], V bn, V gamma, HlldFrontL<V>& o) {
  const V rl = L[0], vl = L[1], rr = Rt[0], vr = Rt[1];
  const V cf = lmax(fast_speed_l(rl, L[4], bn, L[5], L[6], gamma), fast_speed_l(rr, Rt[4], bn, Rt[5], Rt[6], gamma));
  o.sl = lmin(vl, vr) - cf;
  o.sr = lmax(vl, vr) + cf;
  const V bn2 = bn * bn;
  o.ptl = fma(V(0.5f), fma(L[5], L[5], fma(L[6], L[6], bn2)), L[4]);
  o.ptr = fma(V(0.5f), fma(Rt[5], Rt[5], fma(Rt[6], Rt[6], bn2)), Rt[4]);
  const V dl = (o.sl - vl) * rl;
  const V dr = (o.sr - vr) * rr;
  const V ndl = lneg(dl);
  const V inv_dd = linv(dr - dl);
  o.sm = fma(dr, vr, fma(ndl, vl, o.ptl - o.ptr)) * inv_dd;
  o.pts = fma(dr, o.ptl, fma(ndl, o.ptr, dl * dr * (vr - vl))) * inv_dd;
  star_tangential_l(L, bn, bn2, o.sl, dl, o.ptl, o.sm, o.rsl, o.vtl1, o.vtl2, o.btl1, o.btl2, o.den_l);
  star_tangential_l(Rt, bn, bn2, o.sr, dr, o.ptr, o.sm, o.rsr, o.vtr1, o.vtr2, o.btr1, o.btr2, o.den_r);
}

// Where a lane's star denominator is near zero (relative size below kNearDegenerate32),
// that lane's front half is redone in float64 from its float32 inputs.
template <typename V>
__device__ __forceinline__ void hlld_front_checked_l(const V (&L)[7], const V (&Rt)[7], V bn, V gamma,
                                                     HlldFrontL<V>& o) {
  hlld_front_l(L, Rt, bn, gamma, o);
  const V bn2 = bn * bn;
  const V near = V(kNearDegenerate32);
  const auto mask = labs(o.den_l) < near * (o.ptl + bn2) | labs(o.den_r) < near * (o.ptr + bn2);
  if (!any(mask)) return;
#pragma unroll
  for (int i = 0; i < Lanes<V>::kCount; ++i) {
    if (!lane_mask(mask, i)) continue;
    double Ld[7], Rd[7];
#pragma unroll
    for (int c = 0; c < 7; ++c) {
      Ld[c] = lane(L[c], i);
      Rd[c] = lane(Rt[c], i);
    }
    HlldFront<double> d;
    hlld_front<double, MathRefined>(Ld, Rd, double(lane(bn, i)), double(lane(gamma, i)), d);
    set_lane(o.sl, i, float(d.sl)), set_lane(o.sr, i, float(d.sr));
    set_lane(o.ptl, i, float(d.ptl)), set_lane(o.ptr, i, float(d.ptr));
    set_lane(o.sm, i, float(d.sm)), set_lane(o.pts, i, float(d.pts));
    set_lane(o.rsl, i, float(d.rsl)), set_lane(o.vtl1, i, float(d.vtl1)), set_lane(o.vtl2, i, float(d.vtl2));
    set_lane(o.btl1, i, float(d.btl1)), set_lane(o.btl2, i, float(d.btl2)), set_lane(o.den_l, i, float(d.den_l));
    set_lane(o.rsr, i, float(d.rsr)), set_lane(o.vtr1, i, float(d.vtr1)), set_lane(o.vtr2, i, float(d.vtr2));
    set_lane(o.btr1, i, float(d.btr1)), set_lane(o.btr2, i, float(d.btr2)), set_lane(o.den_r, i, float(d.den_r));
  }
}

// HLLD flux of one face per lane (straight-line code: the star / double-star flux of the
// side of the contact the face lies on, selected at the end; as hlld_flux in numerics.cuh).
template <typename V>
__device__ __forceinline__ void hlld_flux_l(const V (&L)[7], const V (&Rt)[7], V bn, V gamma, V inv_gm1,
                                            V (&F)[7]) {
  HlldFrontL<V> fr;
  hlld_front_checked_l(L, Rt, bn, gamma, fr);
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

// Left / right states of a face from four consecutive cells (face between q1 and q2),
// first order where a reconstructed density or pressure is not positive.
template <int LIM, typename V>
__device__ __forceinline__ void reconstruct_l(const V (&q0)[7], const V (&q1)[7], const V (&q2)[7],
                                              const V (&q3)[7], V (&L)[7], V (&Rt)[7]) {
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    const V d1 = q2[c] - q1[c];
    const V s1 = limited_slope_l<LIM>(q1[c] - q0[c], d1);
    const V s2 = limited_slope_l<LIM>(d1, q3[c] - q2[c]);
    L[c] = fma(V(0.5f), s1, q1[c]);
    Rt[c] = fma(V(-0.5f), s2, q2[c]);
  }
  const auto first_order = L[0] <= V(0.0f) | L[4] <= V(0.0f) | Rt[0] <= V(0.0f) | Rt[4] <= V(0.0f);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    L[c] = sel(first_order, q1[c], L[c]);
    Rt[c] = sel(first_order, q2[c], Rt[c]);
  }
}

// The same from the two cells beside the face and their limited slopes, already formed.
template <typename V>
__device__ __forceinline__ void reconstruct_sloped_l(const V (&q1)[7], const V (&q2)[7], const V (&s1)[7],
                                                     const V (&s2)[7], V (&L)[7], V (&Rt)[7]) {
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    L[c] = fma(V(0.5f), s1[c], q1[c]);
    Rt[c] = fma(V(-0.5f), s2[c], q2[c]);
  }
  const auto first_order = L[0] <= V(0.0f) | L[4] <= V(0.0f) | Rt[0] <= V(0.0f) | Rt[4] <= V(0.0f);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    L[c] = sel(first_order, q1[c], L[c]);
    Rt[c] = sel(first_order, q2[c], Rt[c]);
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

__device__ __forceinline__ void hlld_flux(const float (&L)[7], const float (&Rt)[7], float bn, float gamma,
                                          float inv_gm1, float (&F)[7]) {
  L1 l[7], r[7], f[7];
  to_lanes(L, l);
  to_lanes(Rt, r);
  hlld_flux_l<L1>(l, r, L1(bn), L1(gamma), L1(inv_gm1), f);
  from_lanes(f, F);
}

template <int LIM>
__device__ __forceinline__ void reconstruct(const float (&q0)[7], const float (&q1)[7], const float (&q2)[7],
                                            const float (&q3)[7], float (&L)[7], float (&Rt)[7]) {
  L1 a0[7], a1[7], a2[7], a3[7], l[7], r[7];
  to_lanes(q0, a0);
  to_lanes(q1, a1);
  to_lanes(q2, a2);
  to_lanes(q3, a3);
  reconstruct_l<LIM>(a0, a1, a2, a3, l, r);
  from_lanes(l, L);
  from_lanes(r, Rt);
}

__device__ __forceinline__ void reconstruct_sloped(const float (&q1)[7], const float (&q2)[7], const float (&s1)[7],
                                                   const float (&s2)[7], float (&L)[7], float (&Rt)[7]) {
  L1 a1[7], a2[7], b1[7], b2[7], l[7], r[7];
  to_lanes(q1, a1);
  to_lanes(q2, a2);
  to_lanes(s1, b1);
  to_lanes(s2, b2);
  reconstruct_sloped_l(a1, a2, b1, b2, l, r);
  from_lanes(l, L);
  from_lanes(r, Rt);
}

template <int LIM>
__device__ __forceinline__ float limited_slope(float a, float b) {
  return limited_slope_l<LIM>(L1(a), L1(b)).v;
}

}  // namespace wb
