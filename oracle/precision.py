"""The 2D Orszag-Tang step with a chosen float type per phase (test infrastructure only).

ORACLE — a restatement of the reference's periodic 2D step used to find where a
float32 run's error against the float64 one comes from: the state's storage, the
primitive recovery, the reconstruction, the HLLD flux, the CT electric field or the
conserved update, each in float32 or float64 (NumPy float32 is IEEE). Only the tests and
the precision study in the design notes use it; the product never imports it.

The arithmetic follows the reference kernels: primitive recovery
``kernels/mhd_primitive/mhd_primitive_pyccel.py:23-87``; MC-limited PLM with the
first-order fallback ``kernels/mhd_sweep/mhd_sweep_pyccel.py:25-48, 286-307``; HLLD
``mhd_sweep_pyccel.py:51-251``; CT-contact ``kernels/ct_contact/ct_contact_pyccel.py:26-61``;
the Heun step ``carafe/mhd.py:965-994``; the stable step ``mhd_rate_pyccel.py:30-83``.
In float64 it equals the reference's run of config 1 (the committed fixture) to 2e-12.

    python -m oracle.precision 256 store=32          # float32 storage only
    python -m oracle.precision 256 all=32,update=64  # float32 except the update
"""

from __future__ import annotations

import sys
import time

import numpy as np

GAMMA = 5.0 / 3.0
DEGENERATE = 1.0e-12
PHASES = ("store", "prim", "recon", "hlld", "ct", "update")


def _mc(a, b):
    same = a * b > 0
    central = 0.5 * (a + b)
    bound = 2.0 * np.where(np.abs(a) < np.abs(b), a, b)
    return np.where(same, np.sign(central) * np.minimum(np.abs(central), np.abs(bound)), 0 * a)


def _fast(rho, p, bn, bt1, bt2, g):
    a2 = g * p / rho
    b2 = (bn * bn + bt1 * bt1 + bt2 * bt2) / rho
    disc = (a2 + b2) * (a2 + b2) - 4.0 * a2 * bn * bn / rho
    return np.sqrt(0.5 * (a2 + b2 + np.sqrt(np.where(disc > 0, disc, 0 * disc))))


def _side(w, bn, g):
    rho, vn, vt1, vt2, p, bt1, bt2 = w
    mag = 0.5 * (bn * bn + bt1 * bt1 + bt2 * bt2)
    energy = p / (g - 1.0) + 0.5 * rho * (vn * vn + vt1 * vt1 + vt2 * vt2) + mag
    pt = p + mag
    vb = vn * bn + vt1 * bt1 + vt2 * bt2
    u = np.stack((rho, rho * vn, rho * vt1, rho * vt2, energy, bt1, bt2))
    f = np.stack((rho * vn, rho * vn * vn + pt - bn * bn, rho * vn * vt1 - bn * bt1, rho * vn * vt2 - bn * bt2,
                  (energy + pt) * vn - bn * vb, bt1 * vn - bn * vt1, bt2 * vn - bn * vt2))
    return u, f, pt


def _star(w, u, bn, s, d, pt, sm, pts):
    vn = w[1]
    rho_s = d / (s - sm)
    den = d * (s - sm) - bn * bn
    regular = np.abs(den) >= DEGENERATE * (pt + bn * bn)
    safe = np.where(regular, den, 1.0 + 0 * den)
    vt1 = np.where(regular, w[2] - bn * w[5] * (sm - vn) / safe, w[2])
    vt2 = np.where(regular, w[3] - bn * w[6] * (sm - vn) / safe, w[3])
    bt1 = np.where(regular, w[5] * (d * (s - vn) - bn * bn) / safe, w[5])
    bt2 = np.where(regular, w[6] * (d * (s - vn) - bn * bn) / safe, w[6])
    vb = vn * bn + w[2] * w[5] + w[3] * w[6]
    vb_s = sm * bn + vt1 * bt1 + vt2 * bt2
    energy = ((s - vn) * u[4] - pt * vn + pts * sm + bn * (vb - vb_s)) / (s - sm)
    return np.stack((rho_s, rho_s * sm, rho_s * vt1, rho_s * vt2, energy, bt1, bt2)), (vt1, vt2), (bt1, bt2), vb_s


def hlld(L, R, bn, g):
    ul, fl, ptl = _side(L, bn, g)
    ur, fr, ptr = _side(R, bn, g)
    rl, vl, rr, vr = L[0], L[1], R[0], R[1]
    cf = np.maximum(_fast(rl, L[4], bn, L[5], L[6], g), _fast(rr, R[4], bn, R[5], R[6], g))
    sl, sr = np.minimum(vl, vr) - cf, np.maximum(vl, vr) + cf
    dl, dr = (sl - vl) * rl, (sr - vr) * rr
    sm = (dr * vr - dl * vl - ptr + ptl) / (dr - dl)
    pts = (dr * ptl - dl * ptr + dl * dr * (vr - vl)) / (dr - dl)
    usl, vtl, btl, vbl = _star(L, ul, bn, sl, dl, ptl, sm, pts)
    usr, vtr, btr, vbr = _star(R, ur, bn, sr, dr, ptr, sm, pts)
    sql, sqr = np.sqrt(usl[0]), np.sqrt(usr[0])
    sign = np.sign(bn)
    total = sql + sqr
    vt2 = [(sql * vtl[c] + sqr * vtr[c] + (btr[c] - btl[c]) * sign) / total for c in (0, 1)]
    bt2 = [(sql * btr[c] + sqr * btl[c] + sql * sqr * (vtr[c] - vtl[c]) * sign) / total for c in (0, 1)]
    vb2 = sm * bn + vt2[0] * bt2[0] + vt2[1] * bt2[1]

    def double(us, vb_s, sq, sense):
        r = us[0]
        return np.stack((r, r * sm, r * vt2[0], r * vt2[1], us[4] + sense * sq * (vb_s - vb2) * sign, bt2[0], bt2[1]))

    uddl, uddr = double(usl, vbl, sql, -1.0), double(usr, vbr, sqr, 1.0)
    ssl, ssr = sm - np.abs(bn) / sql, sm + np.abs(bn) / sqr
    star_l, star_r = fl + sl * (usl - ul), fr + sr * (usr - ur)
    F = np.where(ssr >= 0, star_r + ssr * (uddr - usr), star_r)
    F = np.where(sm >= 0, star_l + ssl * (uddl - usl), F)
    F = np.where(ssl >= 0, star_l, F)
    F = np.where(sr < 0, fr, F)
    return np.where(sl >= 0, fl, F)


def _upwind(m, pos, neg):
    return np.where(m > 0, pos, np.where(m < 0, neg, 0.5 * (pos + neg)))


class Step:
    """The periodic n^2 Orszag-Tang step on arrays: U (6, n, n), nodal A_z (n, n)."""

    def __init__(self, n, types):
        self.n = n
        self.t = types

    def primitives(self, U, A, ft):
        h = 1.0 / self.n
        rho, mx, my, mz, E, bz = U.astype(ft)
        # face fields from differences of A in its stored type, then the phase's type
        ha = A.dtype.type(h)
        bxf = ((np.roll(A, -1, 1) - A) / ha).astype(ft)
        byf = (-(np.roll(A, -1, 0) - A) / ha).astype(ft)
        bx, by = 0.5 * (bxf + np.roll(bxf, -1, 0)), 0.5 * (byf + np.roll(byf, -1, 1))
        u, v, w = mx / rho, my / rho, mz / rho
        p = (GAMMA - 1.0) * (E - 0.5 * rho * (u * u + v * v + w * w) - 0.5 * (bx * bx + by * by + bz * bz))
        return np.stack((rho, u, v, w, p, bx, by, bz)), bxf, byf, bx * v - by * u

    def rate(self, U, A):
        r, u, v, w, p, bx, by, bz = self.primitives(U, A, np.float64)[0]
        n = self.n
        return float(np.max((np.abs(u) + _fast(r, p, bx, by, bz, GAMMA)) * n + (np.abs(v) + _fast(r, p, by, bx, bz, GAMMA)) * n))

    def sweep(self, q, bn, axis):
        q = q.astype(self.t["recon"])
        a = axis + 1
        dq = q - np.roll(q, 1, a)
        s = _mc(dq, np.roll(dq, -1, a))
        L, R = np.roll(q + 0.5 * s, 1, a), q - 0.5 * s
        bad = (L[0] <= 0) | (L[4] <= 0) | (R[0] <= 0) | (R[4] <= 0)
        L, R = np.where(bad, np.roll(q, 1, a), L), np.where(bad, q, R)
        ht = self.t["hlld"]
        return hlld(L.astype(ht), R.astype(ht), bn.astype(ht), ht(GAMMA))

    def stage(self, U, A, dt, base=None):
        t = self.t
        prim, bxf, byf, ecc = self.primitives(U, A, t["prim"])
        fx = self.sweep(prim[[0, 1, 2, 3, 4, 6, 7]], bxf, 0)
        fy = self.sweep(prim[[0, 2, 1, 3, 4, 5, 7]], byf, 1)
        c = t["ct"]
        fx, fy, e = fx.astype(c), fy.astype(c), ecc.astype(c)
        lower, upper = np.roll(fx[5], 1, 1), fx[5]
        left, right = np.roll(fy[5], 1, 0), fy[5]
        e00, e10, e01 = np.roll(np.roll(e, 1, 0), 1, 1), np.roll(e, 1, 1), np.roll(e, 1, 0)
        dl2 = _upwind(np.roll(fx[0], 1, 1), left - e00, right - e10)
        dr2 = _upwind(fx[0], left - e01, right - e)
        dl1 = _upwind(np.roll(fy[0], 1, 0), -lower - e00, -upper - e01)
        dr1 = _upwind(fy[0], -lower - e10, -upper - e)
        ez = 0.25 * (right + left - upper - lower + dl1 + dr1 + dl2 + dr2)
        ud = t["update"]
        h = ud(1.0 / self.n)
        fx, fy = fx.astype(ud), fy.astype(ud)
        xr, yr = [0, 1, 2, 3, 4, 6], [0, 2, 1, 3, 4, 6]
        div = np.stack([(np.roll(fx[xr[k]], -1, 0) - fx[xr[k]]) / h + (np.roll(fy[yr[k]], -1, 1) - fy[yr[k]]) / h
                        for k in range(6)])
        Un, An = U.astype(ud) - ud(dt) * div, A.astype(ud) - ud(dt) * ez.astype(ud)
        if base is not None:
            Un, An = (Un + base[0].astype(ud)) * ud(0.5), (An + base[1].astype(ud)) * ud(0.5)
        return Un.astype(t["store"]), An.astype(t["store"])

    def run(self, U, A, dts=None, end=0.5, cfl=0.4):
        """Steps to `end` at the stable step (float64), or with the given dts."""
        U, A = U.astype(self.t["store"]), A.astype(self.t["store"])
        taken, t = [], 0.0
        while (t < end * (1.0 - 1e-14)) if dts is None else len(taken) < len(dts):
            dt = min(cfl / self.rate(U, A), end - t) if dts is None else dts[len(taken)]
            U1, A1 = self.stage(U, A, dt)
            U, A = self.stage(U1, A1, dt, base=(U, A))
            t += dt
            taken.append(dt)
        return U, A, taken


def orszag_tang(n):
    """The config-1 initial state (``carafe/mhd.py:533-559``) on n^2 cells."""
    x, xn = (np.arange(n) + 0.5) / n, np.arange(n) / n
    X, Y = np.meshgrid(x, x, indexing="ij")
    XN, YN = np.meshgrid(xn, xn, indexing="ij")
    b0 = 1.0 / np.sqrt(4 * np.pi)
    rho, p = np.full((n, n), 25.0 / (36.0 * np.pi)), np.full((n, n), 5.0 / (12.0 * np.pi))
    u, v = -np.sin(2 * np.pi * Y), np.sin(2 * np.pi * X)
    A = b0 * (np.cos(4 * np.pi * XN) / (4 * np.pi) + np.cos(2 * np.pi * YN) / (2 * np.pi))
    bxf, byf = (np.roll(A, -1, 1) - A) * n, -(np.roll(A, -1, 0) - A) * n
    bx, by = 0.5 * (bxf + np.roll(bxf, -1, 0)), 0.5 * (byf + np.roll(byf, -1, 1))
    E = p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v) + 0.5 * (bx * bx + by * by)
    return np.stack((rho, rho * u, rho * v, 0 * X, E, 0 * X)), A


def types(spec):
    """Phase types from "all=32,update=64"-style specs (float64 where not given)."""
    f = {"32": np.float32, "64": np.float64}
    out = dict.fromkeys(PHASES, np.float64)
    for item in filter(None, spec.split(",")):
        key, value = item.split("=")
        if key == "all":
            out = dict.fromkeys(PHASES, f[value])
        else:
            out[key] = f[value]
    return out


def main():
    n, spec = int(sys.argv[1]), sys.argv[2] if len(sys.argv) > 2 else "all=32"
    U0, A0 = orszag_tang(n)
    start = time.time()
    ref = Step(n, types(""))
    Ur, _, dts = ref.run(U0, A0)
    U, _, _ = Step(n, types(spec)).run(U0, A0, dts)
    rl1 = [float(np.sum(np.abs(U[f] - Ur[f])) / np.sum(np.abs(Ur[f]))) for f in (0, 4)]
    print(f"{n}^2 {spec}: {len(dts)} steps, relative L1 density {rl1[0]:.3e}, energy {rl1[1]:.3e} "
          f"({time.time() - start:.0f} s)")


if __name__ == "__main__":
    main()
