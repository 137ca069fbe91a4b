"""CPU restatement of the reference's six MHD block kernels (test infrastructure only).

ORACLE — this module is the correctness checker for the CUDA path. Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import it; the
product (``wellbalanced_b200``) never does.

Each function restates the arithmetic of one reference kernel (``carafe/kernels``),
vectorised with NumPy over a whole haloed block, float64, with the same argument order
and out-parameter convention as the reference:

* ``limited_slope``  — ``kernels/mhd_sweep/mhd_sweep_pyccel.py:25-48`` and
  ``limiters.py:18-46``;
* ``fast_speed``     — ``mhd_sweep_pyccel.py:51-61`` / ``mhd.py:144-149``;
* ``hlld``           — ``mhd_sweep_pyccel.py:64-251`` (``side_state``, ``star_state``,
  ``hlld_face``) and the vector form ``mhd.py:196-280``;
* ``mhd_sweep``      — ``mhd_sweep_pyccel.py:254-319``;
* ``mhd_primitive``  — ``kernels/mhd_primitive/mhd_primitive_pyccel.py:23-87``;
* ``ct_contact``     — ``kernels/ct_contact/ct_contact_pyccel.py:26-61``;
* ``mhd_rate``       — ``kernels/mhd_rate/mhd_rate_pyccel.py:30-83``;
* ``mhd_resistive``  — ``kernels/mhd_resistive/mhd_resistive_pyccel.py:21-67``;
* ``mhd_conductive`` — ``kernels/mhd_conductive/mhd_conductive_pyccel.py:38-100``.

Pinned against golden vectors produced by the reference itself (``tests/golden``).
"""

from __future__ import annotations

import numpy as np

#: Limiter codes of the ``limiter`` argument (``kernels/mhd_sweep/__init__.py:26-27``).
LIMITER_CODES = ("minmod", "vanleer", "mc", "none")
#: Relative size below which the HLLD star denominator counts as zero (``mhd.py:138``).
DEGENERATE = 1.0e-12


def limited_slope(a, b, limiter: int):
    """Limited PLM slope from backward ``a`` and forward ``b`` differences."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    if limiter == 3:
        return 0.5 * (a + b)
    same = a * b > 0.0
    if limiter == 0:
        pick = np.where(np.abs(a) < np.abs(b), a, b)
        return np.where(same, pick, 0.0)
    if limiter == 1:
        product = a * b
        return np.where(same, 2.0 * product / np.where(same, a + b, 1.0), 0.0)
    if limiter == 2:
        central = 0.5 * (a + b)
        bound = 2.0 * np.where(np.abs(a) < np.abs(b), a, b)
        size = np.minimum(np.abs(central), np.abs(bound))
        return np.where(same, np.sign(central) * size, 0.0)
    raise ValueError(f"limiter code {limiter} is not one of 0..3")


def fast_speed(rho, p, bn, bt1, bt2, gamma):
    """Fast magnetosonic speed along the normal (the discriminant clipped at zero)."""
    a2 = gamma * p / rho
    b2 = (bn * bn + bt1 * bt1 + bt2 * bt2) / rho
    disc = (a2 + b2) * (a2 + b2) - 4.0 * a2 * bn * bn / rho
    root = np.sqrt(np.where(disc > 0.0, disc, 0.0))
    return np.sqrt(0.5 * (a2 + b2 + root))


def _side(w, bn, gamma):
    """Conserved state, flux and total pressure of a normal-frame primitive state."""
    rho, vn, vt1, vt2, p, bt1, bt2 = w
    magnetic = 0.5 * (bn * bn + bt1 * bt1 + bt2 * bt2)
    energy = p / (gamma - 1.0) + 0.5 * rho * (vn * vn + vt1 * vt1 + vt2 * vt2) + magnetic
    pt = p + magnetic
    vb = vn * bn + vt1 * bt1 + vt2 * bt2
    u = np.stack((rho, rho * vn, rho * vt1, rho * vt2, energy, bt1, bt2))
    f = np.stack(
        (
            rho * vn,
            rho * vn * vn + pt - bn * bn,
            rho * vn * vt1 - bn * bt1,
            rho * vn * vt2 - bn * bt2,
            (energy + pt) * vn - bn * vb,
            bt1 * vn - bn * vt1,
            bt2 * vn - bn * vt2,
        )
    )
    return u, f, pt


def _star(w, u, bn, s, d, pt, sm, pts):
    """HLLD star state beside the contact, with its tangential velocity and field."""
    vn = w[1]
    with np.errstate(divide="ignore", invalid="ignore"):
        rho_s = d / (s - sm)
        den = d * (s - sm) - bn * bn
        regular = np.abs(den) >= DEGENERATE * (pt + bn * bn)
        safe = np.where(regular, den, 1.0)
        vt1 = np.where(regular, w[2] - bn * w[5] * (sm - vn) / safe, w[2])
        vt2 = np.where(regular, w[3] - bn * w[6] * (sm - vn) / safe, w[3])
        bt1 = np.where(regular, w[5] * (d * (s - vn) - bn * bn) / safe, w[5])
        bt2 = np.where(regular, w[6] * (d * (s - vn) - bn * bn) / safe, w[6])
        vb = vn * bn + w[2] * w[5] + w[3] * w[6]
        vb_s = sm * bn + vt1 * bt1 + vt2 * bt2
        energy = ((s - vn) * u[4] - pt * vn + pts * sm + bn * (vb - vb_s)) / (s - sm)
    us = np.stack((rho_s, rho_s * sm, rho_s * vt1, rho_s * vt2, energy, bt1, bt2))
    return us, (vt1, vt2), (bt1, bt2), vb_s


def hlld(left, right, bn, gamma):
    """HLLD flux (Miyoshi and Kusano 2005) between normal-frame states ``(7, ...)``."""
    left = np.asarray(left, dtype=float)
    right = np.asarray(right, dtype=float)
    bn = np.broadcast_to(np.asarray(bn, dtype=float), left.shape[1:])
    ul, fl, ptl = _side(left, bn, gamma)
    ur, fr, ptr = _side(right, bn, gamma)
    rl, vl = left[0], left[1]
    rr, vr = right[0], right[1]
    cf = np.maximum(
        fast_speed(rl, left[4], bn, left[5], left[6], gamma),
        fast_speed(rr, right[4], bn, right[5], right[6], gamma),
    )
    sl = np.minimum(vl, vr) - cf
    sr = np.maximum(vl, vr) + cf
    dl = (sl - vl) * rl
    dr = (sr - vr) * rr
    with np.errstate(divide="ignore", invalid="ignore"):
        sm = (dr * vr - dl * vl - ptr + ptl) / (dr - dl)
        pts = (dr * ptl - dl * ptr + dl * dr * (vr - vl)) / (dr - dl)
        usl, vtl, btl, vbl = _star(left, ul, bn, sl, dl, ptl, sm, pts)
        usr, vtr, btr, vbr = _star(right, ur, bn, sr, dr, ptr, sm, pts)
        sql = np.sqrt(usl[0])
        sqr = np.sqrt(usr[0])
        sign = np.where(bn > 0.0, 1.0, np.where(bn < 0.0, -1.0, 0.0))
        total = sql + sqr
        vt2 = [
            (sql * vtl[c] + sqr * vtr[c] + (btr[c] - btl[c]) * sign) / total for c in (0, 1)
        ]
        bt2 = [
            (sql * btr[c] + sqr * btl[c] + sql * sqr * (vtr[c] - vtl[c]) * sign) / total
            for c in (0, 1)
        ]
        vb2 = sm * bn + vt2[0] * bt2[0] + vt2[1] * bt2[1]

        def double(us, vb_s, sq, sense):
            rho_s = us[0]
            return np.stack(
                (
                    rho_s,
                    rho_s * sm,
                    rho_s * vt2[0],
                    rho_s * vt2[1],
                    us[4] + sense * sq * (vb_s - vb2) * sign,
                    bt2[0],
                    bt2[1],
                )
            )

        uddl = double(usl, vbl, sql, -1.0)
        uddr = double(usr, vbr, sqr, 1.0)
        ssl = sm - np.abs(bn) / sql
        ssr = sm + np.abs(bn) / sqr
        star_l = fl + sl * (usl - ul)
        star_r = fr + sr * (usr - ur)
        double_l = fl + sl * (usl - ul) + ssl * (uddl - usl)
        double_r = fr + sr * (usr - ur) + ssr * (uddr - usr)
    flux = np.where(ssr >= 0.0, double_r, star_r)
    flux = np.where(sm >= 0.0, double_l, flux)
    flux = np.where(ssl >= 0.0, star_l, flux)
    flux = np.where(sr < 0.0, fr, flux)
    flux = np.where(sl >= 0.0, fl, flux)
    return flux


def normal_frame(prim, axis: int):
    """The 7 normal-frame rows of ``prim`` (8, ...) for a sweep along block ``axis``.

    Density, normal velocity, the two tangential velocities, pressure and the two
    tangential fields; along x the tangential directions are (y, z), along y (x, z)
    (``mhd_sweep_pyccel.py:277-285``).
    """
    return prim[[0, 1 + axis, 2 - axis, 3, 4, 6 - axis, 7]]


def sweep_lines(q, bn, limiter: int, gamma: float, axis: int):
    """MUSCL + HLLD along ``axis`` (array axis ``1 + axis`` of ``q``, 7 rows first).

    ``q`` has ``n`` cells along the axis; faces ``k = 0 .. n - 4`` lie between cells
    ``k + 1`` and ``k + 2``; ``bn`` is the normal field at those faces. Returns the
    fluxes ``(7, ..., n - 3, ...)`` (``mhd_sweep_pyccel.py:286-319``).
    """
    a = 1 + axis
    n = q.shape[a]

    def cut(start, stop):
        return np.take(q, np.arange(start, stop), axis=a)

    diff = np.diff(q, axis=a)  # q[s + 1] - q[s]
    take = lambda start, stop: np.take(diff, np.arange(start, stop), axis=a)  # noqa: E731
    slope_left = limited_slope(take(0, n - 3), take(1, n - 2), limiter)  # cells 1..n-3
    slope_right = limited_slope(take(1, n - 2), take(2, n - 1), limiter)  # cells 2..n-2
    centre_left = cut(1, n - 2)
    centre_right = cut(2, n - 1)
    left = centre_left + 0.5 * slope_left
    right = centre_right - 0.5 * slope_right
    bad = (left[0] <= 0.0) | (left[4] <= 0.0) | (right[0] <= 0.0) | (right[4] <= 0.0)
    left = np.where(bad, centre_left, left)
    right = np.where(bad, centre_right, right)
    return hlld(left, right, bn, gamma)


def mhd_sweep(prim, bn, axis: int, limiter: int, gamma: float, flux) -> None:
    """Reference ``mhd_sweep(prim, bn, axis, limiter, gamma, flux)``; writes ``flux``."""
    q = normal_frame(np.asarray(prim, dtype=float), axis)
    normal = bn[2:-2, :] if axis == 0 else bn[:, 2:-2]
    flux[...] = sweep_lines(q, normal, limiter, gamma, axis)


def mhd_primitive(
    rho, mx, my, mz, energy, bz, az, dx, dy, b0x, b0y, gamma, prim, bxf, byf, ecc
) -> int:
    """Reference ``mhd_primitive``; writes prim/bxf/byf/ecc, returns the bad-cell count."""
    bxf[...] = (az[:, 1:] - az[:, :-1]) / dy + b0x
    byf[...] = -(az[1:, :] - az[:-1, :]) / dx + b0y
    bx = 0.5 * (bxf[:-1] + bxf[1:])
    by = 0.5 * (byf[:, :-1] + byf[:, 1:])
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        u = mx / rho
        v = my / rho
        w = mz / rho
        p = (gamma - 1.0) * (
            energy - 0.5 * rho * (u * u + v * v + w * w) - 0.5 * (bx * bx + by * by + bz * bz)
        )
        values = (rho, u, v, w, p, bx, by, bz)
        for row, value in enumerate(values):
            prim[row] = value
        ecc[...] = bx * v - by * u
        positive = (rho > 0.0) & (p > 0.0)
        finite = np.ones(rho.shape, dtype=bool)
        for value in values:
            finite &= np.abs(value) <= np.finfo(float).max
    return int(np.count_nonzero(~positive | ~finite))


def _upwind(mass, positive, negative):
    return np.where(
        mass > 0.0, positive, np.where(mass < 0.0, negative, 0.5 * (positive + negative))
    )


def ct_nodes(fx_by, gy_bx, fx_rho, gy_rho, ecc, na, nb):
    """CT-contact E at ``(na, nb)`` nodes, batched over leading axes.

    The last two axes are the block's (a, b) plane: ``fx_by``/``fx_rho`` at a-faces
    ``2 .. `` (index ``k`` is a-face ``k + 2``) and all b-cells, ``gy_bx``/``gy_rho`` at
    all a-cells and b-faces ``2 ..``, ``ecc`` the cell value; node ``(p, q)`` of the
    block is node ``(p + 2, q + 2)`` of the haloed block
    (``ct_contact_pyccel.py:36-61``).
    """

    def s(array, p, q):
        return array[..., p : p + na, q : q + nb]

    lower, upper = s(fx_by, 0, 1), s(fx_by, 0, 2)
    left, right = s(gy_bx, 1, 0), s(gy_bx, 2, 0)
    dl2 = _upwind(s(fx_rho, 0, 1), left - s(ecc, 1, 1), right - s(ecc, 2, 1))
    dr2 = _upwind(s(fx_rho, 0, 2), left - s(ecc, 1, 2), right - s(ecc, 2, 2))
    dl1 = _upwind(s(gy_rho, 1, 0), -lower - s(ecc, 1, 1), -upper - s(ecc, 1, 2))
    dr1 = _upwind(s(gy_rho, 2, 0), -lower - s(ecc, 2, 1), -upper - s(ecc, 2, 2))
    return 0.25 * (right + left - upper - lower + dl1 + dr1 + dl2 + dr2)


def ct_contact(fx_by, gy_bx, fx_rho, gy_rho, ecc, ez) -> None:
    """Reference ``ct_contact``: CT-contact E_z at the block's nodes, written to ``ez``."""
    ez[...] = ct_nodes(fx_by, gy_bx, fx_rho, gy_rho, ecc, *ez.shape)


def mhd_rate(rho, mx, my, mz, energy, bz, az, halo, dx, dy, b0x, b0y, gamma, out) -> None:
    """Reference ``mhd_rate``: ``out = [max (|u|+c_x)/dx + (|v|+c_y)/dy, min rho]``."""
    h = halo
    block = (slice(h, rho.shape[0] - h), slice(h, rho.shape[1] - h))
    nodes = az[h : az.shape[0] - h, h : az.shape[1] - h]
    bxf = (nodes[:, 1:] - nodes[:, :-1]) / dy + b0x
    byf = -(nodes[1:, :] - nodes[:-1, :]) / dx + b0y
    bx = 0.5 * (bxf[:-1] + bxf[1:])
    by = 0.5 * (byf[:, :-1] + byf[:, 1:])
    r = rho[block]
    u, v, w = mx[block] / r, my[block] / r, mz[block] / r
    b = bz[block]
    p = (gamma - 1.0) * (
        energy[block] - 0.5 * r * (u * u + v * v + w * w) - 0.5 * (bx * bx + by * by + b * b)
    )
    cx = fast_speed(r, p, bx, by, b, gamma)
    cy = fast_speed(r, p, by, bx, b, gamma)
    out[0] = np.max((np.abs(u) + cx) / dx + (np.abs(v) + cy) / dy)
    out[1] = np.min(r)


def mhd_resistive(prim, bxf, byf, dx, dy, eta, fx, fy, ez) -> None:
    """Reference ``mhd_resistive``: adds eta J terms to ``fx[4,6]``, ``fy[4,6]``, ``ez``."""
    h = 2
    nx = prim.shape[1] - 2 * h
    ny = prim.shape[2] - 2 * h
    jz = np.zeros((nx + 2 * h, ny + 2 * h))
    jz[1:, 1:] = (byf[1:, 1:-1] - byf[:-1, 1:-1]) / dx - (bxf[1:-1, 1:] - bxf[1:-1, :-1]) / dy
    i = np.arange(nx + 1)[:, None] + h
    j = np.arange(ny)[None, :] + h
    jy = -(prim[7, i, j] - prim[7, i - 1, j]) / dx
    bz_x = 0.5 * (prim[7, i, j] + prim[7, i - 1, j])
    by_x = 0.5 * (prim[6, i, j] + prim[6, i - 1, j])
    jz_x = 0.5 * (jz[i, j] + jz[i, j + 1])
    fx[6, :, h : h + ny] += eta * jy
    fx[4, :, h : h + ny] += eta * (jy * bz_x - jz_x * by_x)
    i = np.arange(nx)[:, None] + h
    j = np.arange(ny + 1)[None, :] + h
    jx = (prim[7, i, j] - prim[7, i, j - 1]) / dy
    bz_y = 0.5 * (prim[7, i, j] + prim[7, i, j - 1])
    bx_y = 0.5 * (prim[5, i, j] + prim[5, i, j - 1])
    jz_y = 0.5 * (jz[i, j] + jz[i + 1, j])
    fy[6, h : h + nx, :] += -eta * jx
    fy[4, h : h + nx, :] += eta * (jz_y * bx_y - jx * bz_y)
    ez += eta * jz[h : h + nx + 1, h : h + ny + 1]


def _mc(a, b):
    return limited_slope(a, b, 2)


def mhd_conductive(prim, bxf, byf, dx, dy, parallel, perpendicular, fx, fy) -> None:
    """Reference ``mhd_conductive``: subtracts the Braginskii heat flux from fx[4], fy[4]."""
    nx, ny = prim.shape[1], prim.shape[2]
    tiny = np.finfo(float).tiny
    t = prim[4] / prim[0]
    across = np.zeros((nx, ny))
    across[:, 1:-1] = _mc((t[:, 2:] - t[:, 1:-1]) / dy, (t[:, 1:-1] - t[:, :-2]) / dy)
    bn = bxf[2 : nx - 1, :]
    bt = 0.5 * (prim[6, 1 : nx - 2] + prim[6, 2 : nx - 1])
    bzf = 0.5 * (prim[7, 1 : nx - 2] + prim[7, 2 : nx - 1])
    magnitude = np.maximum(np.sqrt(bn * bn + bt * bt + bzf * bzf), tiny)
    b_n, b_t = bn / magnitude, bt / magnitude
    normal = (t[2 : nx - 1] - t[1 : nx - 2]) / dx
    transverse = _mc(across[1 : nx - 2], across[2 : nx - 1])
    fx[4] -= parallel * b_n * (b_n * normal + b_t * transverse) + perpendicular * normal
    across = np.zeros((nx, ny))
    across[1:-1, :] = _mc((t[2:, :] - t[1:-1, :]) / dx, (t[1:-1, :] - t[:-2, :]) / dx)
    bn = byf[:, 2 : ny - 1]
    bt = 0.5 * (prim[5, :, 1 : ny - 2] + prim[5, :, 2 : ny - 1])
    bzf = 0.5 * (prim[7, :, 1 : ny - 2] + prim[7, :, 2 : ny - 1])
    magnitude = np.maximum(np.sqrt(bn * bn + bt * bt + bzf * bzf), tiny)
    b_n, b_t = bn / magnitude, bt / magnitude
    normal = (t[:, 2 : ny - 1] - t[:, 1 : ny - 2]) / dy
    transverse = _mc(across[:, 1 : ny - 2], across[:, 2 : ny - 1])
    fy[4] -= parallel * b_n * (b_n * normal + b_t * transverse) + perpendicular * normal
