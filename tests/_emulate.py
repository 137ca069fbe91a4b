"""NumPy emulation of the halo / restriction op kernels (test infrastructure).

Applies `wellbalanced_b200.mesh.Layout` op lists to a host pool with the arithmetic of
``wellbalanced_b200/csrc/halo.cu``, so the host-side op generation can be checked on
the CPU against the oracle's exchange.
"""

from __future__ import annotations

import itertools

import numpy as np


PROXY = 1 << 30  # a dense block standing for a box of another rank's patch


def offset_of(row, i, j, k):
    """Element offset of haloed index (i, j, k); asserts it lies inside the padded field
    (for a proxy block, whose pitches are its box's, only the patch's haloed extents)."""
    n = [int(v) + 5 for v in row["n"]]
    if int(row["flags"]) & PROXY:
        assert 0 <= i < n[0] and 0 <= j < n[1] and (not row["pitch1"] or 0 <= k < n[2]), (i, j, k, n)
        if row["pitch1"]:
            return int(i) * int(row["pitch0"]) + int(j) * int(row["pitch1"]) + int(k)
        return int(i) * int(row["pitch0"]) + int(j)
    if row["pitch1"]:
        assert 0 <= i < n[0] and 0 <= j < n[1] and 0 <= k < n[2], (i, j, k, n)
        assert int(k) < int(row["pitch1"])
        return int(i) * int(row["pitch0"]) + int(j) * int(row["pitch1"]) + int(k)
    assert 0 <= i < n[0] and 0 <= j < n[1] and int(j) < int(row["pitch0"]), (i, j, n)
    return int(i) * int(row["pitch0"]) + int(j)


def apply_copy(pool, rows, ops):
    for op in ops:
        D, A = rows[op["dst"]], rows[op["src1"]]
        B = rows[op["src2"] if op["src2"] >= 0 else op["src1"]]
        n = op["n"]
        writes = []
        for p in itertools.product(range(n[0]), range(n[1]), range(n[2])):
            od = offset_of(D, *(op["d"][a] + p[a] for a in range(3)))
            o1 = offset_of(A, *(op["s1"][a] + op["m1"][a] * p[a] for a in range(3)))
            o2 = offset_of(B, *(op["s2"][a] + op["m2"][a] * p[a] for a in range(3)))
            for f in range(op["field_lo"], op["field_hi"]):
                v = op["w1"] * pool[A["off"] + f * A["fstride"] + o1]
                if op["w2"] != 0.0:
                    v += op["w2"] * pool[B["off"] + f * B["fstride"] + o2]
                if f == op["negate"]:
                    v = -v
                writes.append((D["off"] + f * D["fstride"] + od, v))
        for index, value in writes:
            pool[index] = value


def _weights(node, g):
    if node:
        if g % 2 == 0:
            return g // 2, [1.0]
        return g // 2 - 1, [-1 / 16, 9 / 16, 9 / 16, -1 / 16]
    c = g // 2
    if g % 2 == 0:
        return c - 1, [0.25, 0.75]
    return c, [0.75, 0.25]


def apply_interp(pool, rows, ops):
    for op in ops:
        F, C = rows[op["fine"]], rows[op["coarse"]]
        ndim = int(op["ndim"])
        n = op["n"]
        for q in itertools.product(range(n[0]), range(n[1]), range(n[2])):
            fi = [op["d"][a] + q[a] for a in range(3)]
            starts, weights = [], []
            for a in range(3):
                if a >= ndim:
                    starts.append(0)
                    weights.append([1.0])
                    continue
                g = fi[a] - 2 + op["fine_lo"][a]
                c0, w = _weights((op["node_mask"] >> a) & 1, g)
                starts.append(c0 - op["coarse_lo"][a] + 2)
                weights.append(w)
            od = offset_of(F, fi[0], fi[1], fi[2] if ndim == 3 else 0)
            for f in range(op["field_lo"], op["field_hi"]):
                acc = 0.0
                for a0, w0 in enumerate(weights[0]):
                    for a1, w1 in enumerate(weights[1]):
                        for a2, w2 in enumerate(weights[2]):
                            oc = offset_of(C, starts[0] + a0, starts[1] + a1, starts[2] + a2 if ndim == 3 else 0)
                            acc += w0 * w1 * w2 * pool[C["off"] + f * C["fstride"] + oc]
                pool[F["off"] + f * F["fstride"] + od] = acc


def apply_restrict(pool, rows, ops):
    for op in ops:
        F, C = rows[op["fine"]], rows[op["coarse"]]
        ndim = int(op["ndim"])
        cnt = [2 if (a < ndim and not (op["node_mask"] >> a) & 1) else 1 for a in range(3)]
        n = op["n"]
        for q in itertools.product(range(n[0]), range(n[1]), range(n[2])):
            ci = [op["c"][a] + q[a] for a in range(3)]
            fi = [op["f"][a] + 2 * q[a] for a in range(3)]
            oc = offset_of(C, ci[0], ci[1], ci[2] if ndim == 3 else 0)
            for f in range(op["field_lo"], op["field_hi"]):
                acc = 0.0
                for a0 in range(cnt[0]):
                    for a1 in range(cnt[1]):
                        for a2 in range(cnt[2]):
                            of = offset_of(F, fi[0] + a0, fi[1] + a1, fi[2] + a2 if ndim == 3 else 0)
                            acc += pool[F["off"] + f * F["fstride"] + of]
                total = cnt[0] * cnt[1] * cnt[2]
                pool[C["off"] + f * C["fstride"] + oc] = acc if total == 1 else acc * (1.0 / total)


def fill(pool, layout):
    """The device fill sequence of `Engine.fill` on a host pool."""
    for level, (same, boundary) in enumerate(layout.copy_phases):
        apply_interp(pool, layout.rows, layout.interp_levels[level])
        apply_copy(pool, layout.rows, same)
        for ops in boundary:
            apply_copy(pool, layout.rows, ops)


def view(pool, layout, patch, field):
    return layout.patch_view(pool, patch, field)
