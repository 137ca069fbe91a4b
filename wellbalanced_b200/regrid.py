"""Regridding: clustering tagged cells into patches and moving the state onto them.

The reference delegates this to patchwork (``AMRHierarchy.regrid``, absent here;
``carafe/mhd.py:1043-1056``, ``carafe/mhd3d.py:803-816``): "the conserved fields keep their
integrals, A_z is interpolated ... so the field stays divergence-free". Restated here:

* `cluster_tags` — the tagged cells of a level, grown by ``buffer`` cells, restricted to
  where a finer patch can nest (one cell inside the level's patches), are covered by
  boxes by recursive bisection (Berger–Rigoutsos: cut at a hole of the tag signature,
  else at its strongest inflection, else across the middle of the longest side) until
  each box is at least 70% tagged and at most ``max_size`` cells per side;
* `transfer` — the new hierarchy's level values: where the old hierarchy had a patch on
  that level its values are kept (on a periodic axis the duplicate node planes take the
  kept value from either side, so they agree), elsewhere they are prolongated from the
  new coarser level — cells by minmod-limited linear reconstruction (children c ± s/4 per axis, so
  the mean of the children is the coarse value: integrals kept, no new extrema), the
  potential linearly along node axes and constant along an edge's own axis (so the
  restriction that follows leaves the coarse potential, hence the coarse field,
  unchanged).
"""

from __future__ import annotations

import itertools

import numpy as np

from wellbalanced_b200 import _lib
from wellbalanced_b200.mesh import HALO


def _grow(mask, buffer, periodic):
    out = mask.copy()
    for a in range(mask.ndim):
        grown = out.copy()
        for k in range(1, buffer + 1):
            for sign in (-1, 1):
                if periodic[a]:
                    grown |= np.roll(out, sign * k, axis=a)
                else:
                    shifted = np.zeros_like(out)
                    src = [slice(None)] * mask.ndim
                    dst = [slice(None)] * mask.ndim
                    if sign > 0:
                        src[a], dst[a] = slice(0, -k), slice(k, None)
                    else:
                        src[a], dst[a] = slice(k, None), slice(0, -k)
                    shifted[tuple(dst)] = out[tuple(src)]
                    grown |= shifted
        out = grown
    return out


def nesting_mask(shape, parents, periodic, margin=1):
    """Cells of a level where a finer patch may lie: inside its patches by ``margin`` cells
    (the domain boundary needs no margin)."""
    covered = np.zeros(shape, dtype=bool)
    for box in parents:
        covered[tuple(slice(lo, hi) for lo, hi in box)] = True
    outside = ~covered
    # cells within `margin` of an uncovered cell are excluded
    near = _grow(outside, margin, periodic)
    return covered & ~near


def _signature_cut(sub, axis):
    sig = sub.sum(axis=tuple(b for b in range(sub.ndim) if b != axis))
    n = sig.size
    for k in range(1, n - 1):  # a hole: no tag in a whole slab
        if sig[k] == 0:
            return k
    if n >= 4:
        lap = sig[:-2] - 2 * sig[1:-1] + sig[2:]
        best, where = 0, None
        for k in range(1, lap.size):
            if lap[k - 1] * lap[k] < 0:
                jump = abs(lap[k] - lap[k - 1])
                if jump > best:
                    best, where = jump, k + 1
        if where is not None and 2 <= where <= n - 2:
            return where
    return None


def cluster_tags(tags, *, buffer=1, max_size=None, min_size=4, parents=None, periodic=None, efficiency=0.7):
    """Disjoint boxes ``((lo, hi), ...)`` of the level covering every grown, nestable tagged
    cell (the tags grown by ``buffer`` cells, within the parents by the nesting margin).

    Recursive bisection (Berger-Rigoutsos): a box is kept when it is at most ``max_size``
    cells a side, its tagged fraction reaches ``efficiency`` and it lies in the nestable
    region; else it is cut at a hole or an inflection of its tag signature, or halved,
    down to single cells if need be. Boxes are then grown towards ``min_size`` (the
    smallest side in cells of the REFINED level: ``ceil(min_size / 2)`` cells of this
    level) into nestable cells no other box holds, where there is room; coverage of the
    tags comes first, so a box without room keeps its smaller side.
    """
    tags = np.asarray(tags, dtype=bool)
    ndim = tags.ndim
    periodic = periodic or (False,) * ndim
    parents = parents or [tuple((0, n) for n in tags.shape)]
    grown = _grow(tags, buffer, periodic) if buffer else tags.copy()
    allowed = nesting_mask(tags.shape, parents, periodic, margin=1)
    grown &= allowed
    min_side = max(2, (min_size + 1) // 2)
    max_side = max(1, max_size or max(tags.shape))
    boxes = []

    def shrink(box):
        sub = grown[tuple(slice(lo, hi) for lo, hi in box)]
        if not sub.any():
            return None
        out = []
        for a in range(ndim):
            along = sub.any(axis=tuple(b for b in range(ndim) if b != a))
            idx = np.flatnonzero(along)
            out.append((box[a][0] + int(idx[0]), box[a][0] + int(idx[-1]) + 1))
        return tuple(out)

    def split(box):
        box = shrink(box)
        if box is None:
            return
        sub = grown[tuple(slice(lo, hi) for lo, hi in box)]
        sides = [hi - lo for lo, hi in box]
        fits = all(side <= max_side for side in sides)
        nestable = allowed[tuple(slice(lo, hi) for lo, hi in box)].all()
        small = max(sides) <= min_side
        if fits and nestable and (small or sub.mean() >= efficiency):
            boxes.append(box)
            return
        order = sorted(range(ndim), key=lambda a: -sides[a])
        axis = cut = None
        for a in order:
            if sides[a] < 2 * min_side:
                continue
            c = _signature_cut(sub, a)
            if c is not None and min_side <= c <= sides[a] - min_side:
                axis, cut = a, c
                break
        if axis is None:
            axis = order[0]
            cut = sides[axis] // 2  # >= 1: a box with a side of 1 everywhere is one cell, kept above
        lo, hi = box[axis]
        split(tuple((lo, lo + cut) if b == axis else box[b] for b in range(ndim)))
        split(tuple((lo + cut, hi) if b == axis else box[b] for b in range(ndim)))

    split(tuple((0, n) for n in tags.shape))
    # grow the boxes towards the smallest side through free, nestable cells
    held = np.zeros(tags.shape, dtype=bool)
    for box in boxes:
        held[tuple(slice(lo, hi) for lo, hi in box)] = True
    out = []
    for box in boxes:
        box = list(box)
        for a in range(ndim):
            for _ in range(2 * min_side):
                lo, hi = box[a]
                if hi - lo >= min_side:
                    break
                grew = False
                for new_lo, new_hi, slab in ((lo, hi + 1, (hi, hi + 1)), (lo - 1, hi, (lo - 1, lo))):
                    if slab[0] < 0 or slab[1] > tags.shape[a]:
                        continue
                    region = tuple(slice(*slab) if b == a else slice(*box[b]) for b in range(ndim))
                    if held[region].any() or not allowed[region].all():
                        continue
                    held[region] = True
                    box[a] = (new_lo, new_hi)
                    grew = True
                    break
                if not grew:
                    break
        out.append(tuple(box))
    return out


def _overlap(a, b):
    return all(alo < bhi and blo < ahi for (alo, ahi), (blo, bhi) in zip(a, b, strict=True))


# ---- state transfer ------------------------------------------------------------------------
def _minmod(a, b):
    return np.where(a * b > 0.0, np.where(np.abs(a) < np.abs(b), a, b), 0.0)


def prolong_cells(coarse, periodic):
    """Children of every coarse cell: c + sum_a s_a (+-1/4), s_a minmod-limited slopes."""
    ndim = coarse.ndim
    padded = np.pad(coarse, 1, mode="wrap") if all(periodic) else coarse
    if not all(periodic):
        modes = [(1, 1)] * ndim
        padded = coarse
        for a in range(ndim):
            padded = np.pad(padded, [(1, 1) if b == a else (0, 0) for b in range(ndim)],
                            mode="wrap" if periodic[a] else "edge")
        del modes
    inner = tuple(slice(1, -1) for _ in range(ndim))
    centre = padded[inner]
    slopes = []
    for a in range(ndim):
        lo = [slice(1, -1)] * ndim
        hi = [slice(1, -1)] * ndim
        lo[a] = slice(0, -2)
        hi[a] = slice(2, None)
        slopes.append(_minmod(centre - padded[tuple(lo)], padded[tuple(hi)] - centre))
    fine = np.empty(tuple(2 * n for n in coarse.shape))
    for offsets in itertools.product((0, 1), repeat=ndim):
        value = centre.copy()
        for a, o in enumerate(offsets):
            value = value + slopes[a] * (0.25 if o else -0.25)
        fine[tuple(slice(o, None, 2) for o in offsets)] = value
    return fine


def prolong_potential(coarse, node_axes):
    """Fine potential from coarse: linear along node axes (coincident nodes exact,
    midpoints averaged), constant along cell axes (an edge's own direction)."""
    out = coarse
    for a, node in enumerate(node_axes):
        n = out.shape[a]
        if node:
            shape = list(out.shape)
            shape[a] = 2 * (n - 1) + 1
            fine = np.empty(shape)
            even = [slice(None)] * out.ndim
            even[a] = slice(0, None, 2)
            fine[tuple(even)] = out
            odd = [slice(None)] * out.ndim
            odd[a] = slice(1, None, 2)
            lo = np.take(out, np.arange(0, n - 1), axis=a)
            hi = np.take(out, np.arange(1, n), axis=a)
            fine[tuple(odd)] = 0.5 * (lo + hi)
        else:
            fine = np.repeat(out, 2, axis=a)
        out = fine
    return out


def _merge_periodic_planes(values, mask, extra, periodic, shape):
    """On a periodic axis a node array's last plane duplicates its first: take the kept
    (old-patch) value from either plane, so both planes agree after the transfer."""
    for a, (node, wraps) in enumerate(zip(extra, periodic, strict=True)):
        if not (node and wraps):
            continue
        first = [slice(None)] * values.ndim
        last = [slice(None)] * values.ndim
        first[a], last[a] = 0, shape[a]
        first, last = tuple(first), tuple(last)
        take = mask[last] & ~mask[first]
        values[first] = np.where(take, values[last], values[first])
        mask[first] |= mask[last]
        values[last] = values[first]
        mask[last] = mask[first]


def _cell_field(arrays, ndim, spacing, mean_field):
    """Cell-centred field of a level's dense arrays: the mean of each cell's two faces,
    every face the curl of the potential plus the mean field (2D: B_z the cell field);
    operation by operation as the device (csrc/transfer.cu cell_field)."""
    if ndim == 2:
        A = arrays[6]
        dx, dy = spacing
        fx = np.diff(A, axis=1) / dy + mean_field[0]
        fy = -np.diff(A, axis=0) / dx + mean_field[1]
        return 0.5 * (fx[:-1] + fx[1:]), 0.5 * (fy[:, :-1] + fy[:, 1:]), arrays[5]
    ax, ay, az = arrays[5], arrays[6], arrays[7]
    dx, dy, dz = spacing
    fx = (np.diff(az, axis=1) / dy - np.diff(ay, axis=2) / dz) + mean_field[0]
    fy = (np.diff(ax, axis=2) / dz - np.diff(az, axis=0) / dx) + mean_field[1]
    fz = (np.diff(ay, axis=0) / dx - np.diff(ax, axis=1) / dy) + mean_field[2]
    return 0.5 * (fx[:-1] + fx[1:]), 0.5 * (fy[:, :-1] + fy[:, 1:]), 0.5 * (fz[:, :, :-1] + fz[:, :, 1:])


def _kinetic(r, m0, m1, m2):
    return (0.5 * ((m0 * m0 + m1 * m1) + m2 * m2)) / r


def _magnetic(b):
    return 0.5 * ((b[0] * b[0] + b[1] * b[1]) + b[2] * b[2])


#: a prolonged child below this fraction of its parent's pressure counts as collapsed
#: (csrc/transfer.cu kPressureFraction)
PRESSURE_FRACTION = 0.25


def positivity_fix(fine, coarse, ndim, spacing_fine, spacing_coarse, gamma, mean_field):
    """The positivity pass of the transfer on a level's dense arrays (``fine``, fields as
    the pool's; ``coarse`` the level below), in place: every valid parent whose children
    include a non-positive density or a pressure below ``PRESSURE_FRACTION`` times its own
    gives them its density, momentum (2D: B_z) and the energy E + M_i - mean(M) while
    (gamma - 1)(E - K - mean(M)) is above that fraction of its pressure p, else
    p / (gamma - 1) + K + M_i (M_i a child's magnetic energy from the fine potential;
    ``csrc/transfer.cu`` positivity_ops_kernel, operation by operation). Returns the count
    of parents changed."""
    gm1 = gamma - 1.0
    offsets = list(itertools.product((0, 1), repeat=ndim))

    def child(a, o):
        return a[tuple(slice(x, None, 2) for x in o)]

    bc = _cell_field(coarse, ndim, spacing_coarse, mean_field)
    k = _kinetic(coarse[0], coarse[1], coarse[2], coarse[3])
    pc = gm1 * ((coarse[4] - k) - _magnetic(bc))
    low = PRESSURE_FRACTION * pc
    bf = _cell_field(fine, ndim, spacing_fine, mean_field)
    bad = np.zeros(coarse[0].shape, dtype=bool)
    for o in offsets:
        r = child(fine[0], o)
        kc = _kinetic(r, child(fine[1], o), child(fine[2], o), child(fine[3], o))
        p = gm1 * ((child(fine[4], o) - kc) - _magnetic([child(b, o) for b in bf]))
        with np.errstate(invalid="ignore"):
            bad |= ~((r > 0.0) & (p > low) & np.isfinite(p))
    fix = bad & (coarse[0] > 0.0) & (pc > 0.0)
    if not fix.any():
        return 0
    mags = []
    total = np.zeros(coarse[0].shape)
    for o in offsets:
        b = [child(x, o) for x in bf]
        if ndim == 2:
            b[2] = coarse[5]
        mags.append(_magnetic(b))
        total = total + mags[-1]
    mean = total / float(len(offsets))
    keep = gm1 * ((coarse[4] - k) - mean) > low
    floor = pc / gm1 + k
    for o, mag in zip(offsets, mags, strict=True):
        energy = np.where(keep, coarse[4] + (mag - mean), floor + mag)
        for f in range(4):
            child(fine[f], o)[fix] = coarse[f][fix]
        child(fine[4], o)[fix] = energy[fix]
        if ndim == 2:
            child(fine[5], o)[fix] = coarse[5][fix]
    return int(fix.sum())


def _rounded(values, dtype):
    """Values as the state holds them (float32 states round)."""
    return values.astype(np.float32).astype(np.float64) if dtype == np.float32 else values


def regrid_model_host(model, tags, **options):
    """Regrid ``model`` (an `MHD2D` / `MHD3D`) on ``tags`` with the transfer restated on the
    host, level by level on dense arrays (the state goes to the host and back). The
    solvers regrid with `regrid_model` (the transfer on the device); this restatement is
    what the tests check the device transfer against."""
    import torch

    model._check_ready()
    old_h = model.hierarchy
    extras = model._field_extras()
    periodic = old_h.periodic
    old_levels = {}
    for level in range(old_h.max_level + 1):
        shape = old_h.level_shape(level)
        arrays = []
        for f, extra in enumerate(extras):
            size = tuple(n + e for n, e in zip(shape, extra, strict=True))
            values = np.zeros(size)
            mask = np.zeros(size, dtype=bool)
            for p in old_h.patches_at_level(level):
                index = tuple(slice(lo, hi + e) for (lo, hi), e in zip(p.box, extra, strict=True))
                values[index] = model._gather_field(p, f)
                mask[index] = True
            _merge_periodic_planes(values, mask, extra, periodic, shape)
            arrays.append((values, mask))
        old_levels[level] = arrays
    new_h = old_h.regrid(tags, **options)
    time, steps = model.time, model.steps
    model.hierarchy = new_h
    model._build_engine()
    dtype = np.float32 if model.engine.state.dtype == torch.float32 else np.float64
    new_levels = {}
    for level in range(new_h.max_level + 1):
        arrays = []
        for f, extra in enumerate(extras):
            old = old_levels.get(level)
            if level == 0:
                result = old[f][0]
            else:
                coarse = new_levels[level - 1][f]
                fine = prolong_potential(coarse, extra) if any(extra) else prolong_cells(coarse, periodic)
                result = _rounded(fine if old is None else np.where(old[f][1], old[f][0], fine), dtype)
            arrays.append(result)
        if level:
            positivity_fix(arrays, new_levels[level - 1], new_h.ndim, new_h.spacing(level), new_h.spacing(level - 1),
                           model.gamma, model.engine.mean_field)
            arrays[4] = _rounded(arrays[4], dtype)
        for f, extra in enumerate(extras):
            for p in new_h.patches_at_level(level):
                index = tuple(slice(lo, hi + e) for (lo, hi), e in zip(p.box, extra, strict=True))
                model._write_field(p, f, arrays[f][index])
        new_levels[level] = arrays
    model._after_state(tune=False)
    model.time, model.steps = time, steps
    model.engine.time.fill_(time)


# ---- the transfer on the device ------------------------------------------------------------
#: mirror of the device prolongation op (wellbalanced_b200/csrc/transfer.cu ProlongOp)
PROLONG_OP = np.dtype(
    {
        "names": ["fine", "coarse", "field_lo", "field_hi", "node_mask", "ndim", "n", "d", "fine_lo", "coarse_lo",
                  "coarse_n", "periodic"],
        "formats": ["<i4"] * 6 + [("<i4", 3)] * 5 + ["<i4"],
        "itemsize": 88,
    }
)

#: points per transfer op (one 128-thread block each)
TRANSFER_OP_POINTS = 4096

#: mirror of the device positivity op (csrc/transfer.cu PositivityOp)
POSITIVITY_OP = np.dtype({"names": ["fine", "coarse", "ndim", "pad", "n", "f0", "c0"],
                          "formats": ["<i4"] * 4 + [("<i4", 3)] * 3, "itemsize": 52})

#: parents per positivity op
POSITIVITY_OP_PARENTS = 1024


def _ranges(patches, node_mask, ndim):
    """(lo, hi) level index ranges of the patches' points of a field group: cells, and one
    node more along node axes; arrays (patches, ndim)."""
    lo = np.array([[p.box[a][0] for a in range(ndim)] for p in patches], dtype=np.int64).reshape(-1, ndim)
    hi = np.array([[p.box[a][1] + ((node_mask >> a) & 1) for a in range(ndim)] for p in patches],
                  dtype=np.int64).reshape(-1, ndim)
    return lo, hi


def _cut(n, chunk=TRANSFER_OP_POINTS):
    """Sub-boxes (offset, extent) of a box of extents n (3 axes, the last fastest) of at
    most `chunk` points: whole planes or rows where they fit."""
    inner = int(n[1]) * int(n[2])
    if inner <= chunk:
        step = max(1, chunk // max(1, inner))
        return [((a, 0, 0), (min(step, int(n[0]) - a), int(n[1]), int(n[2]))) for a in range(0, int(n[0]), step)]
    step = max(1, chunk // max(1, int(n[2])))
    return [((a, b, 0), (1, min(step, int(n[1]) - b), int(n[2]))) for a in range(int(n[0]))
            for b in range(0, int(n[1]), step)]


def _pad3(v, fill=0):
    v = [int(x) for x in v]
    return v + [fill] * (3 - len(v))


def transfer_ops(old_h, new_h, groups, ndim):
    """Per level of the new hierarchy: (prolongation ops from the new coarser level,
    kept-value ops from the old hierarchy's patches of that level, periodic images
    included, positivity ops over the parents of the level's cells)."""
    periodic = new_h.periodic
    pmask = sum(1 << a for a in range(ndim) if periodic[a])
    out = []
    for level in range(new_h.max_level + 1):
        shape = new_h.level_shape(level)
        prolong, kept = [], []
        fines = new_h.patches_at_level(level)
        olds = old_h.patches_at_level(level) if level <= old_h.max_level else []
        coarses = new_h.patches_at_level(level - 1) if level else []
        shifts = list(itertools.product(*[(-shape[a], 0, shape[a]) if periodic[a] else (0,) for a in range(ndim)]))
        for g in groups:
            flo, fhi = _ranges(fines, g.node_mask, ndim)
            if olds:
                olo, ohi = _ranges(olds, g.node_mask, ndim)
                for sh in shifts:
                    sh = np.array(sh, dtype=np.int64)
                    lo = np.maximum(flo[:, None, :], olo[None, :, :] + sh)
                    hi = np.minimum(fhi[:, None, :], ohi[None, :, :] + sh)
                    for i, j in zip(*np.nonzero(np.all(hi > lo, axis=2)), strict=True):
                        n = _pad3(hi[i, j] - lo[i, j], 1)
                        for off, ext in _cut(n):
                            d = _pad3(lo[i, j] - flo[i] + HALO)
                            s = _pad3(lo[i, j] - (olo[j] + sh) + HALO)
                            kept.append((fines[i].index, olds[j].index, g.lo, g.hi,
                                         [d[a] + off[a] for a in range(3)], [s[a] + off[a] for a in range(3)], ext))
            if coarses:
                clo = np.array([[c.box[a][0] for a in range(ndim)] for c in coarses], dtype=np.int64)
                chi = np.array([[c.box[a][1] for a in range(ndim)] for c in coarses], dtype=np.int64)
                node = np.array([(g.node_mask >> a) & 1 for a in range(ndim)], dtype=np.int64)
                # fine points whose coarse stencil (the parent cell; the two nodes along a node
                # axis) lies in the coarse patch
                lo = np.maximum(flo[:, None, :], 2 * clo[None, :, :])
                hi = np.minimum(fhi[:, None, :], 2 * chi[None, :, :] + node)
                coarse_n = _pad3(new_h.level_shape(level - 1), 1)
                for i, j in zip(*np.nonzero(np.all(hi > lo, axis=2)), strict=True):
                    n = _pad3(hi[i, j] - lo[i, j], 1)
                    d0 = _pad3(lo[i, j] - flo[i] + HALO)
                    for off, ext in _cut(n):
                        prolong.append((fines[i].index, coarses[j].index, g.lo, g.hi, g.node_mask, ndim, ext,
                                        [d0[a] + off[a] for a in range(3)], _pad3(flo[i]), _pad3(clo[j]), coarse_n,
                                        pmask))
        positivity = []
        if coarses:
            # the parents of each new fine patch's cells over each coarse patch (cell ranges
            # are even, so every parent's children lie in one fine patch)
            flo, fhi = _ranges(fines, 0, ndim)
            clo = np.array([[c.box[a][0] for a in range(ndim)] for c in coarses], dtype=np.int64)
            chi = np.array([[c.box[a][1] for a in range(ndim)] for c in coarses], dtype=np.int64)
            lo = np.maximum(flo[:, None, :], 2 * clo[None, :, :])
            hi = np.minimum(fhi[:, None, :], 2 * chi[None, :, :])
            for i, j in zip(*np.nonzero(np.all(hi > lo, axis=2)), strict=True):
                n = _pad3((hi[i, j] - lo[i, j]) // 2, 1)
                f0 = _pad3(lo[i, j] - flo[i] + HALO)
                c0 = _pad3(lo[i, j] // 2 - clo[j] + HALO)
                for off, ext in _cut(n, POSITIVITY_OP_PARENTS):
                    positivity.append((fines[i].index, coarses[j].index, ndim, 0, ext,
                                       [f0[a] + 2 * off[a] if a < ndim else 0 for a in range(3)],
                                       [c0[a] + off[a] if a < ndim else 0 for a in range(3)]))
        p = np.zeros(len(prolong), PROLONG_OP)
        for k, r in enumerate(prolong):
            p[k] = r
        k_ops = np.zeros(len(kept), _lib.COPY_OP)
        for k, (dst, src, lo_f, hi_f, d, s, ext) in enumerate(kept):
            k_ops[k] = (dst, src, -1, lo_f, hi_f, -1, ext, d, s, (1, 1, 1), (0, 0, 0), (0, 0, 0), 1.0, 0.0)
        q_ops = np.zeros(len(positivity), POSITIVITY_OP)
        for k, r in enumerate(positivity):
            q_ops[k] = r
        out.append((p, k_ops, q_ops))
    return out


def regrid_model_device(model, tags, **options):
    """Regrid ``model`` on ``tags`` with the state moved on the device: the clustering on the
    host (from the tags), the transfer by the prolongation and kept-value kernels level by
    level, the new levels' halos filled between them; no state round trip to the host."""
    import torch

    from wellbalanced_b200.engine import _device_bytes

    model._check_ready()
    old_h, old_engine = model.hierarchy, model.engine
    new_h = old_h.regrid(tags, **options)
    time, steps = model.time, model.steps
    model.hierarchy = new_h
    model._build_engine()
    eng = model.engine
    stream = eng._s()
    for level, (prolong, kept, positivity) in enumerate(transfer_ops(old_h, new_h, eng.layout.groups, eng.ndim)):
        if prolong.size:
            ops = _device_bytes(prolong, eng.device, PROLONG_OP)
            _lib.call("wb_prolong_ops", eng.precision, eng.state.data_ptr(), eng.patches.data_ptr(), ops.data_ptr(),
                      int(prolong.size), stream)
        if kept.size:
            ops = _device_bytes(kept, eng.device, _lib.COPY_OP)
            _lib.call("wb_kept_ops", eng.precision, eng.state.data_ptr(), eng.patches.data_ptr(),
                      old_engine.state.data_ptr(), old_engine.patches.data_ptr(), ops.data_ptr(), int(kept.size),
                      stream)
        if positivity.size:
            ops = _device_bytes(positivity, eng.device, POSITIVITY_OP)
            b = eng.mean_field
            _lib.call("wb_positivity_ops", eng.precision, eng.state.data_ptr(), eng.patches.data_ptr(), ops.data_ptr(),
                      int(positivity.size), b[0], b[1], b[2], float(model.gamma), stream)
        eng.fill(eng.state, levels={level})
    torch.cuda.current_stream(eng.device).synchronize()
    del old_engine
    model._after_state(tune=False)
    model.time, model.steps = time, steps
    eng.time.fill_(time)


def regrid_model(model, tags, **options):
    """Regrid ``model`` on ``tags``: clustering on the host, the state moved on the device."""
    regrid_model_device(model, tags, **options)


# ---- the plain tagger on the device ---------------------------------------------------------
#: where a patch's cells go in the levels' tag arrays (TagPlace in csrc/tags.cu)
TAG_PLACE = np.dtype({"names": ["base", "s0", "s1"], "formats": ["<i8", "<i8", "<i8"], "itemsize": 24})


def device_tags(model, threshold, levels):
    """``current_tags`` by one kernel over every cell of the tagged levels (|J| dx >
    threshold), written into the levels' dense arrays on the device and read back once."""
    import torch

    from wellbalanced_b200.engine import _device_bytes

    model._check_ready()
    h, eng = model.hierarchy, model.engine
    nlev = min(levels, h.max_level + 1)
    shapes = [tuple(h.level_shape(level)) for level in range(nlev)]
    sizes = [int(np.prod(s)) for s in shapes]
    offsets = np.cumsum([0, *sizes])
    place = np.zeros(len(h.patches), TAG_PLACE)
    for p in h.patches:
        if p.level >= nlev:
            continue
        shape = shapes[p.level]
        lo = [b[0] for b in p.box]
        if h.ndim == 2:
            place[p.index] = (offsets[p.level] + lo[0] * shape[1] + lo[1], shape[1], 0)
        else:
            s0, s1 = shape[1] * shape[2], shape[2]
            place[p.index] = (offsets[p.level] + lo[0] * s0 + lo[1] * s1 + lo[2], s0, s1)
    out = torch.zeros(max(int(offsets[-1]), 1), dtype=torch.uint8, device=eng.device)
    if nlev and eng.nchunks:
        b = eng.mean_field
        _lib.call("wb_current_tags", eng.precision, h.ndim, eng.state.data_ptr(), eng.patches.data_ptr(),
                  eng.chunk_patch.data_ptr(), eng.chunk_start.data_ptr(), eng.nchunks,
                  _device_bytes(place, eng.device, TAG_PLACE).data_ptr(), nlev, b[0], b[1], b[2], float(threshold),
                  out.data_ptr(), eng._s())
    host = out.cpu().numpy()
    return {level: host[offsets[level]:offsets[level + 1]].reshape(shapes[level]).astype(bool)
            for level in range(nlev)}
