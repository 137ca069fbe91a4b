"""The patch hierarchy on the device: layout of the state pools and the op lists.

`AMRHierarchy` is the mesh API the solvers use, the part of patchwork's
(``patchwork-amr`` 0.2.0, absent here) that ``carafe.mhd`` calls: levels refined by 2,
each a list of patches with boxes in level indices, periodic axes, spacing, and
``regrid``. `Layout` turns a hierarchy and a field set into what the kernels need:

* a pool layout: every patch's fields with a halo of two, one padded node-shaped array
  per field (``PatchDesc`` rows);
* the work lists of the fused stage kernels (tiles) and of the rate kernel (chunks);
* op lists that replace patchwork's ``exchange_halos`` (copies from same-level patches
  and periodic images, coarse-to-fine interpolation, outflow / wall faces) and
  ``restrict``, and the flux-register ops of refluxing.

Node ownership: a patch computes the nodes ``[lo, hi)`` of each axis, and its upper node
plane too unless same-level patches (or its own periodic image) provide the whole plane;
every other point of its haloed arrays is filled by the op lists.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

from wellbalanced_b200 import _lib

HALO = 2


@dataclass
class Patch:
    level: int
    box: tuple  # ((lo, hi), ...) in level cell indices
    index: int = -1
    is_local: bool = True
    ranks: list = field(default_factory=lambda: [0])

    @property
    def shape(self):
        return tuple(hi - lo for lo, hi in self.box)


class AMRHierarchy:
    """Levels of patches over a Cartesian box (refinement ratio 2).

    Args mirror the patchwork constructor the reference calls
    (``AMRHierarchy(shape, bounds, periodic=..., comm=..., placement=...)``); ``split``
    cuts the base level into that many patches per axis.
    """

    refinement_ratio = 2

    def __init__(self, shape, bounds=None, periodic=None, *, comm=None, placement="all", geometry="cartesian",
                 split=None):
        self.shape = tuple(int(n) for n in shape)
        self.ndim = len(self.shape)
        if self.ndim not in (1, 2, 3):
            raise ValueError("a hierarchy has 1 to 3 axes")
        bounds = bounds or ((0.0, 1.0),) * self.ndim
        self.bounds = tuple((float(lo), float(hi)) for lo, hi in bounds)
        self.lower_bound = tuple(lo for lo, _ in self.bounds)
        self.periodic = tuple(bool(p) for p in (periodic or (False,) * self.ndim))
        self.cylindrical = geometry == "cylindrical"
        self.graded = False
        self.comm = comm
        self.placement = placement
        self.patches: list[Patch] = []
        split = split or (1,) * self.ndim
        cuts = [np.linspace(0, n, s + 1).round().astype(int) for n, s in zip(self.shape, split, strict=True)]
        for index in itertools.product(*(range(s) for s in split)):
            box = tuple((int(c[k]), int(c[k + 1])) for c, k in zip(cuts, index, strict=True))
            self._append(Patch(0, box))

    def _append(self, patch):
        patch.index = len(self.patches)
        self.patches.append(patch)
        return patch

    @property
    def max_level(self):
        return max(p.level for p in self.patches)

    @property
    def local_patches(self):
        return self.patches

    def level_shape(self, level):
        return tuple(n * 2**level for n in self.shape)

    def spacing(self, level):
        return tuple((hi - lo) / n for (lo, hi), n in zip(self.bounds, self.level_shape(level), strict=True))

    def patches_at_level(self, level):
        # grouped once per state of the patch list (patches are only appended; a new list
        # object or a new length regroups)
        key = (id(self.patches), len(self.patches))
        if getattr(self, "_by_level_key", None) != key:
            grouped = {}
            for p in self.patches:
                grouped.setdefault(p.level, []).append(p)
            self._by_level, self._by_level_key = grouped, key
        return list(self._by_level.get(level, ()))

    def add_patch(self, level, box):
        """A patch on ``level`` (>= 1) over ``box``, aligned to the coarse cells."""
        box = tuple((int(lo), int(hi)) for lo, hi in box)
        if level < 1 or level > self.max_level + 1:
            raise ValueError("patches are added one level above an existing one")
        shape = self.level_shape(level)
        for (lo, hi), n in zip(box, shape, strict=True):
            if not 0 <= lo < hi <= n:
                raise ValueError(f"box {box} is outside level {level} of shape {shape}")
            if lo % 2 or hi % 2:
                raise ValueError(f"box {box} is not aligned to the cells of level {level - 1}")
            if hi - lo < 4:
                raise ValueError("a refined patch needs at least 4 cells per axis")
        return self._append(Patch(level, box))

    def regrid(self, tags, *, max_patch_size=None, buffer=1, min_patch_size=4):
        """A new hierarchy with patches covering the tagged cells of each level.

        ``tags[level]`` is a boolean array of that level's shape; the tagged cells grow
        by ``buffer`` cells, are clustered into boxes of at most ``max_patch_size``
        coarse cells per side (``cluster_tags``), and refined. Levels above the tagged
        ones are dropped.
        """
        from wellbalanced_b200.regrid import cluster_tags

        new = AMRHierarchy(self.shape, self.bounds, self.periodic, comm=self.comm, placement=self.placement)
        new.patches = []
        for patch in self.patches_at_level(0):
            new._append(Patch(0, patch.box))
        levels = sorted(tags)
        for level in levels:
            if level > new.max_level:
                break
            boxes = cluster_tags(
                np.asarray(tags[level], dtype=bool),
                buffer=buffer,
                max_size=max_patch_size,
                min_size=min_patch_size,
                parents=[p.box for p in new.patches_at_level(level)],
                periodic=self.periodic,
            )
            for box in boxes:
                new._append(Patch(level + 1, tuple((2 * lo, 2 * hi) for lo, hi in box)))
        return new


# ---- field sets -----------------------------------------------------------------------------
@dataclass(frozen=True)
class FieldGroup:
    lo: int
    hi: int
    node_mask: int  # bit a: axis a is node-centred


def field_groups(ndim):
    """The field groups of the MHD state: 2D (6 cells, A_z nodes), 3D (5 cells, 3 edges)."""
    if ndim == 2:
        return (FieldGroup(0, 6, 0b00), FieldGroup(6, 7, 0b11))
    return (FieldGroup(0, 5, 0b000), FieldGroup(5, 6, 0b110), FieldGroup(6, 7, 0b101), FieldGroup(7, 8, 0b011))


def _boxes_intersect(a, b):
    out = []
    for (alo, ahi), (blo, bhi) in zip(a, b, strict=True):
        lo, hi = max(alo, blo), min(ahi, bhi)
        if lo >= hi:
            return None
        out.append((lo, hi))
    return tuple(out)


#: largest op the host builds (points); `size_ops` cuts a list further when it is small
OP_MAX_POINTS = 1024
#: op blocks resident on a B200 at once (148 SMs x 32 blocks of 64 threads)
OP_WAVE = 148 * 32


def op_points(total):
    """Points per op for a list of `total` points: 64 (one per thread of the op's block)
    while the list fits one wave of blocks, else enough for one wave, up to 1024."""
    per = -(-int(total) // OP_WAVE)
    return int(min(OP_MAX_POINTS, max(64, -(-per // 64) * 64)))


def size_ops(ops):
    """A copy, interpolation or restriction op list cut for the op kernels: small lists
    (a level's halos) into ops of one point per thread, so they run in one wave of short
    blocks; large lists (a big box's halos) into ops of up to 1024 points."""
    ops = np.atleast_1d(np.asarray(ops))
    if ops.size == 0:
        return ops
    total = int(np.prod(ops["n"].astype(np.int64), axis=1).sum())
    return split_box_ops(ops, op_points(total))


def _even_parts(n, size):
    """Starts and counts of `n` cut into near-equal parts of at most `size`."""
    parts = -(-n // size)
    step = -(-n // parts)
    return [(a, min(step, n - a)) for a in range(0, n, step)]


def _box_parts(n, chunk):
    """Sub-boxes (start, count) of a box of n points (axis 2 fastest in the kernels' point
    order, then axis 1) of at most `chunk` points each: whole rows of the fastest axes
    where they fit, so a warp's lanes read consecutive points along the contiguous axis."""
    n = [int(v) for v in n]
    if n[1] * n[2] <= chunk:
        return [((a, 0, 0), (c, n[1], n[2])) for a, c in _even_parts(n[0], max(1, chunk // max(1, n[1] * n[2])))]
    if n[2] <= chunk:
        return [((a, b, 0), (1, c, n[2])) for a in range(n[0]) for b, c in _even_parts(n[1], max(1, chunk // max(1, n[2])))]
    return [((a, b, c0), (1, 1, c)) for a in range(n[0]) for b in range(n[1]) for c0, c in _even_parts(n[2], chunk)]


def split_box_ops(ops, chunk=OP_MAX_POINTS):
    """Copy, interpolation or restriction ops with every box cut into ops of at most
    `chunk` points (the same points, the same arithmetic per point)."""
    ops = np.atleast_1d(np.asarray(ops))
    if ops.size == 0:
        return ops
    dtype = ops.dtype
    big = np.flatnonzero(np.prod(ops["n"].astype(np.int64), axis=1) > chunk)
    if big.size == 0:
        return ops
    out = []
    last = 0
    for b in big:
        if b > last:
            out.append(ops[last:b])  # the ops that fit, unchanged and in order
        last = b + 1
        o = ops[b]
        n = [int(v) for v in o["n"]]
        parts = _box_parts(n, chunk)
        block = np.repeat(np.atleast_1d(o), len(parts))
        starts = np.array([st for st, _ in parts], dtype=np.int64)
        block["n"] = np.array([cnt for _, cnt in parts], dtype=np.int32)
        if "s1" in dtype.names:  # copy: d + p, s1 + m1 p, s2 + m2 p
            block["d"] += starts.astype(np.int32)
            block["s1"] += (block["m1"] * starts).astype(np.int32)
            block["s2"] += (block["m2"] * starts).astype(np.int32)
        elif "fine_lo" in dtype.names:  # interpolation: fine box d + p
            block["d"] += starts.astype(np.int32)
        else:  # restriction: coarse start c, fine start f (2 fine per coarse)
            block["c"] += starts.astype(np.int32)
            block["f"] += (2 * starts).astype(np.int32)
        out.append(block)
    if last < ops.size:
        out.append(ops[last:])
    return np.concatenate(out).astype(dtype)


def _free_boxes(free):
    """Boxes (start, count) covering the True points of a 3-axis boolean array exactly:
    runs along axis 2, merged over equal runs of consecutive rows of axis 1, then of axis 0."""
    n0, n1, _ = free.shape
    planes = []
    for i0 in range(n0):
        boxes = []  # (j0, count1, k0, k1)
        open_ = {}
        for i1 in range(n1):
            row = free[i0, i1]
            runs = []
            k = 0
            while k < row.size:
                if row[k]:
                    e = k
                    while e < row.size and row[e]:
                        e += 1
                    runs.append((k, e))
                    k = e
                else:
                    k += 1
            now = {}
            for run in runs:
                if run in open_:
                    j0, c = open_.pop(run)
                    now[run] = (j0, c + 1)
                else:
                    now[run] = (i1, 1)
            for run, (j0, c) in open_.items():
                boxes.append((j0, c, run[0], run[1]))
            open_ = now
        for run, (j0, c) in open_.items():
            boxes.append((j0, c, run[0], run[1]))
        planes.append(sorted(boxes))
    out = []
    open_ = {}
    for i0, boxes in enumerate(planes):
        now = {}
        for b in boxes:
            now[b] = (open_.pop(b)[0], i0) if b in open_ else (i0, i0)
        for b, (a0, a1) in open_.items():
            out.append(((a0, b[0], b[2]), (a1 - a0 + 1, b[1], b[3] - b[2])))
        open_ = now
    for b, (a0, a1) in open_.items():
        out.append(((a0, b[0], b[2]), (a1 - a0 + 1, b[1], b[3] - b[2])))
    return out


def trim_interp_ops(interp, same):
    """Interpolation ops of a level cut to the halo points that none of the level's
    same-level copy ops writes (the copies overwrite those points after the
    interpolation, so the fill's result is unchanged): a level's interpolation and copies
    then write disjoint points and run in one launch (`wb_fill_ops`)."""
    interp = np.atleast_1d(np.asarray(interp))
    same = np.atleast_1d(np.asarray(same))
    if interp.size == 0 or same.size == 0:
        return interp
    # the copy boxes per (patch, field range), as arrays
    sd = same["d"].astype(np.int64)
    sn = same["n"].astype(np.int64)
    skeys = list(zip(same["dst"].tolist(), same["field_lo"].tolist(), same["field_hi"].tolist(), strict=True))
    groups = {}
    for i, key in enumerate(skeys):
        groups.setdefault(key, []).append(i)
    covers = {key: (sd[idx], sn[idx]) for key, idx in ((k, np.array(v)) for k, v in groups.items())}
    idd = interp["d"].astype(np.int64)
    inn = interp["n"].astype(np.int64)
    ikeys = zip(interp["fine"].tolist(), interp["field_lo"].tolist(), interp["field_hi"].tolist(), strict=True)
    out = []
    for i, key in enumerate(ikeys):
        op = interp[i]
        boxes = covers.get(key)
        if boxes is None:
            out.append(np.atleast_1d(op))
            continue
        d, n = idd[i], inn[i]
        lo = np.maximum(d, boxes[0])
        hi = np.minimum(d + n, boxes[0] + boxes[1])
        meet = np.flatnonzero(np.all(lo < hi, axis=1))
        if meet.size == 0:
            out.append(np.atleast_1d(op))
            continue
        free = np.ones(tuple(int(v) for v in n), dtype=bool)
        for j in meet:
            a, b = lo[j] - d, hi[j] - d
            free[a[0]:b[0], a[1]:b[1], a[2]:b[2]] = False
        if free.all():
            out.append(np.atleast_1d(op))
            continue
        parts = _free_boxes(free)
        if not parts:
            continue
        block = np.repeat(np.atleast_1d(op), len(parts))
        block["d"] = (d + np.array([st for st, _ in parts], dtype=np.int64)).astype(np.int32)
        block["n"] = np.array([cnt for _, cnt in parts], dtype=np.int32)
        out.append(block)
    if not out:
        return np.zeros(0, interp.dtype)
    return np.concatenate(out).astype(interp.dtype)


def number_faces(face_ops):
    """A copy of the interface ops with each op's first coarse face in the flat numbering
    of all ops' faces (`FaceFluxOp.first`: the prefix sum of the lengths, in list order),
    and the total count: the staged register kernel runs one thread per face and finds its
    op by binary search over `first`."""
    ops = np.atleast_1d(np.asarray(face_ops)).copy()
    if ops.size == 0:
        return ops, 0
    lengths = ops["len"].astype(np.int64)
    ops["first"] = np.concatenate([[0], np.cumsum(lengths)[:-1]]).astype(np.int32)
    return ops, int(lengths.sum())


def _concat(arrays, dtype):
    """Records of ``arrays`` in one array of the C layout ``dtype`` (``np.concatenate``
    alone may repack a padded structured dtype)."""
    arrays = [np.atleast_1d(np.asarray(a)) for a in arrays if a is not None and np.asarray(a).size]
    if not arrays:
        return np.zeros(0, dtype)
    return np.concatenate(arrays).astype(dtype)


class Layout:
    """Pool layout, work lists and op lists of a hierarchy for the MHD state."""

    def __init__(self, hierarchy: AMRHierarchy, *, walls=None, precision=32, lx=32, instances=None,
                 align=8, tile=None):
        self.h = hierarchy
        self.ndim = hierarchy.ndim
        if self.ndim not in (2, 3):
            raise ValueError("the MHD state lives on 2D or 3D hierarchies")
        self.nfields = 7 if self.ndim == 2 else 8
        self.groups = field_groups(self.ndim)
        self.precision = precision
        self.lx = lx
        #: 2D: the (tx, ty) tile shape of the stage kernel's work list (None: the default)
        self.tile = None if tile is None else tuple(int(v) for v in tile)
        self.walls = walls or ((False, False),) * self.ndim
        patches = hierarchy.patches
        self.npatches = len(patches)
        self.instances = np.zeros(self.npatches, dtype=np.int32) if instances is None else np.asarray(instances, np.int32)
        self.ninstances = int(self.instances.max()) + 1 if self.npatches else 1
        self._own_last()
        self._pool(align)
        self._tiles()
        self._chunks()
        self.copy_phases = self._copy_ops()
        self.interp_levels = [trim_interp_ops(ops, same) for ops, (same, _) in zip(self._interp_ops(), self.copy_phases,
                                                                                    strict=True)]
        self.restrict_levels = self._restrict_ops()
        self.face_flux_ops, self.reflux_phases, self.register_size = self._reflux_ops()

    # ownership ---------------------------------------------------------------------------
    def _own_last(self):
        """own[p][a]: whether patch p computes its upper node plane along axis a."""
        h = self.h
        self.own = []
        for p in h.patches:
            flags = []
            for a in range(self.ndim):
                flags.append(not self._plane_provided(p, a))
            self.own.append(tuple(flags))

    def _level_lows(self, level):
        """The lower corners of the level's patches (patches x axes), cached."""
        cache = self.__dict__.setdefault("_lows_cache", {})
        if level not in cache:
            cache[level] = np.array([[q.box[b][0] for b in range(self.ndim)] for q in self.h.patches_at_level(level)],
                                    dtype=np.int64).reshape(-1, self.ndim)
        return cache[level]

    def _level_highs(self, level):
        """The upper corners of the level's patches (patches x axes), cached."""
        cache = self.__dict__.setdefault("_highs_cache", {})
        if level not in cache:
            cache[level] = np.array([[q.box[b][1] for b in range(self.ndim)] for q in self.h.patches_at_level(level)],
                                    dtype=np.int64).reshape(-1, self.ndim)
        return cache[level]

    def _plane_provided(self, p, a):
        """Whether same-level patches' lower node planes cover p's upper plane along a."""
        h = self.h
        n_level = h.level_shape(p.level)[a]
        plane = p.box[a][1]
        # transverse node range of the plane, inclusive
        need = [(p.box[b][0], p.box[b][1] + 1) for b in range(self.ndim) if b != a]
        covered = np.zeros([hi - lo for lo, hi in need], dtype=bool)
        same = h.patches_at_level(p.level)
        lows = self._level_lows(p.level)[:, a]
        touch = (lows == plane) | ((lows + n_level == plane) if h.periodic[a] else False)
        for qi in np.flatnonzero(touch):  # the patches whose lower plane is p's upper one
            q = same[qi]
            # q's computed node range along the transverse axes (its lower plane),
            # conservatively [lo, hi) there: its upper nodes may be someone else's
            idx = []
            for (nlo, nhi), b in zip(need, [b for b in range(self.ndim) if b != a], strict=True):
                qlo, qhi = q.box[b]
                s, e = max(nlo, qlo), min(nhi, qhi + 1)
                if s >= e:
                    break
                idx.append(slice(s - nlo, e - nlo))
            else:
                covered[tuple(idx)] = True
        return bool(covered.all())

    # pool ----------------------------------------------------------------------------------
    def _pool(self, align):
        h = self.h
        rows = np.zeros(self.npatches, dtype=_lib.PATCH)
        offset = 0
        bflux = 0
        ncons = 6 if self.ndim == 2 else 5
        self.bflux_size = 0
        for p in h.patches:
            n = list(p.shape) + [1] * (3 - self.ndim)
            dims = [p.shape[a] + 5 for a in range(self.ndim)]  # node-shaped, halo 2
            inner = dims[-1]
            inner = (inner + align - 1) // align * align
            if self.ndim == 2:
                pitch0, pitch1 = inner, 0
                size = dims[0] * inner
            else:
                pitch1 = inner
                pitch0 = dims[1] * inner
                size = dims[0] * pitch0
            size = (size + 31) // 32 * 32
            r = rows[p.index]
            r["off"] = offset
            r["fstride"] = size
            r["pitch0"] = pitch0
            r["pitch1"] = pitch1
            r["n"] = n
            r["instance"] = self.instances[p.index]
            flags = 0
            for a in range(self.ndim):
                lower, upper = self._wall_sides(p, a)
                if lower:
                    flags |= 1 << (2 * a)
                if upper:
                    flags |= 1 << (2 * a + 1)
                if self.own[p.index][a]:
                    flags |= 1 << (8 + a)
            r["flags"] = flags
            r["level"] = p.level
            r["dx"] = list(h.spacing(p.level)) + [1.0] * (3 - self.ndim)
            r["bflux"] = bflux
            faces = sum(2 * int(np.prod([p.shape[b] for b in range(self.ndim) if b != a])) for a in range(self.ndim))
            bflux += faces * ncons
            offset += self.nfields * size
        self.rows = rows
        self.pool_size = offset
        self.bflux_size = bflux

    def _wall_sides(self, p, a):
        shape = self.h.level_shape(p.level)
        lower_wall, upper_wall = self.walls[a]
        return (lower_wall and p.box[a][0] == 0, upper_wall and p.box[a][1] == shape[a])

    def patch_view(self, pool, p, f):
        """A view of field f of patch p in `pool` (a 1-D tensor/array), haloed shape."""
        r = self.rows[p.index]
        start = int(r["off"] + f * r["fstride"])
        if self.ndim == 2:
            X, P0 = p.shape[0] + 5, int(r["pitch0"])
            view = pool[start : start + X * P0].reshape(X, P0)
            return view[:, : p.shape[1] + 5]
        X, Y = p.shape[0] + 5, p.shape[1] + 5
        P0, P1 = int(r["pitch0"]), int(r["pitch1"])
        view = pool[start : start + X * P0].reshape(X, Y, P1)
        return view[:, :, : p.shape[2] + 5]

    # work lists ----------------------------------------------------------------------------
    def _tiles(self):
        lib = _lib.load()
        import ctypes

        a, b = ctypes.c_int(), ctypes.c_int()
        _lib.call("wb_tile_shape", self.ndim, self.precision, ctypes.addressof(a), ctypes.addressof(b))
        self.tile_shape = (a.value, b.value)
        self.default_tile = self.tile_shape
        if getattr(self, "tile", None) is not None:
            if self.tile not in _lib.tile_shapes(self.ndim, self.precision):
                raise ValueError(f"no {self.tile} tile shape; built: {_lib.tile_shapes(self.ndim, self.precision)}")
            self.tile_shape = self.tile
        del lib
        self._cut_tiles()

    def set_tile(self, tile):
        """Cut the stage kernel's work list into `tile` tiles: (tx, ty) in 2D, (ty, tz)
        columns in 3D (one of the shapes `_lib.tile_shapes` lists)."""
        tile = tuple(int(v) for v in tile)
        if tile not in _lib.tile_shapes(self.ndim, self.precision):
            raise ValueError(f"no {self.ndim}D tile shape {tile} for precision code {self.precision}")
        self.tile = self.tile_shape = tile
        self._cut_tiles()

    def _cut_tiles(self):
        """The stage kernel's work list: every patch's computed cells and nodes in tiles."""
        tiles = []
        for index in range(self.npatches):
            n = [int(v) for v in self.rows[index]["n"]]
            own = [n[a] + (1 if self.own[index][a] else 0) for a in range(self.ndim)]
            if self.ndim == 2:
                tx, ty = self.tile_shape
                for x0 in range(0, own[0], tx):
                    for y0 in range(0, own[1], ty):
                        tiles.append((index, x0, y0, 0))
            else:
                ty, tz = self.tile_shape
                for x0 in range(0, own[0], self.lx):
                    for y0 in range(0, own[1], ty):
                        for z0 in range(0, own[2], tz):
                            tiles.append((index, x0, y0, z0))
        self.tiles = np.array(tiles, dtype=np.int32).view(_lib.TILE).reshape(-1) if tiles else np.zeros(0, _lib.TILE)

    def _chunks(self, per=2048):
        patch, start = [], []
        for p in self.h.patches:
            cells = int(np.prod(p.shape))
            if cells + per >= 2**31:  # the rate kernels index a patch's cells in 32 bits
                raise ValueError(f"patch {p.box} has {cells} cells; split the level into patches below 2**31 cells")
            for s in range(0, cells, per):
                patch.append(p.index)
                start.append(s)
        self.chunk_patch = np.array(patch, dtype=np.int32)
        self.chunk_start = np.array(start, dtype=np.int32)
        # finest sum of inverse squared spacings per instance (diffusion limit), and the
        # sum of each (instance, level) holding a patch (0 where it holds none)
        inv = np.zeros(self.ninstances)
        levels = np.zeros((self.ninstances, self.h.max_level + 1))
        for p in self.h.patches:
            s = sum(d**-2 for d in self.h.spacing(p.level))
            inv[self.instances[p.index]] = max(inv[self.instances[p.index]], s)
            levels[self.instances[p.index], p.level] = s
        self.inv_dx2_sum = inv
        self.inv_dx2_levels = levels

    # same-level copies and physical boundaries ----------------------------------------------
    def _computed_box(self, p, g):
        """Computed points of patch p for field group g, as haloed index ranges."""
        out = []
        for a in range(self.ndim):
            node = (g.node_mask >> a) & 1
            n = p.shape[a]
            hi = HALO + n + (1 if node and self.own[p.index][a] else 0)
            out.append((HALO, hi))
        return tuple(out)

    def _haloed_size(self, p, g, a):
        return p.shape[a] + 4 + ((g.node_mask >> a) & 1)

    def _halo_slabs(self, p, g):
        """The halo of p (haloed box minus computed box) as disjoint boxes."""
        full = [(0, self._haloed_size(p, g, a)) for a in range(self.ndim)]
        comp = self._computed_box(p, g)
        slabs = []
        for a in range(self.ndim):
            for side in (0, 1):
                box = []
                for b in range(self.ndim):
                    if b < a:
                        box.append(comp[b])
                    elif b == a:
                        box.append((full[a][0], comp[a][0]) if side == 0 else (comp[a][1], full[a][1]))
                    else:
                        box.append(full[b])
                if all(lo < hi for lo, hi in box):
                    slabs.append(tuple(box))
        return slabs

    def _copy_ops(self):
        """Per level: same-level copy ops, then boundary ops per axis (op arrays)."""
        h = self.h
        phases = []
        for level in range(h.max_level + 1):
            same = []
            patches = h.patches_at_level(level)
            n_level = h.level_shape(level)
            shifts = list(itertools.product(*[(0,) if not h.periodic[a] else (-n_level[a], 0, n_level[a])
                                              for a in range(self.ndim)]))
            qlo = np.array([[q.box[a][0] for a in range(self.ndim)] for q in patches], dtype=np.int64)
            qhi = np.array([[q.box[a][1] for a in range(self.ndim)] for q in patches], dtype=np.int64)
            offsets = np.array(shifts, dtype=np.int64)
            for p in patches:
                # the (source, shift) pairs whose points can reach p's haloed box (its cells
                # and one node more, HALO around): the rest give no op
                plo = np.array([p.box[a][0] - HALO for a in range(self.ndim)], dtype=np.int64)
                phi = np.array([p.box[a][1] + HALO + 1 for a in range(self.ndim)], dtype=np.int64)
                reach = np.all((qlo[None, :, :] + offsets[:, None, :] < phi)
                               & (qhi[None, :, :] + 1 + offsets[:, None, :] > plo), axis=2)
                near = [(int(qi), [shifts[si] for si in np.flatnonzero(reach[:, qi])])
                        for qi in np.flatnonzero(reach.any(axis=0))]
                for g in self.groups:
                    slabs = self._halo_slabs(p, g)
                    for qi, reaching in near:
                        q = patches[qi]
                        comp_q = self._computed_box(q, g)
                        for shift in reaching:
                            # q's computed points in p's haloed coordinates
                            src = tuple(
                                (lo + q.box[a][0] + shift[a] - p.box[a][0], hi + q.box[a][0] + shift[a] - p.box[a][0])
                                for a, (lo, hi) in enumerate(comp_q)
                            )
                            for slab in slabs:
                                box = _boxes_intersect(slab, src)
                                if box is None:
                                    continue
                                n = [hi - lo for lo, hi in box] + [1] * (3 - self.ndim)
                                d = [lo for lo, _ in box] + [0] * (3 - self.ndim)
                                s1 = [lo - q.box[a][0] - shift[a] + p.box[a][0] for a, (lo, _) in enumerate(box)]
                                s1 += [0] * (3 - self.ndim)
                                # a COPY_OP record, fields in order
                                same.append((p.index, q.index, -1, g.lo, g.hi, -1, n, d, s1, (1, 1, 1), (0, 0, 0),
                                             (0, 0, 0), 1.0, 0.0))
            boundary = [[] for _ in range(self.ndim)]
            for p in patches:
                for a in range(self.ndim):
                    if h.periodic[a]:
                        continue
                    lower = p.box[a][0] == 0
                    upper = p.box[a][1] == n_level[a]
                    wall = self.walls[a]
                    for g in self.groups:
                        boundary[a] += self._boundary_ops(p, g, a, lower, upper, wall)
            phases.append((self._pack(same, _lib.COPY_OP), [self._pack(b, _lib.COPY_OP) for b in boundary]))
        return phases

    def _boundary_ops(self, p, g, a, lower, upper, wall):
        ops = []
        size = [self._haloed_size(p, g, b) for b in range(self.ndim)]
        node = (g.node_mask >> a) & 1
        N = size[a]

        def make(d_lo, count, s1, m1a, w1, s2=0, m2a=0, w2=0.0, negate=-1):
            op = np.zeros((), dtype=_lib.COPY_OP)
            op["dst"], op["src1"], op["src2"] = p.index, p.index, p.index
            op["field_lo"], op["field_hi"], op["negate"] = g.lo, g.hi, negate
            n = list(size) + [1] * (3 - self.ndim)
            n[a] = count
            d = [0, 0, 0]
            d[a] = d_lo
            src1 = [0, 0, 0]
            src1[a] = s1
            m1 = [1, 1, 1]
            m1[a] = m1a
            src2 = [0, 0, 0]
            src2[a] = s2
            m2 = [1, 1, 1]
            m2[a] = m2a
            op["n"], op["d"], op["s1"], op["m1"], op["s2"], op["m2"] = n, d, src1, m1, src2, m2
            op["w1"], op["w2"] = w1, w2
            return op

        for side, active in ((0, lower), (1, upper)):
            if not active:
                continue
            is_wall = wall[side]
            if g.node_mask == 0 or (self.ndim == 3 and not node and g.lo >= 5):
                # cell-centred along a
                if self.ndim == 3 and g.lo >= 5:
                    # edge potentials along their own (cell-centred) axis: linear extrapolation
                    ops += self._node_extrapolation(make, side, N)
                    continue
                negate = (1 + a) if is_wall else -1
                if not is_wall:
                    if side == 0:
                        ops.append(make(0, HALO, HALO, 0, 1.0))
                    else:
                        ops.append(make(N - HALO, HALO, N - HALO - 1, 0, 1.0))
                else:
                    if side == 0:  # dst 1-k <- src 2+k
                        ops.append(make(0, HALO, 2 * HALO - 1, -1, 1.0, negate=negate))
                    else:  # dst N-2+k <- src N-3-k
                        ops.append(make(N - HALO, HALO, N - HALO - 1, -1, 1.0, negate=negate))
            else:
                if is_wall:
                    for k in range(1, HALO + 1):
                        if side == 0:  # moved[h-k] = 2 moved[h] - moved[h+k]
                            ops.append(make(HALO - k, 1, HALO, 0, 2.0, HALO + k, 0, -1.0))
                        else:
                            e = N - HALO - 1
                            ops.append(make(e + k, 1, e, 0, 2.0, e - k, 0, -1.0))
                else:
                    ops += self._node_extrapolation(make, side, N)
        return ops

    @staticmethod
    def _node_extrapolation(make, side, N):
        ops = []
        for k in range(1, HALO + 1):
            if side == 0:  # moved[h-k] = (1+k) moved[h] - k moved[h+1]
                ops.append(make(HALO - k, 1, HALO, 0, 1.0 + k, HALO + 1, 0, -float(k)))
            else:
                e = N - HALO - 1
                ops.append(make(e + k, 1, e, 0, 1.0 + k, e - 1, 0, -float(k)))
        return ops

    # coarse-fine ---------------------------------------------------------------------------
    def _interp_ops(self):
        """Per level >= 1: ops interpolating every halo point of its patches from below."""
        h = self.h
        levels = [np.zeros(0, _lib.INTERP_OP)]
        for level in range(1, h.max_level + 1):
            ops = []
            n_coarse = h.level_shape(level - 1)
            coarses = h.patches_at_level(level - 1)
            shifts = list(itertools.product(*[(0,) if not h.periodic[a] else (-n_coarse[a], 0, n_coarse[a])
                                              for a in range(self.ndim)]))
            clo_all = np.array([[c.box[a][0] for a in range(self.ndim)] for c in coarses], dtype=np.int64)
            chi_all = np.array([[c.box[a][1] for a in range(self.ndim)] for c in coarses], dtype=np.int64)
            offsets = np.array(shifts, dtype=np.int64)
            for f in h.patches_at_level(level):
                # the (coarse patch, shift) pairs whose children (and upper nodes) can reach
                # f's haloed box: the rest give no op
                flo = np.array([f.box[a][0] - HALO for a in range(self.ndim)], dtype=np.int64)
                fhi = np.array([f.box[a][1] + HALO + 1 for a in range(self.ndim)], dtype=np.int64)
                reach = np.all((2 * (clo_all[None, :, :] + offsets[:, None, :]) < fhi)
                               & (2 * (chi_all[None, :, :] + offsets[:, None, :] + 1) > flo), axis=2)
                near = [(int(ci), [shifts[si] for si in np.flatnonzero(reach[:, ci])])
                        for ci in np.flatnonzero(reach.any(axis=0))]
                for g in self.groups:
                    slabs = self._halo_slabs(f, g)
                    for ci, reaching in near:
                        c = coarses[ci]
                        for shift in reaching:
                            # fine haloed points whose coarse parent lies in c (+ shift)
                            region = []
                            for a in range(self.ndim):
                                node = (g.node_mask >> a) & 1
                                clo = c.box[a][0] + shift[a]
                                chi = c.box[a][1] + shift[a] + node  # node parents include hi
                                # parent(g) = floor(g / 2) in [clo, chi)  <=>  g in [2 clo, 2 chi)
                                glo, ghi = 2 * clo, 2 * chi
                                region.append((glo - f.box[a][0] + HALO, ghi - f.box[a][0] + HALO))
                            for slab in slabs:
                                box = _boxes_intersect(slab, tuple(region))
                                if box is None:
                                    continue
                                # an INTERP_OP record, fields in order
                                ops.append((f.index, c.index, g.lo, g.hi, g.node_mask, self.ndim,
                                            [hi - lo for lo, hi in box] + [1] * (3 - self.ndim),
                                            [lo for lo, _ in box] + [0] * (3 - self.ndim),
                                            [f.box[a][0] for a in range(self.ndim)] + [0] * (3 - self.ndim),
                                            [c.box[a][0] + shift[a] for a in range(self.ndim)] + [0] * (3 - self.ndim)))
            levels.append(self._pack(ops, _lib.INTERP_OP))
        return levels

    def _restrict_ops(self):
        """Per level >= 1, ops setting the level below from it, per field group.

        Periodic images count: on a periodic axis a fine node plane on the domain's upper
        face is also coarse node plane 0. Only nodes the fine patch computes are read: its
        upper plane, when a neighbour or its own periodic image provides it, holds the
        previous fill's values until the halo fill that follows the restriction.
        """
        h = self.h
        levels = {0: {}}
        for level in range(1, h.max_level + 1):
            n_fine = h.level_shape(level)
            coarses = h.patches_at_level(level - 1)
            clo_all = np.array([[c.box[a][0] for a in range(self.ndim)] for c in coarses], dtype=np.int64)
            chi_all = np.array([[c.box[a][1] for a in range(self.ndim)] for c in coarses], dtype=np.int64)
            # per fine patch, the coarse patches its points (an upper node plane included, on
            # any periodic image) can restrict into: the rest give no op
            near = {}
            for f in h.patches_at_level(level):
                reach = np.zeros(len(coarses), dtype=bool)
                for shift in itertools.product(*[(0, -n_fine[a], n_fine[a]) if h.periodic[a] else (0,)
                                                 for a in range(self.ndim)]):
                    lo = np.array([(f.box[a][0] + shift[a]) // 2 for a in range(self.ndim)], dtype=np.int64)
                    hi = np.array([(f.box[a][1] + shift[a]) // 2 + 1 for a in range(self.ndim)], dtype=np.int64)
                    reach |= np.all((clo_all < hi) & (chi_all + 1 > lo), axis=1)
                near[f.index] = np.flatnonzero(reach)
            per_group = {}
            for g in self.groups:
                ops = []
                for f in h.patches_at_level(level):
                    shifts = [
                        (0, -n_fine[a], n_fine[a]) if h.periodic[a] and (g.node_mask >> a) & 1 else (0,)
                        for a in range(self.ndim)
                    ]
                    for ci in near[f.index]:
                        c = coarses[ci]
                        cbox = self._computed_box(c, g)
                        for shift in itertools.product(*shifts):
                            ranges = []
                            for a in range(self.ndim):
                                # a fine patch's upper node plane counts only where it computes
                                # it (else it is a copy filled after the restriction)
                                node = (g.node_mask >> a) & 1 and self.own[f.index][a]
                                flo, fhi = f.box[a][0] + shift[a], f.box[a][1] + shift[a]
                                lo = max(flo // 2, c.box[a][0])
                                hi = min(fhi // 2 + node, c.box[a][0] + cbox[a][1] - HALO)
                                if lo >= hi:
                                    break
                                ranges.append((lo, hi, flo))
                            else:
                                op = np.zeros((), dtype=_lib.RESTRICT_OP)
                                op["fine"], op["coarse"] = f.index, c.index
                                op["field_lo"], op["field_hi"] = g.lo, g.hi
                                op["node_mask"], op["ndim"] = g.node_mask, self.ndim
                                op["n"] = [hi - lo for lo, hi, _ in ranges] + [1] * (3 - self.ndim)
                                op["c"] = [lo - c.box[a][0] + HALO for a, (lo, _, _) in enumerate(ranges)] + [0] * (3 - self.ndim)
                                op["f"] = [2 * lo - flo + HALO for lo, _, flo in ranges] + [0] * (3 - self.ndim)
                                ops.append(op)
                per_group[g] = self._pack(ops, _lib.RESTRICT_OP)
            levels[level] = per_group
        return levels

    # batches ------------------------------------------------------------------------------
    @classmethod
    def merge(cls, layouts):
        """One layout holding independent problems: instance k is ``layouts[k]``.

        Patch, pool, instance and register indices of each part are shifted past the
        previous parts; no op couples two parts (each keeps its own periodic images).
        Parts may repeat (a batch of same-sized problems shares one part layout).
        """
        first = layouts[0]
        out = cls.__new__(cls)
        out.h = None
        out.ndim = first.ndim
        out.nfields = first.nfields
        out.groups = first.groups
        out.precision = first.precision
        out.lx = first.lx
        out.tile_shape = first.tile_shape
        out.tile = getattr(first, "tile", None)
        out.default_tile = getattr(first, "default_tile", first.tile_shape)
        out.walls = first.walls
        rows, tiles, chunk_patch, chunk_start, inv, inv_levels = [], [], [], [], [], []
        same_levels, boundary_levels, interp_levels = {}, {}, {}
        restrict_levels, face_ops = {}, []
        reflux_phases = [[] for _ in range(2 * first.ndim)]
        own, instances = [], []
        patch_shift = pool_shift = reg_shift = 0
        for k, part in enumerate(layouts):
            r = part.rows.copy()
            r["off"] += pool_shift
            r["instance"] = k
            rows.append(r)
            own.extend(part.own)
            instances.extend([k] * part.npatches)
            t = part.tiles.copy()
            t["patch"] += patch_shift
            tiles.append(t)
            chunk_patch.append(part.chunk_patch + patch_shift)
            chunk_start.append(part.chunk_start)
            inv.append(part.inv_dx2_sum[:1])
            inv_levels.append(part.inv_dx2_levels[0])

            def shifted(ops, fields):
                ops = ops.copy()
                for name in fields:
                    mask = ops[name] >= 0
                    ops[name][mask] += patch_shift
                return ops

            for level, (same, boundary) in enumerate(part.copy_phases):
                same_levels.setdefault(level, []).append(shifted(same, ("dst", "src1", "src2")))
                for axis, ops in enumerate(boundary):
                    boundary_levels.setdefault((level, axis), []).append(shifted(ops, ("dst", "src1", "src2")))
            for level, ops in enumerate(part.interp_levels):
                interp_levels.setdefault(level, []).append(shifted(ops, ("fine", "coarse")))
            for level, groups in part.restrict_levels.items():
                for g, ops in groups.items():
                    restrict_levels.setdefault(level, {}).setdefault(g, []).append(shifted(ops, ("fine", "coarse")))
            f = shifted(part.face_flux_ops, ("coarse", "fine"))
            f["reg_off"] += reg_shift
            face_ops.append(f)
            for phase, ops in enumerate(part.reflux_phases):
                rf = shifted(ops, ("coarse",))
                rf["reg_off"] += reg_shift
                reflux_phases[phase].append(rf)
            patch_shift += part.npatches
            pool_shift += part.pool_size
            reg_shift += part.register_size
        out.rows = _concat(rows, _lib.PATCH)
        out.npatches = patch_shift
        out.pool_size = pool_shift
        out.own = own
        out.instances = np.array(instances, dtype=np.int32)
        out.ninstances = len(layouts)
        out.tiles = _concat(tiles, _lib.TILE)
        out.chunk_patch = np.concatenate(chunk_patch).astype(np.int32)
        out.chunk_start = np.concatenate(chunk_start).astype(np.int32)
        out.inv_dx2_sum = np.concatenate(inv)
        width = max(len(row) for row in inv_levels)
        out.inv_dx2_levels = np.zeros((len(layouts), width))
        for k, row in enumerate(inv_levels):
            out.inv_dx2_levels[k, : len(row)] = row
        nlevels = max(len(part.copy_phases) for part in layouts)
        naxes = first.ndim
        out.copy_phases = []
        for level in range(nlevels):
            same = _concat(same_levels.get(level, []), _lib.COPY_OP)
            boundary = [_concat(boundary_levels.get((level, a), []), _lib.COPY_OP) for a in range(naxes)]
            out.copy_phases.append((same, boundary))
        out.interp_levels = [_concat(interp_levels.get(level, []), _lib.INTERP_OP) for level in range(nlevels)]
        out.restrict_levels = {0: {}}
        for level, groups in restrict_levels.items():
            if level == 0:
                continue
            out.restrict_levels[level] = {g: _concat(ops, _lib.RESTRICT_OP) for g, ops in groups.items()}
        out.face_flux_ops = _concat(face_ops, _lib.FACE_FLUX_OP)
        out.reflux_phases = [_concat(ops, _lib.REFLUX_OP) for ops in reflux_phases]
        out.register_size = reg_shift
        out.max_level = max(part.max_level for part in layouts)
        return out

    @property
    def max_level(self):
        return self.__dict__.get("_max_level", self.h.max_level if self.h is not None else 0)

    @max_level.setter
    def max_level(self, value):
        self.__dict__["_max_level"] = value

    # refluxing ----------------------------------------------------------------------------
    @property
    def reflux_ops(self):
        """All RefluxOps, phase after phase (`reflux_phases`)."""
        return _concat(self.reflux_phases, _lib.REFLUX_OP)

    def _reflux_ops(self):
        """Coarse-fine interfaces: one FaceFluxOp and one RefluxOp per (fine side, coarse patch).

        The coarse cell outside fine patch F across its side along axis a (wrapped on a
        periodic axis) takes the correction; its face shared with F's region is recomputed
        in the coarse patch holding that cell, the fine faces in F.

        A coarse cell between fine patches takes corrections from several sides, so the
        RefluxOps are grouped into phases applied one after the other, each one race-free
        launch. Taken per (axis, side), two ops of one group never meet in a cell (the
        fine patches of a level do not overlap); `_reflux_groups` then merges these 2 ndim
        groups where no cell is shared, keeping the order of the corrections of every
        cell (usually fewer launches, the same arithmetic).
        """
        h = self.h
        ncons = 6 if self.ndim == 2 else 5
        face_ops = []
        phases = [[] for _ in range(2 * self.ndim)]
        offset = 0
        for f in h.patches:
            if f.level == 0:
                continue
            n_coarse = h.level_shape(f.level - 1)
            dx = h.spacing(f.level - 1)
            for a in range(self.ndim):
                trans = [b for b in range(self.ndim) if b != a]
                for side in (0, 1):
                    plane_f = f.box[a][side]
                    plane_c = plane_f // 2
                    outside = plane_c - 1 if side == 0 else plane_c
                    if h.periodic[a]:
                        outside_w = outside % n_coarse[a]
                    elif 0 <= outside < n_coarse[a]:
                        outside_w = outside
                    else:
                        continue
                    face_c = outside_w + 1 if side == 0 else outside_w
                    coarses = h.patches_at_level(f.level - 1)
                    lows, highs = self._level_lows(f.level - 1)[:, a], self._level_highs(f.level - 1)[:, a]
                    for ci in np.flatnonzero((lows <= outside_w) & (outside_w < highs)):
                        c = coarses[ci]
                        ranges = []
                        for b in trans:
                            lo = max(f.box[b][0] // 2, c.box[b][0])
                            hi = min(f.box[b][1] // 2, c.box[b][1])
                            if lo >= hi:
                                break
                            ranges.append((lo, hi))
                        else:
                            counts = [hi - lo for lo, hi in ranges]
                            length = int(np.prod(counts))
                            width = counts[1] if self.ndim == 3 else 1
                            op = np.zeros((), dtype=_lib.FACE_FLUX_OP)
                            op["coarse"], op["fine"] = c.index, f.index
                            op["ndim"], op["axis"] = self.ndim, a
                            op["t1"] = trans[0]
                            op["t2"] = trans[1] if self.ndim == 3 else -1
                            op["coarse_plane"] = face_c - c.box[a][0] + HALO
                            op["fine_plane"] = plane_f - f.box[a][0] + HALO
                            op["coarse_t0"] = [lo - c.box[b][0] + HALO for b, (lo, _) in zip(trans, ranges, strict=True)] + [0] * (3 - self.ndim)
                            op["fine_t0"] = [2 * lo - f.box[b][0] + HALO for b, (lo, _) in zip(trans, ranges, strict=True)] + [0] * (3 - self.ndim)
                            op["len"], op["width"] = length, width
                            op["reg_off"] = offset
                            face_ops.append(op)
                            rop = np.zeros((), dtype=_lib.REFLUX_OP)
                            rop["coarse"] = c.index
                            rop["len"], rop["width"], rop["ncomp"] = length, width, ncons
                            cidx = [0, 0, 0]
                            cidx[a] = outside_w - c.box[a][0] + HALO
                            for b, (lo, _) in zip(trans, ranges, strict=True):
                                cidx[b] = lo - c.box[b][0] + HALO
                            rop["c"] = cidx
                            rop["t1"] = trans[0]
                            rop["t2"] = trans[1] if self.ndim == 3 else -1
                            rop["field"] = list(range(ncons)) + [0] * (8 - ncons)
                            rop["sign"] = 1.0 if side == 0 else -1.0
                            rop["dx"] = dx[a]
                            rop["reg_off"] = offset
                            phases[2 * a + side].append(rop)
                            offset += ncons * length
        phases = self._reflux_groups(phases)
        return (self._pack(face_ops, _lib.FACE_FLUX_OP), [self._pack(ops, _lib.REFLUX_OP) for ops in phases], offset)

    @staticmethod
    def _reflux_groups(phases):
        """Reflux ops regrouped into as few race-free launches as the order of the
        corrections allows: each op goes to the group after the last group holding an
        earlier op (in the given order) that shares one of its coarse cells, so every cell
        takes its corrections in the same order as before."""
        last = {}  # coarse cell -> group of the latest op that corrected it
        groups = []
        for ops in phases:
            for op in ops:
                t1, t2 = int(op["t1"]), int(op["t2"])
                cells = []
                for s in range(int(op["len"])):
                    idx = [int(v) for v in op["c"]]
                    idx[t1] += s // int(op["width"])
                    if t2 >= 0:
                        idx[t2] += s % int(op["width"])
                    cells.append((int(op["coarse"]), *idx))
                g = 1 + max((last[c] for c in cells if c in last), default=-1)
                while len(groups) <= g:
                    groups.append([])
                groups[g].append(op)
                for c in cells:
                    last[c] = g
        return groups

    @staticmethod
    def _pack(ops, dtype, chunk=OP_MAX_POINTS):
        """Op array; halo, interpolation and restriction boxes are cut into ops of at most
        `chunk` points (default `OP_MAX_POINTS`; the engine cuts small lists further)."""
        if not ops:
            return np.zeros(0, dtype)
        if isinstance(ops[0], tuple):  # records given as tuples of their fields, in order
            packed = np.array(ops, dtype=dtype)
        else:
            packed = np.array([np.asarray(o).reshape(()) for o in ops], dtype=dtype)
        if dtype not in (_lib.COPY_OP, _lib.INTERP_OP, _lib.RESTRICT_OP):
            return packed
        points = np.prod(packed["n"].astype(np.int64), axis=1)
        if np.any(points >= 2**31):  # the op kernels index an op's points in 32 bits
            raise ValueError(f"an op of {int(points.max())} points; the kernels take below 2**31")
        lo, hi = packed["field_lo"], packed["field_hi"]
        if np.any((lo < 0) | (lo > hi) | (hi > 8)):  # the copy kernel holds 8 fields
            raise ValueError("op fields outside 0..7")
        return split_box_ops(packed, chunk)
