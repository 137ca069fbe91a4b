"""CPU patch hierarchy for the oracle solvers (test infrastructure only).

ORACLE — imported only by the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg.

The reference keeps its mesh in the external package ``patchwork-amr`` 0.2.0 (git
``max-models/patchwork@9042e879``, ``uv.lock:3139-3141``), whose source is not
available. This module restates the semantics the reference solver relies on, as its
docstrings and tests describe them:

* levels refined by 2, each a set of patches with boxes in level indices; fields are
  cell-, node- or edge-centred with a halo (``mhd.py:467-472``, ``mhd3d.py:219-223``);
* ``exchange_halos``: halo values from same-level patches and periodic images, else
  interpolated from the level below — linear in each cell-centred direction ("the
  conserved fields' bilinearly") and, for node/edge potentials, the coarse value at
  coincident nodes and the symmetric 4-point midpoint rule (exact for cubics, so at
  least the "quadratic" accuracy of ``mhd.py:55-58`` / ``CHANGELOG.md:10-13``);
* ``restrict``: covered coarse cells take the mean of their fine cells; coarse nodes
  shared with a finer patch take the fine value (``mhd.py:52-55``); coarse edges take
  the mean of the two fine edges along them (``mhd3d.py:33-36``);
* ``FluxRegister``: ``update`` applies ``U -= dt * sum_a dF_a/dx_a`` on every patch and
  records ``scale * F`` on coarse faces next to finer patches and on the fine faces
  over them; ``reflux`` replaces, in the coarse leaf cells beside a finer patch, the
  recorded coarse flux by the mean of the recorded fine fluxes (Berger–Colella; the
  identity of ``tests/unit/test_fluid2d_patches.py:162-240``), then averages the
  covered coarse cells down (standard Berger–Colella; whether patchwork does this is
  not documented).

Parity with patchwork itself is therefore unpinned for coarse–fine behaviour; single
level runs are pinned against the reference through the golden vectors.
"""

from __future__ import annotations

import itertools

import numpy as np

_NODE_AXES = {
    "cell": lambda ndim: (0,) * ndim,
    "node": lambda ndim: (1,) * ndim,
    "x-edge": lambda ndim: (0, 1, 1),
    "y-edge": lambda ndim: (1, 0, 1),
    "z-edge": lambda ndim: (1, 1, 0),
}


class Field:
    """The haloed array of one field on one patch; ``local`` is a view without halo."""

    def __init__(self, shape, extra, halo):
        self.extra = tuple(extra)
        self.halo = halo
        self.local_with_halos = np.zeros(
            tuple(n + e + 2 * halo for n, e in zip(shape, extra, strict=True))
        )
        self.local = self.local_with_halos[
            tuple(slice(halo, halo + n + e) for n, e in zip(shape, extra, strict=True))
        ]


class Patch:
    def __init__(self, level, box):
        self.level = int(level)
        self.box = tuple((int(lo), int(hi)) for lo, hi in box)
        self.shape = tuple(hi - lo for lo, hi in self.box)
        self.fields: dict[str, Field] = {}
        self.is_local = True
        self.ranks = [0]

    def field(self, name):
        return self.fields[name]

    def coordinates(self, hierarchy, extra):
        spacing = hierarchy.spacing(self.level)
        axes = []
        for a, (lo, hi) in enumerate(self.box):
            start = hierarchy.lower_bound[a]
            if extra[a]:
                axes.append(start + np.arange(lo, hi + 1) * spacing[a])
            else:
                axes.append(start + (np.arange(lo, hi) + 0.5) * spacing[a])
        return np.meshgrid(*axes, indexing="ij")


class Hierarchy:
    """Levels of patches over a box; level 0 must be covered by its patches."""

    def __init__(self, shape, bounds=None, periodic=None, split=None):
        self.shape = tuple(int(n) for n in shape)
        self.ndim = len(self.shape)
        self.bounds = tuple(
            (float(lo), float(hi)) for lo, hi in (bounds or ((0.0, 1.0),) * self.ndim)
        )
        self.lower_bound = tuple(lo for lo, _ in self.bounds)
        self.periodic = tuple(bool(p) for p in (periodic or (False,) * self.ndim))
        self.refinement_ratio = 2
        self.patches: list[Patch] = []
        self.centering: dict[str, tuple[tuple[int, ...], int, bool]] = {}
        split = split or (1,) * self.ndim
        cuts = [
            np.linspace(0, n, s + 1).round().astype(int)
            for n, s in zip(self.shape, split, strict=True)
        ]
        for index in itertools.product(*(range(s) for s in split)):
            box = tuple((int(c[k]), int(c[k + 1])) for c, k in zip(cuts, index, strict=True))
            self.patches.append(Patch(0, box))

    # geometry -------------------------------------------------------------------------
    @property
    def max_level(self):
        return max(p.level for p in self.patches)

    @property
    def local_patches(self):
        return self.patches

    def level_shape(self, level):
        return tuple(n * 2**level for n in self.shape)

    def spacing(self, level):
        return tuple(
            (hi - lo) / n for (lo, hi), n in zip(self.bounds, self.level_shape(level), strict=True)
        )

    def patches_at_level(self, level):
        return [p for p in self.patches if p.level == level]

    def add_patch(self, level, box):
        patch = Patch(level, box)
        for name, (extra, halo, _) in self.centering.items():
            patch.fields[name] = Field(patch.shape, extra, halo)
        self.patches.append(patch)
        return patch

    def allocate_field(self, name, halo=2, centering="cell", conservative=False):
        extra = _NODE_AXES[centering](self.ndim)
        self.centering[name] = (extra, halo, conservative)
        for patch in self.patches:
            patch.fields[name] = Field(patch.shape, extra, halo)

    # level composites -----------------------------------------------------------------
    def _composite(self, name, level):
        """The level's values (with a halo of padding) and the mask of covered points."""
        extra, h, _ = self.centering[name]
        size = tuple(n + e + 2 * h for n, e in zip(self.level_shape(level), extra, strict=True))
        values = np.zeros(size)
        mask = np.zeros(size, dtype=bool)
        for patch in self.patches_at_level(level):
            index = tuple(
                slice(h + lo, h + hi + e) for (lo, hi), e in zip(patch.box, extra, strict=True)
            )
            values[index] = patch.field(name).local
            mask[index] = True
        return values, mask

    def _wrap(self, name, level, arrays):
        extra, h, _ = self.centering[name]
        shape = self.level_shape(level)
        for a in range(self.ndim):
            if not self.periodic[a]:
                continue
            n, e = shape[a], extra[a]
            if e and len(arrays) == 2:
                # node n and node 0 are one node: take it from whichever patch covers it
                values = np.moveaxis(arrays[0], a, 0)
                mask = np.moveaxis(arrays[1], a, 0)
                first, last = mask[h].copy(), mask[h + n].copy()
                values[h + n] = np.where(~last & first, values[h], values[h + n])
                values[h] = np.where(~first & last, values[h + n], values[h])
                mask[h] = first | last
                mask[h + n] = first | last
            for array in arrays:
                moved = np.moveaxis(array, a, 0)
                for k in range(1, h + 1):
                    moved[h - k] = moved[h + n - k]
                for k in range(h):
                    moved[h + n + e + k] = moved[h + e + k]

    def _interpolate(self, name, level, coarse):
        """Values at every point of ``level`` (with padding) interpolated from ``coarse``.

        ``coarse`` is the level below with padding ``h``; cell-centred directions are
        linear (weights 3/4, 1/4 toward the nearer neighbour), node directions take the
        coincident coarse node or the 4-point midpoint rule (-1, 9, 9, -1) / 16.
        """
        extra, h, _ = self.centering[name]
        size = tuple(n + e + 2 * h for n, e in zip(self.level_shape(level), extra, strict=True))
        result = coarse
        for a in range(self.ndim):
            n_fine = size[a]
            f = np.arange(n_fine) - h  # fine index along a
            parts = []
            if extra[a]:
                even = f % 2 == 0
                c = f // 2
                rows = []
                for k in range(n_fine):
                    ck = c[k] + h
                    if even[k]:
                        rows.append({ck: 1.0})
                    else:
                        rows.append(
                            {ck - 1: -1 / 16, ck: 9 / 16, ck + 1: 9 / 16, ck + 2: -1 / 16}
                        )
            else:
                c = f // 2
                offset = f - 2 * c
                rows = []
                for k in range(n_fine):
                    ck = c[k] + h
                    other = ck - 1 if offset[k] == 0 else ck + 1
                    rows.append({ck: 0.75, other: 0.25})
            moved = np.moveaxis(result, a, 0)
            for weights in rows:
                acc = 0.0
                for index, weight in weights.items():
                    index = min(max(index, 0), moved.shape[0] - 1)
                    acc = acc + weight * moved[index]
                parts.append(acc)
            result = np.moveaxis(np.stack(parts), 0, a)
        return result

    def exchange_level(self, name, level, coarse=None):
        """Fill the halos of ``level``: same level and periodic images, else interpolated.

        ``coarse``: the padded composite of the level below (after its own halos and
        boundaries were filled); returns this level's padded composite.
        """
        extra, h, _ = self.centering[name]
        values, mask = self._composite(name, level)
        self._wrap(name, level, (values, mask))
        if level > 0 and coarse is not None:
            interpolated = self._interpolate(name, level, coarse)
            values = np.where(mask, values, interpolated)
        for patch in self.patches_at_level(level):
            index = tuple(
                slice(lo, hi + e + 2 * h) for (lo, hi), e in zip(patch.box, extra, strict=True)
            )
            field = patch.field(name)
            halo_mask = np.ones(field.local_with_halos.shape, dtype=bool)
            halo_mask[tuple(slice(h, h + n + e) for n, e in zip(patch.shape, extra, strict=True))] = False
            field.local_with_halos[halo_mask] = values[index][halo_mask]
        return values

    def padded(self, name, level):
        """The level's padded composite from its patches' haloed arrays (halos included)."""
        extra, h, _ = self.centering[name]
        size = tuple(n + e + 2 * h for n, e in zip(self.level_shape(level), extra, strict=True))
        values = np.zeros(size)
        for patch in self.patches_at_level(level):
            index = tuple(
                slice(lo, hi + e + 2 * h) for (lo, hi), e in zip(patch.box, extra, strict=True)
            )
            values[index] = patch.field(name).local_with_halos
        for patch in self.patches_at_level(level):  # interiors win over others' halos
            index = tuple(
                slice(h + lo, h + hi + e) for (lo, hi), e in zip(patch.box, extra, strict=True)
            )
            values[index] = patch.field(name).local
        return values

    # restriction ----------------------------------------------------------------------
    def restrict(self, name):
        """Coarse values under finer patches from the fine ones, finest level first.

        Cell-centred directions average the two fine values, node directions take the
        coincident fine value: mean of the fine cells for cell fields, injection for
        nodes, mean of the two fine edges along an edge.
        """
        if self.max_level == 0:
            return
        extra, _, _ = self.centering[name]
        for level in range(self.max_level, 0, -1):
            for fine in self.patches_at_level(level):
                for coarse in self.patches_at_level(level - 1):
                    self._restrict_pair(name, extra, fine, coarse)

    def _restrict_pair(self, name, extra, fine, coarse):
        """Restrict ``fine`` into ``coarse``, periodic images included (a fine node plane
        on the domain's upper face is also the coarse node plane 0)."""
        shifts = []
        for a in range(self.ndim):
            n_fine = self.level_shape(fine.level)[a]
            shifts.append((0, -n_fine, n_fine) if self.periodic[a] and extra[a] else (0,))
        for shift in itertools.product(*shifts):
            self._restrict_shifted(name, extra, fine, coarse, shift)

    def _restrict_shifted(self, name, extra, fine, coarse, shift):
        source = fine.field(name).local
        target = coarse.field(name).local
        coarse_index, fine_parts = [], []
        for a in range(self.ndim):
            flo, fhi = fine.box[a][0] + shift[a], fine.box[a][1] + shift[a]
            clo, chi = coarse.box[a]
            e = extra[a]
            lo = max(flo // 2, clo)
            hi = min(fhi // 2 + e, chi + e)
            if lo >= hi:
                return
            coarse_index.append(slice(lo - clo, hi - clo))
            start = 2 * lo - flo
            if e:
                fine_parts.append([slice(start, start + 2 * (hi - lo) - 1, 2)])
            else:
                fine_parts.append(
                    [slice(start, start + 2 * (hi - lo), 2), slice(start + 1, start + 2 * (hi - lo), 2)]
                )
        total = 0.0
        count = 0
        for combo in itertools.product(*fine_parts):
            total = total + source[combo]
            count += 1
        target[tuple(coarse_index)] = total / count

    # leaf cells -----------------------------------------------------------------------
    def covered(self, patch):
        """Mask of the patch's cells covered by a patch of the next finer level."""
        mask = np.zeros(patch.shape, dtype=bool)
        for fine in self.patches_at_level(patch.level + 1):
            index = []
            for a in range(self.ndim):
                (flo, fhi), (lo, hi) = fine.box[a], patch.box[a]
                start, stop = max(flo // 2, lo), min(fhi // 2, hi)
                if start >= stop:
                    break
                index.append(slice(start - lo, stop - lo))
            else:
                mask[tuple(index)] = True
        return mask

    def integral(self, name):
        """The integral of a cell field over the domain, from the leaf cells."""
        total = 0.0
        for patch in self.patches:
            volume = float(np.prod(self.spacing(patch.level)))
            values = patch.field(name).local
            total += float(np.sum(values[~self.covered(patch)])) * volume
        return total

    def gather(self, patch, name):
        return np.array(patch.field(name).local)


class FluxRegister:
    """Berger–Colella flux register over a hierarchy (see the module docstring).

    ``update(name, fluxes, dt, scale)``: ``fluxes(patch)`` returns one array per axis,
    the fluxes through the patch's own faces (``(nx + 1, ny)``, ``(nx, ny + 1)`` in 2D).
    """

    def __init__(self, hierarchy):
        self.hierarchy = hierarchy
        self.records: dict[str, list] = {}

    def reset(self):
        self.records = {}

    def _interfaces(self):
        """Per coarse patch and axis and side: the coarse faces under a finer patch's side.

        Yields ``(coarse, fine, axis, side, coarse_face_plane, transverse ranges)``
        where the face lies on the fine patch's boundary and the coarse cell on the
        outer side is a leaf cell of ``coarse``.
        """
        h = self.hierarchy
        for fine in h.patches:
            if fine.level == 0:
                continue
            for coarse in h.patches_at_level(fine.level - 1):
                for a in range(h.ndim):
                    for side in (0, 1):
                        plane = fine.box[a][side] // 2  # coarse face index along a
                        # the coarse cell outside the fine patch
                        cell = plane - 1 if side == 0 else plane
                        n_level = h.level_shape(coarse.level)[a]
                        if h.periodic[a]:
                            cell_w = cell % n_level
                        else:
                            if cell < 0 or cell >= n_level:
                                continue
                            cell_w = cell
                        shift = cell_w - cell
                        lo, hi = coarse.box[a]
                        if not lo <= cell_w < hi:
                            continue
                        ranges = []
                        for b in range(h.ndim):
                            if b == a:
                                continue
                            flo, fhi = fine.box[b]
                            clo, chi = coarse.box[b]
                            start, stop = max(flo // 2, clo), min(fhi // 2, chi)
                            if start >= stop:
                                break
                            ranges.append((b, start, stop))
                        else:
                            yield coarse, fine, a, side, plane, shift, ranges

    def update(self, name, fluxes, dt, scale=1.0):
        h = self.hierarchy
        records = self.records.setdefault(name, {})
        computed = {}
        for patch in h.patches:
            parts = fluxes(patch)
            computed[id(patch)] = parts
            spacing = h.spacing(patch.level)
            divergence = 0.0
            for a, flux in enumerate(parts):
                divergence = divergence + np.diff(flux, axis=a) / spacing[a]
            patch.field(name).local[...] -= dt * divergence
        for coarse, fine, a, side, plane, shift, ranges in self._interfaces():
            key = (id(coarse), id(fine), a, side)
            cflux = computed[id(coarse)][a]
            fflux = computed[id(fine)][a]
            c_index = [None] * h.ndim
            f_parts = [None] * h.ndim
            c_index[a] = plane + shift - coarse.box[a][0]
            fplane = fine.box[a][side] - fine.box[a][0]
            f_parts[a] = [slice(fplane, fplane + 1)]
            for b, start, stop in ranges:
                c_index[b] = slice(start - coarse.box[b][0], stop - coarse.box[b][0])
                f0 = 2 * start - fine.box[b][0]
                f1 = 2 * stop - fine.box[b][0]
                f_parts[b] = [slice(f0, f1, 2), slice(f0 + 1, f1, 2)]
            coarse_part = scale * cflux[tuple(c_index)]
            fine_sum = 0.0
            count = 0
            for combo in itertools.product(*f_parts):
                fine_sum = fine_sum + np.squeeze(fflux[combo], axis=a)
                count += 1
            fine_part = scale * fine_sum / count
            old = records.get(key)
            if old is None:
                records[key] = [coarse_part, fine_part, tuple(c_index), a, side, coarse]
            else:
                old[0] = old[0] + coarse_part
                old[1] = old[1] + fine_part

    def reflux(self, name):
        """Correct the coarse leaf cells beside finer patches, then average down."""
        h = self.hierarchy
        records = self.records.pop(name, {})
        for coarse_part, fine_part, c_index, a, side, coarse in records.values():
            dx = h.spacing(coarse.level)[a]
            values = coarse.field(name).local
            index = list(c_index)
            # the coarse cell outside the fine patch: below the face for side 0
            plane = index[a]
            index[a] = plane - 1 if side == 0 else plane
            sign = 1.0 if side == 0 else -1.0  # face is the cell's upper (side 0) or lower face
            values[tuple(index)] -= sign * (fine_part - coarse_part) / dx
        h.restrict(name)
