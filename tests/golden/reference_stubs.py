"""Minimal stand-ins that let the reference's own MHD code run in this container.

Used ONLY by ``make_golden.py`` (fixture generation). The reference solver
(``carafe.mhd.MHD2D``, ``carafe.mhd3d.MHD3D`` and the NumPy / Pyccel-as-Python
kernels of ``carafe/kernels``) is imported unchanged from a reference checkout;
the packages it needs and that are absent here are replaced by small stubs:

* ``patchwork``: one refinement level covered by one or more patches, periodic
  halo exchange between them, ``FluxRegister.update`` as the plain divergence
  ``U -= dt * sum_a (F_a[k+1] - F_a[k]) / dx_a`` and a no-op ``reflux`` (there
  are no coarse-fine faces on one level), a no-op ``restrict``;
* ``cunumpy``: ``KernelPackage.from_folder`` dispatching to ``<name>_numpy`` or
  ``<name>_pyccel`` (the latter run as plain Python);
* ``methodcard``, ``scope_profiler``: identity decorators;
* ``maybempi``: a one-rank communicator;
* ``xarray``: a dict-backed Dataset/Variable.

Nothing here is shipped or imported by the product.
"""

from __future__ import annotations

import contextlib
import importlib
import itertools
import sys
import types

import numpy as np

_CHOICE = ["numpy"]


# -- methodcard / scope_profiler -------------------------------------------------------
def _identity_decorator(*_args, **_kwargs):
    def wrap(obj):
        return obj

    return wrap


class ConvergenceProblem:
    def __init__(self, error, steps):
        self.error, self.steps = error, steps


# -- xarray ------------------------------------------------------------------------------
class Variable:
    def __init__(self, dims, values, attrs=None):
        self.dims = (dims,) if isinstance(dims, str) else tuple(dims)
        self.values = np.asarray(values)
        self.attrs = dict(attrs or {})

    def min(self):
        return Variable((), np.nanmin(self.values))

    def max(self):
        return Variable((), np.nanmax(self.values))

    def __float__(self):
        return float(self.values)

    def __array__(self, dtype=None, copy=None):
        return np.asarray(self.values, dtype=dtype)

    def __sub__(self, other):
        return Variable(self.dims, self.values - np.asarray(other))


class Dataset:
    def __init__(self, data, coords=None, attrs=None):
        self._data = dict(data)
        self._coords = dict(coords or {})
        self.attrs = dict(attrs or {})

    @property
    def data_vars(self):
        return list(self._data)

    def __getitem__(self, name):
        if name in self._data:
            return self._data[name]
        return self._coords[name]

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        try:
            return self[name]
        except KeyError as error:
            raise AttributeError(name) from error


# -- maybempi ----------------------------------------------------------------------------
class _Comm:
    def allreduce(self, value, op=None):
        return value

    def bcast(self, value, root=0):
        return value

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1


class _MPI:
    MIN = "min"
    MAX = "max"
    SUM = "sum"
    COMM_WORLD = _Comm()
    COMM_SELF = _Comm()


# -- patchwork (one level) ---------------------------------------------------------------
_EXTRA = {
    "cell": None,
    "node": "all",
    "x-edge": (0, 1, 1),
    "y-edge": (1, 0, 1),
    "z-edge": (1, 1, 0),
}


def _extra(centering, ndim):
    spec = _EXTRA[centering]
    if spec is None:
        return (0,) * ndim
    if spec == "all":
        return (1,) * ndim
    return tuple(spec)


class _Field:
    def __init__(self, shape, extra, halo):
        self.extra = extra
        self.halo = halo
        self.local_with_halos = np.zeros(
            tuple(n + e + 2 * halo for n, e in zip(shape, extra, strict=True))
        )
        self.local = self.local_with_halos[
            tuple(slice(halo, halo + n + e) for n, e in zip(shape, extra, strict=True))
        ]


class Patch:
    def __init__(self, box, level=0):
        self.box = tuple(tuple(b) for b in box)
        self.level = level
        self.shape = tuple(hi - lo for lo, hi in self.box)
        self._fields = {}
        self.is_local = True
        self.ranks = [0]

    def field(self, name):
        return self._fields[name]

    def _axes(self, hierarchy, extra):
        spacing = hierarchy.spacing(self.level)
        axes = []
        for a, (lo, hi) in enumerate(self.box):
            start = hierarchy.lower_bound[a]
            if extra[a]:
                axes.append(start + np.arange(lo, hi + 1) * spacing[a])
            else:
                axes.append(start + (np.arange(lo, hi) + 0.5) * spacing[a])
        return np.meshgrid(*axes, indexing="ij")

    def local_cell_centers(self, hierarchy, name):
        return self._axes(hierarchy, (0,) * len(self.box))

    def local_node_coordinates(self, hierarchy, name):
        return self._axes(hierarchy, (1,) * len(self.box))

    def local_coordinates(self, hierarchy, name):
        return self._axes(hierarchy, self._fields[name].extra)


class AMRHierarchy:
    """One level of ``shape`` cells over ``bounds``, covered by ``split`` patches."""

    def __init__(
        self,
        shape,
        bounds=None,
        periodic=None,
        comm=None,
        placement=None,
        geometry=None,
        split=None,
    ):
        self.shape = tuple(int(n) for n in shape)
        self.ndim = len(self.shape)
        self.bounds = tuple(
            tuple(float(v) for v in b) for b in (bounds or ((0.0, 1.0),) * self.ndim)
        )
        self.lower_bound = tuple(b[0] for b in self.bounds)
        self.periodic = tuple(bool(p) for p in (periodic or (False,) * self.ndim))
        self.cylindrical = geometry == "cylindrical"
        self.graded = False
        self.comm = comm or _MPI.COMM_WORLD
        self.max_level = 0
        self.refinement_ratio = 2
        split = split or (1,) * self.ndim
        cuts = [np.linspace(0, n, s + 1).round().astype(int) for n, s in zip(self.shape, split, strict=True)]
        self.patches = [
            Patch(tuple((int(c[k]), int(c[k + 1])) for c, k in zip(cuts, index, strict=True)))
            for index in itertools.product(*(range(s) for s in split))
        ]
        self.local_patches = self.patches
        self._centering = {}

    def level_shape(self, level):
        return self.shape

    def spacing(self, level):
        return tuple((hi - lo) / n for (lo, hi), n in zip(self.bounds, self.shape, strict=True))

    def patches_at_level(self, level):
        return self.patches if level == 0 else []

    def allocate_field(self, name, halo=0, split=None, conservative=False, centering="cell"):
        extra = _extra(centering, self.ndim)
        self._centering[name] = (extra, halo)
        for patch in self.patches:
            patch._fields[name] = _Field(patch.shape, extra, halo)

    def gather(self, patch, name):
        return np.array(patch.field(name).local)

    def integral(self, name):
        volume = float(np.prod(self.spacing(0)))
        return float(sum(np.sum(p.field(name).local) for p in self.patches) * volume)

    def restrict(self, name):
        return None

    def exchange_halos(self, name, interpolation=None):
        extra, h = self._centering[name]
        size = tuple(n + e + 2 * h for n, e in zip(self.shape, extra, strict=True))
        level = np.zeros(size)
        for patch in self.patches:
            index = tuple(
                slice(h + lo, h + hi + e) for (lo, hi), e in zip(patch.box, extra, strict=True)
            )
            level[index] = patch.field(name).local
        for a in range(self.ndim):
            if not self.periodic[a]:
                continue
            n = self.shape[a]
            moved = np.moveaxis(level, a, 0)
            for k in range(1, h + 1):
                moved[h - k] = moved[h + n - k]
            e = extra[a]
            for k in range(h):
                moved[h + n + e + k] = moved[h + e + k]
        for patch in self.patches:
            index = tuple(
                slice(lo, hi + e + 2 * h) for (lo, hi), e in zip(patch.box, extra, strict=True)
            )
            patch.field(name).local_with_halos[...] = level[index]

    def add_patch(self, level, box):
        raise NotImplementedError("the one-level stand-in has no refinement")

    def regrid(self, tags, **options):
        raise NotImplementedError("the one-level stand-in has no refinement")


class FluxRegister:
    def __init__(self, hierarchy, cells=None):
        self.hierarchy = hierarchy

    def reset(self):
        return None

    def update(self, name, fluxes, dt, scale=1.0):
        spacing = self.hierarchy.spacing(0)
        for patch in self.hierarchy.patches:
            parts = fluxes(patch)
            divergence = 0.0
            for a, flux in enumerate(parts):
                divergence = divergence + np.diff(flux, axis=a) / spacing[a]
            patch.field(name).local[...] -= dt * divergence

    def reflux(self, name):
        return None


# -- cunumpy -----------------------------------------------------------------------------
class _Kernel:
    def __init__(self, module_name):
        self.module_name = module_name
        self.short = module_name.rsplit(".", 1)[1]

    def _function(self):
        module = importlib.import_module(f"{self.module_name}.{self.short}_{_CHOICE[0]}")
        return getattr(module, self.short)

    def __call__(self, *args):
        return self._function()(*args)

    def selected(self):
        return _CHOICE[0]


class KernelPackage:
    def __init__(self, name):
        self.name = name

    def from_folder(self, module_name, missing_cuda="fallback"):
        return _Kernel(module_name)


@contextlib.contextmanager
def use_host_kernel_implementation(which):
    previous = _CHOICE[0]
    _CHOICE[0] = {"pyccel": "pyccel", "numpy": "numpy"}[which]
    try:
        yield
    finally:
        _CHOICE[0] = previous


def install(reference_src):
    """Register the stubs and a ``carafe`` package object over ``reference_src/carafe``."""
    modules = {}
    methodcard = types.ModuleType("methodcard")
    methodcard.method = _identity_decorator
    methodcard.ConvergenceProblem = ConvergenceProblem
    modules["methodcard"] = methodcard
    profiler = types.ModuleType("scope_profiler")
    profiler.profile = _identity_decorator
    modules["scope_profiler"] = profiler
    xarray = types.ModuleType("xarray")
    xarray.Dataset = Dataset
    xarray.Variable = Variable
    modules["xarray"] = xarray
    mpi = types.ModuleType("maybempi")
    mpi.MPI = _MPI
    modules["maybempi"] = mpi
    patchwork = types.ModuleType("patchwork")
    patchwork.AMRHierarchy = AMRHierarchy
    patchwork.FluxRegister = FluxRegister
    patchwork.Patch = Patch
    modules["patchwork"] = patchwork
    cunumpy = types.ModuleType("cunumpy")
    kernels = types.ModuleType("cunumpy.kernels")
    kernels.KernelPackage = KernelPackage
    kernels.use_host_kernel_implementation = use_host_kernel_implementation
    cunumpy.kernels = kernels
    modules["cunumpy"] = cunumpy
    modules["cunumpy.kernels"] = kernels
    carafe = types.ModuleType("carafe")
    carafe.__path__ = [f"{reference_src}/carafe"]
    modules["carafe"] = carafe
    sys.modules.update(modules)
