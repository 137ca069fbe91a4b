"""A small labelled-array container returned by ``dataset()``.

The reference returns an ``xarray.Dataset`` (``carafe/datasets.py:25-30``); xarray is
not a dependency here, so this mirrors the part of its interface the reference's tests
and examples use: ``ds["name"].values``, ``ds.name``, ``ds.data_vars``, ``ds.attrs``,
coordinates ``ds.x.values``, ``.min()`` / ``.max()``, element-wise arithmetic of
variables and ``long_name`` attributes.
"""

from __future__ import annotations

import numpy as np


class Variable:
    def __init__(self, dims, values, long_name="", units=""):
        self.dims = (dims,) if isinstance(dims, str) else tuple(dims)
        self.values = np.asarray(values)
        self.attrs = {"long_name": long_name}
        if units:
            self.attrs["units"] = units

    def min(self):
        return Variable((), np.nanmin(self.values))

    def max(self):
        return Variable((), np.nanmax(self.values))

    def __float__(self):
        return float(self.values)

    def __array__(self, dtype=None, copy=None):
        return np.asarray(self.values, dtype=dtype)

    # element-wise arithmetic with numbers, arrays and variables of the same dims, as
    # xarray does for aligned variables (``ds.pressure / ds.density``)
    def _apply(self, other, op):
        return Variable(self.dims, op(self.values, np.asarray(other)))

    def __add__(self, other):
        return self._apply(other, np.add)

    def __radd__(self, other):
        return self._apply(other, lambda a, b: b + a)

    def __sub__(self, other):
        return self._apply(other, np.subtract)

    def __rsub__(self, other):
        return self._apply(other, lambda a, b: b - a)

    def __mul__(self, other):
        return self._apply(other, np.multiply)

    def __rmul__(self, other):
        return self._apply(other, lambda a, b: b * a)

    def __truediv__(self, other):
        return self._apply(other, np.true_divide)

    def __rtruediv__(self, other):
        return self._apply(other, lambda a, b: b / a)

    def __neg__(self):
        return Variable(self.dims, -self.values)

    def __abs__(self):
        return Variable(self.dims, np.abs(self.values))

    def __repr__(self):
        return f"Variable(dims={self.dims}, shape={self.values.shape})"


class Dataset:
    def __init__(self, data, coords=None, attrs=None):
        self._data = dict(data)
        self._coords = dict(coords or {})
        self.attrs = dict(attrs or {})

    @property
    def data_vars(self):
        return list(self._data)

    @property
    def coords(self):
        return dict(self._coords)

    def __getitem__(self, name):
        if name in self._data:
            return self._data[name]
        return self._coords[name]

    def __contains__(self, name):
        return name in self._data or name in self._coords

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        try:
            return self[name]
        except KeyError as error:
            raise AttributeError(name) from error

    def __repr__(self):
        return f"Dataset(vars={self.data_vars}, attrs={self.attrs})"
