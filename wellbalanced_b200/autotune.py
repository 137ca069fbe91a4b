"""Autotuner of the stage kernels' schedule and tile shapes.

The 3D stage kernel marches each 16 x 16 or 8 x 16 (y, z) tile over ``lx`` x-planes: a
longer march reads fewer halo planes per cell (two extra planes per tile) but gives fewer
tiles to spread over the 148 SMs, and the smaller tile fits twice the CTAs on an SM at
more halo work per cell, so the best pair depends on the patch sizes. The 2D
stage kernel is built for a few tile shapes (``wb_tile_shapes``): small tiles waste less
of small patches and give more blocks, large ones re-read fewer halo cells. `tune_lx` and
`tune_tile2d` time the stage kernel (its stage-1 form, which writes only the scratch pool)
on an engine's own layout and state for each candidate and keep the fastest; results are
remembered per (precision, limiter, patch shapes) for the process. ``MHD3D(...,
lx="auto")`` and ``MHD2D(..., tile="auto")`` tune when their state is first set.
"""

from __future__ import annotations

import torch

from wellbalanced_b200 import _lib

CANDIDATES = (8, 16, 32, 64, 128)
_CACHE: dict[tuple, object] = {}


def _key(engine):
    shapes = tuple(sorted({tuple(int(v) for v in r["n"]) for r in engine.layout.rows}))
    return (engine.precision, engine.limiter, shapes)


def _set_lx(engine, lx):
    layout = engine.layout
    layout.lx = int(lx)
    layout._tiles()
    from wellbalanced_b200.engine import _device_bytes

    engine.tiles = _device_bytes(layout.tiles, engine.device, _lib.TILE)
    engine.ntiles = int(layout.tiles.size)


def tune_lx(engine, candidates=CANDIDATES, repeats=5, use_cache=True):
    """The fastest (tile shape, x-march length) of the 3D stage kernel for `engine`; the
    engine is left set to it (the non-ideal kernel keeps the default shape and tunes the
    march only).

    Returns ``(lx, {"TYxTZ/lx": mean ms per stage launch})`` (an empty dict when cached);
    the chosen shape is ``engine.layout.tile_shape``."""
    if engine.ndim != 3:
        raise ValueError("the x-march length applies to the 3D stage kernel")
    key = _key(engine) + (engine.physics is not None,)
    if use_cache and key in _CACHE:
        tile, lx = _CACHE[key]
        engine.layout.set_tile(tile)
        _set_lx(engine, lx)
        return lx, {}
    longest = max(int(r["n"][0]) + 1 for r in engine.layout.rows)
    shapes = _lib.tile_shapes(3, engine.precision)
    if engine.physics is not None:
        shapes = shapes[:1]
    timings = {}
    bad = engine.bad.clone()
    for tile in shapes:
        engine.layout.set_tile(tile)
        for lx in candidates:
            if lx > 2 * longest and lx != candidates[0]:
                continue
            _set_lx(engine, lx)
            engine.stage(engine.state, None, engine.stage_pool)  # warm-up
            torch.cuda.synchronize(engine.device)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            for _ in range(repeats):
                engine.stage(engine.state, None, engine.stage_pool)
            end.record()
            torch.cuda.synchronize(engine.device)
            timings[(tile, lx)] = start.elapsed_time(end) / repeats
    engine.bad.copy_(bad)
    best_tile, best_lx = min(timings, key=timings.get)
    engine.layout.set_tile(best_tile)
    _set_lx(engine, best_lx)
    _CACHE[key] = (best_tile, best_lx)
    return best_lx, {f"{t[0]}x{t[1]}/{lx}": ms for (t, lx), ms in timings.items()}


def _set_tile(engine, tile):
    from wellbalanced_b200.engine import _device_bytes

    engine.layout.set_tile(tile)
    engine.tiles = _device_bytes(engine.layout.tiles, engine.device, _lib.TILE)
    engine.ntiles = int(engine.layout.tiles.size)


def tune_tile2d(engine, repeats=5, use_cache=True):
    """The fastest tile shape of the 2D stage kernel for `engine`; the engine is left set
    to it. Returns ``((tx, ty), {"TXxTY": mean ms per stage launch})`` (an empty dict when
    cached). Ideal MHD only: the non-ideal kernel runs on the default tiles."""
    if engine.ndim != 2:
        raise ValueError("the tile shapes apply to the 2D stage kernel")
    if engine.physics is not None:
        raise ValueError("the non-ideal 2D kernel runs on the default tile shape")
    key = ("tile2d", *_key(engine))
    if use_cache and key in _CACHE:
        _set_tile(engine, _CACHE[key])
        return _CACHE[key], {}
    timings = {}
    bad = engine.bad.clone()
    for tile in _lib.tile_shapes_2d(engine.precision):
        _set_tile(engine, tile)
        engine.stage(engine.state, None, engine.stage_pool)  # warm-up
        torch.cuda.synchronize(engine.device)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(repeats):
            engine.stage(engine.state, None, engine.stage_pool)
        end.record()
        torch.cuda.synchronize(engine.device)
        timings[tile] = start.elapsed_time(end) / repeats
    engine.bad.copy_(bad)
    best = min(timings, key=timings.get)
    _set_tile(engine, best)
    _CACHE[key] = best
    return best, {f"{tx}x{ty}": ms for (tx, ty), ms in timings.items()}


def describe(timings):
    return {str(k): round(float(v), 4) for k, v in sorted(timings.items())} if timings else None

