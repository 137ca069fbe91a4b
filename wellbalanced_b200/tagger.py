"""Learned refinement tagger: predicts where the plain tagger will flag cells soon.

The reference regrids on its plain tagger, ``current_tags`` (``|J| dx > threshold``,
``carafe/mhd3d.py:771-801``), evaluated on the current state, so a hierarchy regridded
every K steps lags the flow by up to K steps. `LearnedTagger` is a small MLP on 3 x 3 x 3
stencil features of the state (log rho, log p, |B|: values, central differences and the
largest neighbour deviation; ``wb_tag_features``) that predicts which cells the plain
tagger will flag at any of the next K steps; regridding on its tags every K steps keeps
the refined region ahead of the flow. Network: 16 -> 64 -> 64 -> 1 with ReLU, bfloat16
weights and float32 accumulation; forward pass on the tensor cores (``wb_mlp_forward``),
backward pass and Adam on the device (``wb_mlp_backward``, ``wb_mlp_adam``); the float64
NumPy restatement ``oracle/mlp.py`` checks them. The plain tagger stays the referee: the
miss rate is the fraction of its flagged cells the learned tags do not cover.

`multiblast` builds the 3D magnetised multi-blast problem (eight seeded overpressure
spheres, p = 10 in p = 0.1, rho = 1, B = (1, 1, 0)/sqrt(2)); `collect` runs it and pairs
each step's features with the union of the plain tags of the next K steps; `experiment`
trains on the early steps and measures the miss rate and the refined fraction on the later
ones, beside the plain tagger grown by a buffer of cells (what the reference would do to
look ahead).
"""

from __future__ import annotations

import numpy as np
import torch

from wellbalanced_b200 import _lib

FEATURES, HIDDEN, PARAMS = 16, 64, 5313
_W1, _W2, _W3 = slice(0, 1024), slice(1088, 5184), slice(5248, 5312)


class LearnedTagger:
    """The MLP, its Adam state, the feature normalisation and the decision threshold."""

    def __init__(self, *, device="cuda", seed=0, lr=2e-3, betas=(0.9, 0.999), eps=1e-8):
        if not torch.cuda.is_available():
            raise RuntimeError("the learned tagger runs on a CUDA device (there is no CPU path)")
        _lib.load()
        rng = np.random.default_rng(seed)
        p = np.zeros(PARAMS, dtype=np.float32)
        p[_W1] = rng.normal(0.0, np.sqrt(2.0 / FEATURES), _W1.stop - _W1.start)
        p[_W2] = rng.normal(0.0, np.sqrt(2.0 / HIDDEN), _W2.stop - _W2.start)
        p[_W3] = rng.normal(0.0, np.sqrt(1.0 / HIDDEN), _W3.stop - _W3.start)
        self.device = torch.device(device)
        self.params = torch.from_numpy(p).to(self.device)
        self.grads = torch.zeros(PARAMS, dtype=torch.float32, device=self.device)
        self.m = torch.zeros_like(self.grads)
        self.v = torch.zeros_like(self.grads)
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.lr, self.betas, self.eps = float(lr), betas, float(eps)
        self.steps = 0
        self.mean = torch.zeros(FEATURES, dtype=torch.float32, device=self.device)
        self.inv_std = torch.ones(FEATURES, dtype=torch.float32, device=self.device)
        self.threshold = 0.0  # logit above which a cell is tagged

    @staticmethod
    def _s():
        return torch.cuda.current_stream().cuda_stream

    # features ------------------------------------------------------------------------------------
    def features(self, model, *, raw=False):
        """Feature rows (N, 16) of every interior cell of `model`'s patches (3D), patch after
        patch in (i, j, k) order, normalised unless ``raw``; and each patch's first row."""
        eng = model.engine
        if eng.ndim != 3:
            raise ValueError("the stencil features are defined on 3D hierarchies")
        counts = [int(np.prod(p.shape)) for p in model.hierarchy.patches]
        starts = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
        row_start = torch.from_numpy(starts).to(self.device)
        out = torch.empty((int(sum(counts)), FEATURES), dtype=torch.float32, device=self.device)
        mean = torch.zeros_like(self.mean) if raw else self.mean
        inv_std = torch.ones_like(self.inv_std) if raw else self.inv_std
        b = eng.mean_field
        _lib.call("wb_tag_features", eng.precision, eng.state.data_ptr(), eng.patches.data_ptr(),
                  eng.chunk_patch.data_ptr(), eng.chunk_start.data_ptr(), eng.nchunks, row_start.data_ptr(),
                  b[0], b[1], b[2], eng.gamma, mean.data_ptr(), inv_std.data_ptr(), out.data_ptr(), self._s())
        return out, starts

    def fit_normalisation(self, raw):
        """Per-feature mean and 1/std of raw feature rows (constant features keep scale 1)."""
        mean = raw.mean(dim=0)
        std = raw.std(dim=0)
        self.mean = mean.contiguous()
        self.inv_std = torch.where(std > 1e-12, 1.0 / std, torch.ones_like(std)).contiguous()

    def normalise(self, raw):
        return ((raw - self.mean) * self.inv_std).contiguous()

    # network -------------------------------------------------------------------------------------
    def logits(self, X):
        X = X.contiguous()
        out = torch.empty(X.shape[0], dtype=torch.float32, device=self.device)
        _lib.call("wb_mlp_forward", X.data_ptr(), X.shape[0], self.params.data_ptr(), out.data_ptr(), self._s())
        return out

    def gradient(self, X, y, pos_weight=1.0):
        """(summed loss, gradient) of a batch, without an update (the grads are cleared)."""
        self.grads.zero_()
        self.loss.zero_()
        X, y = X.contiguous(), y.to(torch.float32).contiguous()
        _lib.call("wb_mlp_backward", X.data_ptr(), y.data_ptr(), X.shape[0], self.params.data_ptr(),
                  float(pos_weight), self.grads.data_ptr(), self.loss.data_ptr(), self._s())
        out = (float(self.loss.item()), self.grads.clone())
        self.grads.zero_()
        return out

    def train_step(self, X, y, pos_weight=1.0):
        """One Adam step on the mean weighted loss of the batch (returned, on the device)."""
        self.loss.zero_()
        X, y = X.contiguous(), y.to(torch.float32).contiguous()
        _lib.call("wb_mlp_backward", X.data_ptr(), y.data_ptr(), X.shape[0], self.params.data_ptr(),
                  float(pos_weight), self.grads.data_ptr(), self.loss.data_ptr(), self._s())
        self.steps += 1
        _lib.call("wb_mlp_adam", self.params.data_ptr(), self.grads.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                  PARAMS, self.lr, float(self.betas[0]), float(self.betas[1]), self.eps, self.steps,
                  1.0 / X.shape[0], self._s())
        return self.loss / X.shape[0]

    def fit(self, X, y, *, iterations=400, batch=16384, pos_weight=None, seed=0):
        """Mini-batch training on rows X (normalised) and 0/1 targets y; returns the losses."""
        y = y.to(torch.float32)
        positive = float(y.sum().item())
        if pos_weight is None:
            pos_weight = min(50.0, max(1.0, (y.numel() - positive) / max(positive, 1.0)))
        generator = torch.Generator(device=self.device)
        generator.manual_seed(seed)
        losses = []
        for _ in range(iterations):
            index = torch.randint(0, X.shape[0], (min(batch, X.shape[0]),), device=self.device, generator=generator)
            losses.append(self.train_step(X[index], y[index], pos_weight))
        return [float(v.item()) for v in losses]

    def choose_threshold(self, X, y, miss=0.005):
        """Set the logit threshold so that a fraction ``miss`` of the positive rows fall below it."""
        z = self.logits(X)[y.to(torch.bool)]
        self.threshold = float(torch.quantile(z.float(), miss).item()) if z.numel() else 0.0
        return self.threshold

    def predict(self, X):
        return self.logits(X) > self.threshold

    def tags(self, model, levels):
        """Tags per level like ``current_tags``: cells whose logit exceeds the threshold."""
        X, starts = self.features(model)
        flags = self.predict(X).cpu().numpy()
        h = model.hierarchy
        tags = {level: np.zeros(h.level_shape(level), dtype=bool) for level in range(min(levels, h.max_level + 1))}
        for patch, start in zip(h.patches, starts, strict=True):
            if patch.level in tags:
                cells = flags[start : start + int(np.prod(patch.shape))].reshape(patch.shape)
                tags[patch.level][tuple(slice(lo, hi) for lo, hi in patch.box)] |= cells
        return tags


# ---- the multi-blast experiment --------------------------------------------------------------------------
def multiblast(n, *, seed=0, precision=32, limiter="minmod", **options):
    """Eight seeded overpressure spheres (p = 10, radius 0.05-0.1) in rho = 1, p = 0.1 with
    B = (1, 1, 0)/sqrt(2), periodic unit cube of n^3 cells. The limiter defaults to minmod:
    with MC the reference's step itself (the float64 oracle) goes negative at 32^3 after
    11 steps on this problem."""
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D
    from wellbalanced_b200.problems import multi_blast_3d

    field = 1.0 / np.sqrt(2.0)
    model = MHD3D(AMRHierarchy((n,) * 3, ((0.0, 1.0),) * 3, periodic=(True,) * 3), precision=precision,
                  mean_field=(field, field, 0.0), limiter=limiter, cfl=0.3, **options)
    model.set_state(1.0, (0.0, 0.0, 0.0), multi_blast_3d(n, seed=seed))
    return model


def collect(model, tagger, *, steps, horizon, threshold, every=1):
    """Run `model` for ``steps + horizon`` steps; rows of raw level-0 features at every
    ``every``-th step t < steps and, as targets, the union of the plain level-0 tags of steps
    t + 1 .. t + horizon. Also the plain tags of each kept step."""
    tags = []
    feats = []
    for t in range(steps + horizon + 1):
        if t < steps and t % every == 0:
            raw, _ = tagger.features(model, raw=True)
            feats.append((t, raw))
        tags.append(torch.from_numpy(model.current_tags(threshold, 1)[0].ravel()).to(tagger.device))
        model.step()
    X, Y, now = [], [], []
    for t, raw in feats:
        ahead = torch.zeros_like(tags[0])
        for s in range(t + 1, t + horizon + 1):
            ahead |= tags[s]
        X.append(raw)
        Y.append(ahead)
        now.append(tags[t])
    return torch.cat(X), torch.cat(Y), torch.cat(now)


def grow(flags, n, cells):
    """Cells within ``cells`` cells (periodic, a cube) of a flagged cell, for rows of n^3 blocks."""
    blocks = flags.reshape(-1, n, n, n).float()
    if cells <= 0:
        return blocks.bool().reshape(-1)
    k = 2 * cells + 1
    pad = torch.nn.functional.pad(blocks[:, None], (cells,) * 6, mode="circular")
    grown = torch.nn.functional.max_pool3d(pad, kernel_size=k, stride=1)
    return (grown[:, 0] > 0).reshape(-1)


def experiment(n=32, *, train_steps=48, test_steps=24, horizon=8, threshold=0.05, every=2, seed=0,
               iterations=600, miss=0.005):
    """Train on the first steps of one multi-blast run and evaluate on the later ones.

    Returns the training losses and, on the test steps, for the learned tags and for the
    plain tags grown by 0..4 cells: the miss rate (fraction of the cells the plain tagger
    flags within the next ``horizon`` steps that are not tagged) and the tagged fraction.
    """
    tagger = LearnedTagger(seed=seed)
    model = multiblast(n, seed=seed)
    X_raw, Y, now = collect(model, tagger, steps=train_steps + test_steps, horizon=horizon, threshold=threshold,
                            every=every)
    per_step = n**3
    split = (train_steps // every) * per_step
    tagger.fit_normalisation(X_raw[:split])
    X = tagger.normalise(X_raw)
    losses = tagger.fit(X[:split], Y[:split], iterations=iterations, seed=seed)
    tagger.choose_threshold(X[:split], Y[:split], miss=miss)
    pred = tagger.predict(X[split:])
    target = Y[split:]
    total = max(int(target.sum().item()), 1)
    out = {
        "cells": n**3,
        "horizon": horizon,
        "train_rows": split,
        "test_rows": int(target.numel()),
        "loss_first": losses[0],
        "loss_last": float(np.mean(losses[-20:])),
        "learned": {"miss": int((target & ~pred).sum().item()) / total, "tagged": float(pred.float().mean().item())},
        "plain_grown": {},
    }
    for cells in range(5):
        grown = grow(now[split:], n, cells)
        out["plain_grown"][cells] = {"miss": int((target & ~grown).sum().item()) / total,
                                     "tagged": float(grown.float().mean().item())}
    return out, tagger


# ---- regridding on the learned tags: the interval the tags allow -----------------------------------
def covered(model, level):
    """Cells of `level` under a patch of the next level (bool, the level's shape)."""
    h = model.hierarchy
    out = np.zeros(h.level_shape(level), dtype=bool)
    for p in h.patches_at_level(level + 1):
        out[tuple(slice(lo // 2, (hi + 1) // 2) for lo, hi in p.box)] = True
    return out


def covered_level0(model):
    """Level-0 cells under a level-1 patch (bool, the level-0 shape)."""
    return covered(model, 0)


def amr_run(model, tags_of, *, interval, steps, threshold, levels=1, buffer=1, max_patch_size=8, uniform=None):
    """Advance a model with `levels` refined levels for `steps` steps, regridding on
    ``tags_of(model)`` (tags per level, as ``current_tags``) before every ``interval``-th
    step (the first regrid repeated `levels` times, so that every level exists from the
    start); after each step the plain tagger scores the hierarchy: the fraction of the
    level-0 cells it flags (|J| dx > threshold) that no level-1 patch covers.

    The flags come from ``uniform``, a uniform run of the same problem advanced in lockstep
    (the refined run's dt), when given: the plain tagger on the refined run's own level 0
    also flags the coarse cells beside each coarse-fine boundary, where the central
    differences straddle restricted fine values, and those flags follow the patches rather
    than the flow. Without it, the refined run's own level-0 flags.

    Returns the largest such miss over the steps, the mean fraction of level-0 cells under
    level 1 (the refinement's cost), the mean count of refined cells, the regrid count and
    the seconds spent regridding and stepping."""
    import time

    import torch

    worst, refined, fine_cells, regrids = 0.0, [], [], 0
    regrid_seconds = step_seconds = 0.0
    for t in range(steps):
        if t % interval == 0:
            start = time.perf_counter()
            for _ in range(levels if t == 0 else 1):
                tags = tags_of(model)
                model.regrid({lev: tags[lev] for lev in tags if lev < levels}, buffer=buffer,
                             max_patch_size=max_patch_size)
            regrids += 1
            torch.cuda.synchronize()
            regrid_seconds += time.perf_counter() - start
        start = time.perf_counter()
        dt = model.step()
        if uniform is not None:
            uniform.step(dt)
        torch.cuda.synchronize()
        step_seconds += time.perf_counter() - start
        flagged = (uniform if uniform is not None else model).current_tags(threshold, 1)[0]
        under = covered(model, 0)
        if flagged.any():
            worst = max(worst, float((flagged & ~under).sum()) / float(flagged.sum()))
        refined.append(float(under.mean()))
        fine_cells.append(sum(int(np.prod(p.shape)) for p in model.hierarchy.patches if p.level > 0))
    return {"miss": worst, "refined": float(np.mean(refined)), "refined_cells": float(np.mean(fine_cells)),
            "regrids": regrids, "regrid_seconds": regrid_seconds, "step_seconds": step_seconds}


def interval_study(n=32, *, intervals=(2, 4, 8), train_steps=48, test_steps=24, threshold=0.05, seed=0,
                   iterations=600, miss=0.005, levels=1, buffer=1, max_patch_size=8, every=2, fallback=True):
    """The regrid interval each tagger reaches on the multi-blast run with `levels` refined levels.

    For every interval K: a tagger trained on the first ``train_steps`` steps of a uniform
    run to predict the plain flags of the next K steps, then two refined runs over the next
    ``test_steps`` steps from the same state, one regridded every K steps on the learned
    tags, one on the plain tags of the regrid step (``current_tags``, grown by the
    clustering's ``buffer`` like the other); the plain tagger on a uniform run of the same
    problem advanced in lockstep scores both after every step.
    With ``fallback`` the learned run regrids on the union of the learned tags and the plain
    tags of the regrid step (the plain tagger as the fallback: every cell it flags now is
    refined, the learned tags add the cells it will flag). The interval a tagger reaches is
    the largest K whose worst miss stays under 1%."""
    out = {"cells": n**3, "threshold": threshold, "intervals": {}}
    for K in intervals:
        tagger = LearnedTagger(seed=seed)
        model = multiblast(n, seed=seed)
        X_raw, Y, _ = collect(model, tagger, steps=train_steps, horizon=K, threshold=threshold, every=every)
        tagger.fit_normalisation(X_raw)
        X = tagger.normalise(X_raw)
        tagger.fit(X, Y, iterations=iterations, seed=seed)
        tagger.choose_threshold(X, Y, miss=miss)
        runs = {}
        def learned(m, tagger=tagger):
            tags = tagger.tags(m, levels)
            if fallback:
                plain = m.current_tags(threshold, levels)
                tags = {lev: tags[lev] | plain[lev] for lev in tags}
            return tags

        for name, tags_of in (("learned", learned), ("plain", lambda m: m.current_tags(threshold, levels))):
            model = multiblast(n, seed=seed)
            model.advance(train_steps)
            uniform = multiblast(n, seed=seed)
            uniform.advance(train_steps)
            runs[name] = amr_run(model, tags_of, interval=K, steps=test_steps, threshold=threshold, levels=levels,
                                 buffer=buffer, max_patch_size=max_patch_size, uniform=uniform)
        out["intervals"][K] = runs
    for name in ("learned", "plain"):
        ok = [K for K in intervals if out["intervals"][K][name]["miss"] < 0.01]
        out[f"{name}_interval"] = max(ok) if ok else 0
    return out
