"""The learned refinement tagger on the GPU: kernels against the oracle, training, and
what it gains over the plain tagger.

`oracle/mlp.py` (float64 NumPy) checks the stencil features of a 3D state, the forward
pass on the tensor cores and the gradient of the backward kernel; a separable problem
checks that training converges; the magnetised multi-blast run checks the purpose: tags
predicted K steps ahead miss under 1% of the cells the plain current tagger flags within
those steps, where the plain tags of the regrid step miss far more.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _tagger(seed=0):
    from wellbalanced_b200.tagger import LearnedTagger

    return LearnedTagger(seed=seed)


def test_features_match_the_oracle():
    from oracle import mlp
    from wellbalanced_b200.tagger import multiblast

    model = multiblast(12, seed=3, precision=64)
    for _ in range(3):
        model.step()
    tagger = _tagger()
    got, starts = tagger.features(model, raw=True)
    (patch,) = model.hierarchy.patches
    eng = model.engine
    fields = [eng.view(eng.state, patch, f).cpu().numpy() for f in range(8)]
    want = mlp.features(fields, patch.shape, model.hierarchy.spacing(0), mean_field=model.mean_field)
    np.testing.assert_allclose(got.cpu().numpy(), want, rtol=2e-5, atol=2e-5)
    # normalisation is applied in the kernel
    tagger.fit_normalisation(got)
    normed, _ = tagger.features(model)
    np.testing.assert_allclose(normed.cpu().numpy(), tagger.normalise(got).cpu().numpy(), rtol=1e-5, atol=1e-5)


def test_forward_and_gradient_match_the_oracle():
    from oracle import mlp

    rng = np.random.default_rng(4)
    tagger = _tagger(seed=4)
    params = tagger.params.cpu().numpy().astype(np.float64)
    params[1024:1088] = rng.normal(0.0, 0.2, 64)  # biases too
    params[5184:5248] = rng.normal(0.0, 0.2, 64)
    params[5312] = 0.3
    tagger.params.copy_(torch.from_numpy(params.astype(np.float32)))
    params = tagger.params.cpu().numpy().astype(np.float64)
    X = rng.normal(size=(3001, 16)).astype(np.float32)  # not a multiple of 16 or 64 rows
    y = (rng.random(3001) < 0.2).astype(np.float32)
    Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    logits = tagger.logits(Xd).cpu().numpy()
    want, _ = mlp.forward(params, X)
    scale = np.max(np.abs(want))
    assert np.median(np.abs(logits - want)) < 1e-5 * scale
    assert np.max(np.abs(logits - want)) < 2e-3 * scale  # a bfloat16 rounding of h1 may flip
    loss, grad = tagger.gradient(Xd, yd, pos_weight=4.0)
    want_loss, want_grad = mlp.loss_and_gradients(params, X, y, 4.0)
    assert abs(loss - want_loss) < 1e-4 * abs(want_loss)
    grad = grad.cpu().numpy()
    for name, part in mlp.SLICES.items():
        size = np.max(np.abs(want_grad[part]))
        assert np.max(np.abs(grad[part] - want_grad[part])) < 2e-3 * size, name


def test_training_separates_a_simple_rule():
    rng = np.random.default_rng(5)
    tagger = _tagger(seed=5)
    X = rng.normal(size=(40000, 16)).astype(np.float32)
    y = ((X[:, 0] + 0.5 * X[:, 3] > 0.7) | (X[:, 5] < -1.5)).astype(np.float32)
    Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    losses = tagger.fit(Xd, yd, iterations=300, batch=4096, pos_weight=1.0)
    assert losses[-1] < 0.25 * losses[0]
    accuracy = float(((tagger.logits(Xd) > 0).float() == yd).float().mean().item())
    assert accuracy > 0.97


def test_learned_tags_anticipate_the_plain_tagger():
    from wellbalanced_b200.tagger import experiment

    out, _ = experiment(32, train_steps=48, test_steps=24, horizon=8, every=2, iterations=600)
    learned, plain = out["learned"], out["plain_grown"]
    assert out["loss_last"] < out["loss_first"]
    assert learned["miss"] < 0.01
    # the plain tags of the regrid step miss much of what is flagged in the next 8 steps
    assert plain[0]["miss"] > 5 * max(learned["miss"], 1e-3)
    # growing them by the smallest buffer that brings the miss rate under 1% tags more cells
    buffer = min(c for c in plain if plain[c]["miss"] < 0.01)
    assert buffer >= 1 and learned["tagged"] < plain[buffer]["tagged"]


def test_learned_tags_allow_a_longer_regrid_interval():
    """Regridding a refined multi-blast run (32^3 base, one refined level) on the learned
    tags keeps the cells the plain tagger flags on a uniform run of the same problem under
    refined patches (under 1% missed) for a longer regrid interval than regridding on the
    plain tags of the regrid step. Boxes without a buffer: with a buffer cell and the boxes'
    slack, the plain tags of the regrid step already cover the next 32 steps at this size
    (every interval up to 32 misses nothing), so only the tags themselves are compared."""
    from wellbalanced_b200.tagger import interval_study

    out = interval_study(32, intervals=(2, 8), train_steps=32, test_steps=16, buffer=0)
    print({K: {k: round(v["miss"], 4) for k, v in runs.items()} for K, runs in out["intervals"].items()},
          out["learned_interval"], out["plain_interval"])
    assert out["learned_interval"] > out["plain_interval"]
    assert out["intervals"][out["learned_interval"]]["learned"]["miss"] < 0.01
