"""The per-phase precision restatement (`oracle.precision`) against the reference's own
run (CPU): in float64 it is the reference's Orszag-Tang step (the committed fixture of
the reference's 32^2 run to t = 0.5 via the oracle), and its float32 variants stay close."""

from __future__ import annotations

import numpy as np


def test_float64_restatement_equals_the_oracle_run():
    from oracle import precision
    from oracle.mhd2d import MHD2D

    n = 32
    model = MHD2D.orszag_tang(n, limiter="mc", cfl=0.4)
    model.run(0.5)
    want = model.state()
    U0, A0 = precision.orszag_tang(n)
    U, _, dts = precision.Step(n, precision.types("")).run(U0, A0)
    assert len(dts) == model.steps
    np.testing.assert_allclose(U[0], want["density"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(U[4], want["energy"], rtol=0, atol=1e-13)


def test_float32_storage_error_is_small_at_32():
    from oracle import precision

    n = 32
    U0, A0 = precision.orszag_tang(n)
    Ur, _, dts = precision.Step(n, precision.types("")).run(U0, A0)
    U, _, _ = precision.Step(n, precision.types("store=32")).run(U0, A0, dts)
    err = np.sum(np.abs(U[0] - Ur[0])) / np.sum(np.abs(Ur[0]))
    assert 0 < err < 1e-5
