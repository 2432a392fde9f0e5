"""The seeded input generators behind every parity test and benchmark:
the same seed gives the same columns, and the GCM-state batch is the column
state of the tracer batch it is derived from."""
import numpy as np

import oracle
from mgcm_rt import synth


def _same(a, b):
    for k, v in a.items():
        if isinstance(v, np.ndarray):
            np.testing.assert_array_equal(v, b[k], err_msg=k)


def test_generators_are_reproducible():
    _same(synth.make_batch(40, L=24, seed=5, cloud=True), synth.make_batch(40, L=24, seed=5, cloud=True))
    _same(synth.make_tracer_batch(40, L=36, seed=6), synth.make_tracer_batch(40, L=36, seed=6))
    _same(synth.make_state_batch(40, L=48, seed=7), synth.make_state_batch(40, L=48, seed=7))
    a = synth.make_batch(40, L=24, seed=5, cloud=True)
    b = synth.make_batch(40, L=24, seed=6, cloud=True)
    assert not np.array_equal(a["tlev"], b["tlev"])


def test_state_batch_matches_its_tracer_batch():
    """The state's layer temperatures, TSTRAT and GT are the tracer batch's
    TLEV at the even levels, level 1 and the ground, and the prep rebuilds
    that batch's PLEV and even-level TLEV exactly."""
    L = 24
    tb = synth.make_tracer_batch(32, L=L, seed=9, active_dust=False, cloudon=True)
    st = synth.make_state_batch(32, L=L, seed=9, active_dust=False, cloudon=True)
    lev = 2 * L + 3
    np.testing.assert_array_equal(st["t"], tb["tlev"][:, 3:lev - 1:2])
    np.testing.assert_array_equal(st["tstrat"], tb["tlev"][:, 0])
    np.testing.assert_array_equal(st["gt"], tb["tlev"][:, lev - 1])
    got = oracle.prep(st)
    np.testing.assert_array_equal(got["plev"], tb["plev"])
    np.testing.assert_array_equal(got["tlev"][:, 3:lev - 1:2], tb["tlev"][:, 3:lev - 1:2])
    assert np.all(got["tauref"] >= 0.0)
