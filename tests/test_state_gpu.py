"""mgcm_rt_run_state: the column prep (PL, FILLPT, QH2O, DUSTPROFILE +
FILLTAUCUM) on the device from the GCM state, then the aerosol optics and
the radiation.  The prepared level arrays equal the oracle's restatement
bit for bit; the FP64 results equal the oracle chain (prep, aerosols,
radiation) to 1e-12 and mgcm_rt_run_tracers on the oracle's prepared arrays
bit for bit; MIXED stays within its tolerances."""
import numpy as np
import pytest

import oracle
from helpers import compare, mixed_errors, to_numpy
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu

CASES = [  # active_dust, cloudon, active_water, vary_conr
    (0, 1, 1, 0),
    (0, 0, 0, 1),
    (1, 1, 1, 0),
    (1, 0, 0, 0),
]


@pytest.fixture(scope="module")
def aero(data_dir):
    return oracle.AeroTables(data_dir)


def _device(t):
    import torch
    return {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
            for k, v in t.items()}


def _state(ncol, L, seed, case):
    d, c, w, v = case
    return synth.make_state_batch(ncol, L=L, seed=seed, active_dust=bool(d), cloudon=bool(c),
                                  active_water=bool(w), vary_conr=bool(v))


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("L", [24, 36, 48])
def test_state_prep_bit_exact_and_fp64_parity(data_dir, otables, aero, case, L):
    st = _state(193, L, 700 + L + 7 * CASES.index(case), case)
    tb = oracle.prep(st)
    ref = oracle.run_batch(otables, oracle.aerosols(aero, tb))
    rt = abi.Radiation(data_dir, max_layers=48, precision=abi.FP64, validate=True)
    try:
        for s in (st, _device(st)):
            got = to_numpy(rt.run_state(s, return_levels=True))
            for k in abi.PREP_FIELDS:
                if tb[k] is None:
                    assert k not in got
                    continue
                np.testing.assert_array_equal(got[k], tb[k], err_msg=k)
            err = compare(tb, got, ref, 1e-12)
            assert max(err.values()) <= 1e-12, err
    finally:
        rt.close()


@pytest.mark.parametrize("L", [1, 2, 99])
def test_state_layer_count_edges(data_dir, otables, aero, L):
    """The smallest layer counts (FILLPT's interpolation loop empty or one
    level long) and the largest the library accepts."""
    st = _state(65, L, 790 + L, CASES[0])
    tb = oracle.prep(st)
    ref = oracle.run_batch(otables, oracle.aerosols(aero, tb))
    rt = abi.Radiation(data_dir, max_layers=99, precision=abi.FP64, validate=True)
    try:
        got = to_numpy(rt.run_state(st, return_levels=True))
        for k in abi.PREP_FIELDS:
            np.testing.assert_array_equal(got[k], tb[k], err_msg=k)
        err = compare(tb, got, ref, 1e-12)
        assert max(err.values()) <= 1e-12, err
    finally:
        rt.close()


def test_state_equals_tracers_on_prepared_arrays(data_dir):
    """After the prep the device path is the tracer path: same bits."""
    st = _state(300, 24, 760, CASES[0])
    tb = oracle.prep(st)
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        a = to_numpy(rt.run_state(st))
        b = to_numpy(rt.run_tracers(tb))
        for k in b:
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    finally:
        rt.close()


@pytest.mark.parametrize("case", [CASES[0], CASES[2]])
def test_state_mixed_within_tolerance(data_dir, otables, aero, case):
    st = _state(512, 24, 761 + CASES.index(case), case)
    tb = oracle.prep(st)
    ref = oracle.run_batch(otables, oracle.aerosols(aero, tb))
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.MIXED, validate=True)
    try:
        got = rt.run_state(st, return_levels=True)
        for k in abi.PREP_FIELDS:   # the prep is FP64 in both modes
            if tb[k] is not None:
                np.testing.assert_array_equal(got[k], tb[k], err_msg=k)
        err = mixed_errors(tb, got, ref)
        assert err["flux_max"] <= 1e-3 and err["heat_dT_Ksol_max"] <= 1e-2, err
    finally:
        rt.close()


def test_state_large_batch_crosses_jobs(data_dir, otables, aero):
    """More columns than one job: each job preps its own column range."""
    st = _state(20000, 24, 762, CASES[0])
    got = None
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        got = to_numpy(rt.run_state(st, return_levels=True))
    finally:
        rt.close()
    for sl in (slice(0, 200), slice(8100, 8300), slice(-200, None)):
        sub = {k: (v[sl] if isinstance(v, np.ndarray) and k not in ("sigma", "sol") else v)
               for k, v in st.items()}
        sub["ncol"] = 200
        tb = oracle.prep(sub)
        for k in abi.PREP_FIELDS:
            np.testing.assert_array_equal(got[k][sl], tb[k], err_msg=k)
        ref = oracle.run_batch(otables, oracle.aerosols(aero, tb))
        err = compare(tb, {k: v[sl] for k, v in got.items()}, ref, 1e-12)
        assert max(err.values()) <= 1e-12, err


def test_state_single_and_empty(data_dir, otables, aero):
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=True)
    try:
        st = _state(1, 24, 763, CASES[0])
        tb = oracle.prep(st)
        ref = oracle.run_batch(otables, oracle.aerosols(aero, tb))
        err = compare(tb, to_numpy(rt.run_state(st)), ref, 1e-12)
        assert max(err.values()) <= 1e-12, err
        empty = _state(1, 24, 763, CASES[0])
        empty = {k: (v[:0] if isinstance(v, np.ndarray) and k not in ("sigma", "sol") else v)
                 for k, v in empty.items()}
        empty["ncol"] = 0
        out = rt.run_state(empty)
        assert out["qrad"].shape == (0, 25)
    finally:
        rt.close()


def test_state_argument_errors(data_dir):
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        st = _state(4, 24, 764, CASES[0])
        for bad, code in ((dict(st, tautot=None), -1), (dict(st, vapour=None), -1),
                          (dict(st, t=np.zeros((4, 24)), tstrat=None), -1),
                          (dict(st, L=30), -4), (dict(st, psf=float("nan")), -2),
                          (dict(st, rptau=0.0), -2)):
            with pytest.raises(abi.RTError) as e:
                rt.run_state(bad)
            assert e.value.code == code
    finally:
        rt.close()
