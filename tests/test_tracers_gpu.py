"""mgcm_rt_run_tracers: aerosol optics on the device from tracer mixing
ratios (OPT_DST / prescribed dust / OPT_CLD), then the radiation.  FP64
results equal the oracle's aerosol restatement followed by the oracle
radiation to 1e-12; MIXED stays within its tolerances."""
import numpy as np
import pytest

import oracle
from helpers import compare, mixed_errors, to_numpy
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def aero(data_dir):
    return oracle.AeroTables(data_dir)


def _device(t):
    import torch
    return {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
            for k, v in t.items()}


@pytest.mark.parametrize("active_dust,cloudon", [(1, 1), (0, 1), (1, 0), (0, 0)])
@pytest.mark.parametrize("L", [24, 36])
def test_tracers_fp64_match_oracle(data_dir, otables, aero, active_dust, cloudon, L):
    tb = synth.make_tracer_batch(257, L=L, seed=400 + 10 * L + 2 * active_dust + cloudon,
                                 active_dust=bool(active_dust), cloudon=bool(cloudon))
    ref = oracle.run_batch(otables, oracle.aerosols(aero, tb))
    rt = abi.Radiation(data_dir, max_layers=48, precision=abi.FP64, validate=True)
    try:
        for t in (tb, _device(tb)):
            err = compare(tb, to_numpy(rt.run_tracers(t)), ref, 1e-12)
            assert max(err.values()) <= 1e-12, err
    finally:
        rt.close()


def test_tracers_mixed_within_tolerance(data_dir, otables, aero):
    tb = synth.make_tracer_batch(512, L=24, seed=450, active_dust=True, cloudon=True)
    ref = oracle.run_batch(otables, oracle.aerosols(aero, tb))
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.MIXED, validate=True)
    try:
        err = mixed_errors(tb, rt.run_tracers(tb), ref)
        assert err["flux_max"] <= 1e-3 and err["heat_dT_Ksol_max"] <= 1e-2, err
    finally:
        rt.close()


def test_tracers_large_batch_crosses_jobs(data_dir, otables, aero):
    """More columns than one job: the two slots alternate."""
    tb = synth.make_tracer_batch(40000, L=24, seed=451, active_dust=True, cloudon=True)
    sub = {k: (v[:300] if isinstance(v, np.ndarray) and k not in ("sigma", "sol") else v) for k, v in tb.items()}
    sub["ncol"] = 300
    sub2 = {k: (v[-300:] if isinstance(v, np.ndarray) and k not in ("sigma", "sol") else v) for k, v in tb.items()}
    sub2["ncol"] = 300
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        got = to_numpy(rt.run_tracers(tb))
        for s, sl in ((sub, slice(0, 300)), (sub2, slice(-300, None))):
            ref = oracle.run_batch(otables, oracle.aerosols(aero, s))
            part = {k: v[sl] for k, v in got.items()}
            err = compare(s, part, ref, 1e-12)
            assert max(err.values()) <= 1e-12, err
    finally:
        rt.close()


def test_tracers_argument_errors(data_dir):
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        tb = synth.make_tracer_batch(4, L=24, seed=452, active_dust=True, cloudon=True)
        bad = dict(tb, dust_number=None)
        with pytest.raises(abi.RTError) as e:
            rt.run_tracers(bad)
        assert e.value.code == -1
        bad = dict(tb, L=30)
        with pytest.raises(abi.RTError) as e:
            rt.run_tracers(bad)
        assert e.value.code == -4
    finally:
        rt.close()


@pytest.mark.parametrize("active_dust,cloudon", [(0, 1), (1, 1), (0, 0)])
def test_tracers_equal_arrays_path_bitwise(data_dir, aero, active_dust, cloudon):
    """The tracer call (device aerosol optics; prescribed dust read as band
    constants; ice properties read only where TAUREFCLD != 0) gives the same
    bits as the drop-in call on the oracle's full per-level aerosol arrays."""
    tb = synth.make_tracer_batch(300, L=24, seed=470 + 2 * active_dust + cloudon,
                                 active_dust=bool(active_dust), cloudon=bool(cloudon))
    full = oracle.aerosols(aero, tb)
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=True)
    try:
        a = to_numpy(rt.run_tracers(tb))
        b = to_numpy(rt.run(full))
        for k in b:
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    finally:
        rt.close()
