"""FP64 CUDA path vs the oracle, through the C ABI (host and device pointers).

Tolerance: 1e-12 relative on fluxes (floor 1e-3 of the column's flux scale),
1e-12 of the column flux scale on SUNTOT/IRTOTAL and scalars, the same scaled
by 1/(CP*YM*OM) on QRAD; DETAU/CUMTAUV 1e-12 relative.  Bins (tpindex,
Planck index) are exercised at their edges: a wrong bin moves fluxes by far
more than the tolerance."""
import numpy as np
import pytest

import oracle
from helpers import compare, edge_batch, to_numpy
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu
RTOL = 1e-12


@pytest.fixture(scope="module")
def rt(data_dir):
    h = abi.Radiation(data_dir, max_layers=99, precision=abi.FP64, validate=True)
    yield h
    h.close()


def check(b, got, ref, rtol=RTOL):
    err = compare(b, to_numpy(got), ref, rtol)
    bad = {k: v for k, v in err.items() if not v <= rtol}
    assert not bad, f"max normalised errors above {rtol}: {bad}"
    return err


@pytest.mark.parametrize("ncol,L,cloud,seed", [
    (192, 24, False, 1), (192, 24, True, 2), (96, 36, True, 3), (64, 48, True, 4),
    (16, 1, True, 5), (8, 99, True, 6), (1, 24, True, 7)])
def test_fp64_matches_oracle(rt, otables, ncol, L, cloud, seed):
    b = synth.make_batch(ncol, L=L, seed=seed, cloud=cloud)
    ref = oracle.run_batch(otables, b)
    got = rt.run(b)
    check(b, got, ref)


def test_device_pointers_match_host(rt, otables):
    import torch
    b = synth.make_batch(128, L=24, seed=11, cloud=True)
    ref = oracle.run_batch(otables, b)
    bd = {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
          for k, v in b.items()}
    got = rt.run(bd)
    check(b, got, ref)


def test_edges_match_oracle(rt, otables):
    b = edge_batch(otables)
    ref = oracle.run_batch(otables, b)
    assert ref["fluxdnv"][11].sum() == 0.0 and ref["fluxdnv"][10].sum() > 0.0
    got = rt.run(b)
    check(b, got, ref)


def test_all_night_and_all_day(rt, otables):
    for nf in (0.0, 1.0):
        b = synth.make_batch(64, L=24, seed=13, cloud=True, night_frac=nf)
        check(b, rt.run(b), oracle.run_batch(otables, b))


def test_uneven_multi_grid_batch(rt, otables):
    bs = [synth.make_batch(40, L=24, seed=21, cloud=True),
          synth.make_batch(30, L=36, seed=22, cloud=True),
          synth.make_batch(20, L=48, seed=23, cloud=False)]
    outs = rt.run_multi(bs)
    for b, o in zip(bs, outs):
        check(b, o, oracle.run_batch(otables, b))


def test_empty_batch(rt):
    b = synth.make_batch(1, L=24, seed=1)
    b["ncol"] = 0
    for k, v in list(b.items()):
        if isinstance(v, np.ndarray) and k not in ("sigma", "sol"):
            b[k] = v[:0]
    out = rt.run(b)
    assert out["qrad"].shape == (0, 25)


def test_dsolflux_matches_oracle(rt, otables):
    b = synth.make_batch(200, L=24, seed=14)
    ref = oracle.run_batch(otables, b)
    ds_ref = oracle.dsolflux(otables, b["sol"], b["acosz"], ref["detau"]) + ref["dndiffv"]
    got = rt.dsolflux(b["sol"], b["acosz"], ref["detau"], ref["dndiffv"])
    np.testing.assert_allclose(got, ds_ref, rtol=1e-12, atol=1e-12)


def test_input_errors_are_status_codes(rt):
    b = synth.make_batch(8, L=24, seed=15)
    bad = dict(b)
    bad["tmid"] = b["tmid"].copy()
    bad["tmid"][3, 10] = np.nan
    with pytest.raises(abi.RTError) as e:
        rt.run(bad)
    assert e.value.code == -2
    bad = dict(b)
    bad["tlev"] = b["tlev"].copy()
    bad["tlev"][2, 20] = 40.0
    with pytest.raises(abi.RTError) as e:
        rt.run(bad)
    assert e.value.code == -3
    bad = dict(b)
    bad["L"] = 100
    with pytest.raises(abi.RTError) as e:
        rt.run(bad)
    assert e.value.code == -4
    bad = dict(b)
    bad["qh2o"] = None
    with pytest.raises(abi.RTError) as e:
        rt.run(bad)
    assert e.value.code == -1
    # the handle is still usable afterwards
    rt.run(b)


@pytest.mark.parametrize("L", [1, 2, 3, 5, 24, 27, 28, 36, 48, 51])
def test_four_lane_and_thread_solvers_match_oracle(data_dir, otables, L):
    """Every solver form (one thread per system with its arrays in local
    memory; four lanes per system for L <= 51; one thread per system with its
    arrays on chip, in shared memory or in tensor memory and shared memory;
    the persistent fused kernel) reproduces the oracle at 1e-12, at layer
    counts that split unevenly over the four lanes."""
    b = synth.make_batch(48, L=L, seed=900 + L, cloud=True)
    ref = oracle.run_batch(otables, b)
    for solver in (abi.SOLVER_THREAD, abi.SOLVER_QUAD, abi.SOLVER_ONCHIP, abi.SOLVER_TMEM, abi.SOLVER_FUSED):
        rt = abi.Radiation(data_dir, max_layers=max(L, 1), precision=abi.FP64, validate=True, solver=solver)
        try:
            err = compare(b, to_numpy(rt.run(b)), ref, RTOL)
            assert max(err.values()) <= RTOL, (solver, err)
        finally:
            rt.close()
