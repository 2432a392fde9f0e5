"""Mixed-precision path (FP32 opacities/optics, FP64 solves and sums) vs the
FP64 oracle.  Tolerances: 1e-3 relative on fluxes; 1e-2 K/sol on heating
rates, taken as the temperature tendency dT/dt = QRAD*OM in K per sol."""
import numpy as np
import pytest

import oracle
from helpers import mixed_errors
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu
FLUX_TOL, HEAT_TOL = 1e-3, 1e-2


@pytest.fixture(scope="module")
def rtm(data_dir):
    h = abi.Radiation(data_dir, max_layers=99, precision=abi.MIXED, validate=True)
    yield h
    h.close()


@pytest.mark.parametrize("ncol,L,cloud,seed", [(512, 24, True, 41), (512, 24, False, 42),
                                               (128, 36, True, 43), (96, 48, True, 44)])
def test_mixed_within_tolerance(rtm, otables, ncol, L, cloud, seed):
    b = synth.make_batch(ncol, L=L, seed=seed, cloud=cloud)
    ref = oracle.run_batch(otables, b)
    err = mixed_errors(b, rtm.run(b), ref)
    print(err)
    assert err["flux_max"] <= FLUX_TOL, err
    assert err["heat_dT_Ksol_max"] <= HEAT_TOL, err


@pytest.mark.parametrize("L", [24, 48, 99])
def test_mixed_onchip_solver_within_tolerance(data_dir, otables, L):
    """MIXED with the on-chip solver form, against the oracle."""
    b = synth.make_batch(256 if L < 99 else 16, L=L, seed=45 + L, cloud=True)
    ref = oracle.run_batch(otables, b)
    rt = abi.Radiation(data_dir, max_layers=L, precision=abi.MIXED, validate=True, solver=abi.SOLVER_ONCHIP)
    try:
        err = mixed_errors(b, rt.run(b), ref)
    finally:
        rt.close()
    assert err["flux_max"] <= FLUX_TOL, err
    assert err["heat_dT_Ksol_max"] <= HEAT_TOL, err
