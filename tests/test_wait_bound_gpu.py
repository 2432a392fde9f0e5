"""The kernels' device waits are bounded: a wait that can never be satisfied
(an mbarrier armed for bytes that no copy delivers, waited on with the same
bounded wait the reduce kernel uses) gives up after about a second, sets the
status word, and the kernel returns normally -- no fault, no hang -- so the
handle stays usable."""
import pytest

import oracle
from helpers import compare, to_numpy
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu


def test_unsatisfiable_wait_gives_up_and_reports(data_dir, otables):
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=True)
    try:
        sec = rt.check_wait_bound()
        assert 0.1 < sec < 10.0, sec
        b = synth.make_batch(16, L=24, seed=101, cloud=True)
        err = compare(b, to_numpy(rt.run(b)), oracle.run_batch(otables, b), 1e-12)
        assert max(err.values()) <= 1e-12, err
        assert rt.stats()["status"] == 0
    finally:
        rt.close()
