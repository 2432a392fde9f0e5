"""Device-pointer calls and graphs large enough to run as concurrent parts:
members of three layer counts whose column total splits into 4 parts at
columns that fall inside members, so part boundaries cut segments.  Every
member matches the oracle (FP64: 1e-12), through mgcm_rt_run_multi on device
pointers and through a captured graph, and the DETAU / CUMTAUV arrays the call
updates match too."""
import numpy as np
import pytest

import oracle
from helpers import compare, to_numpy
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu

# 52,000 columns: 4 parts of 13,000, boundaries inside the first, second and
# third members
SPECS = [(20000, 24, 301), (15000, 36, 302), (17000, 48, 303)]


def _device(b):
    import torch
    return {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
            for k, v in b.items()}


def _check(host, outs, otables):
    # outs carry the members' DETAU / CUMTAUV, updated in place on the device
    for b, o in zip(host, outs):
        ref = oracle.run_batch(otables, b)
        err = compare(b, to_numpy(o), ref, 1e-12)
        assert max(err.values()) <= 1e-12, err


def test_run_multi_in_parts_matches_oracle(data_dir, otables):
    rt = abi.Radiation(data_dir, max_layers=48, precision=abi.FP64, validate=True)
    try:
        host = [synth.make_batch(n, L=L, seed=s, cloud=True) for n, L, s in SPECS]
        dev = [_device(b) for b in host]
        outs = rt.run_multi(dev)
        st = rt.stats()
        assert st["columns"] == sum(n for n, _, _ in SPECS) and st["status"] == 0
        assert st["kernels"] >= 4 * 5, st   # four parts of at least five kernels each
        _check(host, outs, otables)
    finally:
        rt.close()


def test_graph_in_parts_matches_oracle(data_dir, otables):
    import torch
    rt = abi.Radiation(data_dir, max_layers=48, precision=abi.FP64, validate=False)
    try:
        host = [synth.make_batch(n, L=L, seed=s, cloud=True) for n, L, s in SPECS]
        dev = [_device(b) for b in host]
        g = rt.graph(dev, autotune=False)
        try:
            assert g.info()["kernels"] >= 4 * 5, g.info()
            for _ in range(2):   # replays are idempotent
                g.launch()
                torch.cuda.synchronize()
                assert g.status() == 0
            _check(host, g.outs, otables)
        finally:
            g.close()
    finally:
        rt.close()
