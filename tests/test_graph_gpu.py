"""Captured uneven batches (mgcm_rt_graph_*): members of different layer
counts in one CUDA graph, autotuned, replayed; every member matches the
oracle (FP64: 1e-12) and the same batches through mgcm_rt_run_multi."""
import numpy as np
import pytest

import oracle
from helpers import compare, to_numpy
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu


def _device(b):
    import torch
    return {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
            for k, v in b.items()}


@pytest.mark.parametrize("autotune", [False, True])
def test_graph_uneven_members_fp64(data_dir, otables, autotune):
    import torch
    rt = abi.Radiation(data_dir, max_layers=48, precision=abi.FP64, validate=False)
    try:
        specs = [(300, 24, 81), (200, 36, 82), (150, 48, 83), (1, 48, 84), (257, 24, 85)]
        host = [synth.make_batch(n, L=L, seed=s, cloud=True) for n, L, s in specs]
        dev = [_device(b) for b in host]
        g = rt.graph(dev, autotune=autotune)
        try:
            info = g.info()
            assert info["columns"] == sum(n for n, _, _ in specs)
            assert info["kernels"] >= 5 and info["candidates"] >= 1
            for _ in range(3):   # replays are idempotent
                g.launch()
                torch.cuda.synchronize()
                assert g.status() == 0
            multi = rt.run_multi(host)
            for b, o, m in zip(host, g.outs, multi):
                ref = oracle.run_batch(otables, b)
                got = to_numpy(o)
                err = compare(b, got, ref, 1e-12)
                assert max(err.values()) <= 1e-12, err
                err = compare(b, got, m, 1e-12)
                assert max(err.values()) <= 1e-12, err
        finally:
            g.close()
    finally:
        rt.close()


def test_graph_rejects_host_batches(data_dir):
    """Host batches are refused: by the wrapper before any C call, and by the
    C ABI itself (device_ptrs = 0 -> EINVAL, nothing launched)."""
    import ctypes as C
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        b = synth.make_batch(8, L=24, seed=86, cloud=True)
        with pytest.raises(ValueError):
            rt.graph([b], outs=[abi.alloc_outputs(8, 24)])
        keep = []
        o = abi.alloc_outputs(8, 24)
        ins = (abi.BatchIn * 1)(abi.make_in(b, False, keep))
        outs = (abi.BatchOut * 1)(abi.make_out(o))
        g = C.c_void_p()
        rc = abi.lib().mgcm_rt_graph_create(rt._h, 1, ins, outs, 0, C.byref(g))
        assert rc == -1 and not g.value
    finally:
        rt.close()
