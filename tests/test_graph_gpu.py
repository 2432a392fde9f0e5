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


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
def test_graph_fused_persistent_kernel(data_dir, otables, precision):
    """The persistent fused form captured as a graph: one kernel launch per
    replay over members of three layer counts, autotuned over its launch
    shapes; FP64 matches the oracle to 1e-12, MIXED stays within 1e-3 on
    fluxes and 1e-2 K/sol on heating."""
    import torch
    from helpers import mixed_errors
    rt = abi.Radiation(data_dir, max_layers=48, precision=precision, validate=False, solver=abi.SOLVER_FUSED)
    try:
        specs = [(400, 24, 91), (250, 36, 92), (180, 48, 93), (1, 36, 94), (333, 24, 95)]
        host = [synth.make_batch(n, L=L, seed=s, cloud=True) for n, L, s in specs]
        dev = [_device(b) for b in host]
        g = rt.graph(dev, autotune=True)
        try:
            info = g.info()
            assert info["kernels"] == 1, info
            # the tuner's pick among the fused launch shapes (128 to 512 threads)
            assert info["candidates"] >= 2 and info["threads_per_cta"] in (128, 256, 320, 384, 512), info
            for _ in range(2):
                g.launch()
                torch.cuda.synchronize()
                assert g.status() == 0
            for b, o in zip(host, g.outs):
                ref = oracle.run_batch(otables, b)
                got = to_numpy(o)
                if precision == abi.FP64:
                    err = compare(b, got, ref, 1e-12)
                    assert max(err.values()) <= 1e-12, err
                else:
                    e = mixed_errors(b, got, ref)
                    assert e["flux_max"] <= 1e-3 and e["heat_dT_Ksol_max"] <= 1e-2, e
        finally:
            g.close()
    finally:
        rt.close()


def test_fused_uneven_multi_grid_and_host_calls(data_dir, otables):
    """The fused form through run_multi (uneven grids in one launch) and the
    host-buffer call, FP64 against the oracle."""
    rt = abi.Radiation(data_dir, max_layers=99, precision=abi.FP64, validate=True, solver=abi.SOLVER_FUSED)
    try:
        bs = [synth.make_batch(70, L=24, seed=96, cloud=True), synth.make_batch(33, L=99, seed=97, cloud=True),
              synth.make_batch(41, L=2, seed=98, cloud=False)]
        outs = rt.run_multi([_device(b) for b in bs])
        for b, o in zip(bs, outs):
            err = compare(b, to_numpy(o), oracle.run_batch(otables, b), 1e-12)
            assert max(err.values()) <= 1e-12, err
        b = synth.make_batch(9000, L=24, seed=99, cloud=True)
        err = compare(b, to_numpy(rt.run(b)), oracle.run_batch(otables, b), 1e-12)
        assert max(err.values()) <= 1e-12, err
    finally:
        rt.close()
