"""The no-allocation entry point (mgcm_rt_run_noalloc) against mgcm_rt_run.

mgcm_rt_run_noalloc serves callers that must not allocate device memory
after start-up (a host whose device memory belongs to another allocator, a
time-stepping loop that forbids allocation, a process under a device-memory
quota): its scratch lives in a static device array inside the library.  This
file is named to be collected last; it must pass on its own in a fresh
process and after every other test.  Two calls in a row check that the
shared scratch is reset between calls."""
import ctypes as C

import numpy as np
import pytest

from helpers import compare, to_numpy
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _noalloc(rt, b, out):
    L = abi.lib()
    L.mgcm_rt_run_noalloc.argtypes = [C.c_void_p, C.POINTER(abi.BatchIn), C.POINTER(abi.BatchOut)]
    keep = []
    bi = abi.make_in(b, True, keep)
    bo = abi.make_out(out)
    return L.mgcm_rt_run_noalloc(rt._h, C.byref(bi), C.byref(bo))


def _device(b):
    import torch
    return {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
            for k, v in b.items()}


@pytest.mark.parametrize("ncol,L,cloud,seed", [(300, 24, True, 31), (40, 48, True, 32), (6, 99, True, 33)])
def test_noalloc_matches_run_twice(data_dir, ncol, L, cloud, seed):
    import torch
    rt = abi.Radiation(data_dir, max_layers=99, precision=abi.FP64, validate=False)
    try:
        b = synth.make_batch(ncol, L=L, seed=seed, cloud=cloud)
        ref = to_numpy(rt.run(_device(b)))
        for _ in range(2):
            bd = _device(b)    # fresh DETAU/CUMTAUV: they are in/out
            out = abi.alloc_outputs(ncol, L, device=torch.device("cuda", 0))
            rc = _noalloc(rt, bd, out)
            assert rc == 0, abi.lib().mgcm_rt_strerror(rc)
            out["detau"], out["cumtauv"] = bd["detau"], bd["cumtauv"]
            err = compare(b, to_numpy(out), ref, RTOL)
            assert max(err.values()) <= RTOL, err
    finally:
        rt.close()


def test_noalloc_rejects_host_buffers(data_dir):
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64)
    try:
        b = synth.make_batch(4, L=24, seed=34)
        L = abi.lib()
        L.mgcm_rt_run_noalloc.argtypes = [C.c_void_p, C.POINTER(abi.BatchIn), C.POINTER(abi.BatchOut)]
        keep = []
        bi = abi.make_in(b, False, keep)
        out = abi.alloc_outputs(4, 24)
        assert L.mgcm_rt_run_noalloc(rt._h, C.byref(bi), C.byref(abi.make_out(out))) == -1
    finally:
        rt.close()
