"""The no-allocation entry point (mgcm_rt_run_noalloc) against the oracle and
against the allocating entry point (mgcm_rt_run) on the same inputs.

mgcm_rt_run_noalloc serves callers that must not allocate device memory
after start-up (a host whose device memory belongs to another allocator, a
time-stepping loop that forbids allocation, a process under a device-memory
quota): its scratch lives in a static device array inside the library.  This
file is named to be collected last; it must pass on its own in a fresh
process and after every other test.  Two calls in a row check that the
shared scratch is reset between calls; the device's free memory is read
before and after each call, which must not change it (the handle's creation
has already placed the array and the kernels on the device)."""
import ctypes as C

import numpy as np
import pytest

import oracle
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


def _free_bytes():
    """cudaMemGetInfo's free bytes on device 0."""
    import torch
    return torch.cuda.mem_get_info(0)[0]


@pytest.mark.parametrize("ncol,L,cloud,seed", [(300, 24, True, 31), (40, 48, True, 32), (6, 99, True, 33)])
def test_noalloc_matches_oracle_twice(data_dir, otables, ncol, L, cloud, seed):
    import torch
    rt = abi.Radiation(data_dir, max_layers=99, precision=abi.FP64, validate=True)
    try:
        b = synth.make_batch(ncol, L=L, seed=seed, cloud=cloud)
        ref = oracle.run_batch(otables, b)
        # the allocating entry point (mgcm_rt_run) on the same inputs
        run_out = to_numpy(rt.run(_device(b)))
        for rep in range(2):
            bd = _device(b)    # fresh DETAU/CUMTAUV: they are in/out
            out = abi.alloc_outputs(ncol, L, device=torch.device("cuda", 0))
            torch.cuda.synchronize()
            free0 = _free_bytes()
            rc = _noalloc(rt, bd, out)
            free1 = _free_bytes()
            assert rc == 0, abi.lib().mgcm_rt_strerror(rc)
            assert free1 == free0, f"call {rep}: device free memory changed by {free0 - free1} bytes"
            out["detau"], out["cumtauv"] = bd["detau"], bd["cumtauv"]
            got = to_numpy(out)
            err = compare(b, got, ref, RTOL)
            assert max(err.values()) <= RTOL, err
            err = compare(b, got, run_out, RTOL)
            assert max(err.values()) <= RTOL, ("against mgcm_rt_run", err)
    finally:
        rt.close()


def test_noalloc_validates_when_asked(data_dir):
    import torch
    b = synth.make_batch(8, L=24, seed=35)
    b["tmid"] = b["tmid"].copy()
    b["tmid"][2, 7] = np.nan
    for validate, want in ((True, -2), (False, 0)):
        rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=validate)
        try:
            out = abi.alloc_outputs(8, 24, device=torch.device("cuda", 0))
            assert _noalloc(rt, _device(b), out) == want
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
