"""Asynchronous calls on the caller's stream (mgcm_rt_set_stream +
mgcm_rt_enqueue): work the caller queues on that stream after the call sees
the whole call finished -- every concurrent part of it -- without
mgcm_rt_sync; the results match the oracle."""
import numpy as np
import pytest

import oracle
from helpers import compare
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu


def test_enqueue_orders_the_callers_stream(data_dir, otables):
    import torch
    n = 52000   # four concurrent parts
    b = synth.make_batch(n, L=24, seed=311, cloud=True)
    ref = oracle.run_batch(otables, b)
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        dev = {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
               for k, v in b.items()}
        out = abi.alloc_outputs(n, 24, device=torch.device("cuda"))   # zeros until written
        s = torch.cuda.Stream()
        rt.set_stream(s)
        for _ in range(2):
            for v in out.values():
                v.zero_()
            torch.cuda.synchronize()
            rt.enqueue(dev, out)
            with torch.cuda.stream(s):   # the caller's next work on its stream
                snap = {k: v.clone() for k, v in out.items()}
                snap["detau"], snap["cumtauv"] = dev["detau"].clone(), dev["cumtauv"].clone()
            s.synchronize()
            got = {k: v.cpu().numpy() for k, v in snap.items()}
            err = compare(b, got, ref, 1e-12)
            assert max(err.values()) <= 1e-12, err
            rt.sync()
            assert rt.stats()["status"] == 0 and rt.stats()["columns"] == n
    finally:
        rt.close()
