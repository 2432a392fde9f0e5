"""Serving: requests submitted while others run are admitted onto slots as
they free up and overlap on the device; every result equals the same batch
run alone (FP64: to 1e-12; mixed: the same bits, the kernels being the same)."""
import numpy as np
import pytest

from helpers import compare, to_numpy
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu


def _device(b):
    import torch
    return {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
            for k, v in b.items()}


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
def test_results_same_alone_and_in_the_mix(data_dir, precision):
    rt = abi.Radiation(data_dir, max_layers=48, precision=precision, validate=False)
    try:
        specs = [(5000, 24, 51), (40000, 24, 52), (700, 36, 53), (9000, 48, 54), (33000, 24, 55),
                 (1, 24, 56), (12000, 36, 57), (2500, 48, 58)]
        batches = [synth.make_batch(n, L=L, seed=s, cloud=True) for n, L, s in specs]
        alone = [to_numpy(rt.run(b)) for b in batches]
        # the mix: host and device requests submitted back to back
        inflight = []
        for i, b in enumerate(batches):
            bb = _device(b) if i % 2 else dict(b, detau=b["detau"].copy(), cumtauv=b["cumtauv"].copy())
            t, out = rt.submit(bb)
            inflight.append((t, out))
        assert all(rt.poll(t) in (0, 1) for t, _ in inflight)
        for (t, out), b, ref in zip(inflight, batches, alone):
            rt.wait(t, 60.0)
            err = compare(b, to_numpy(out), ref, 1e-12)
            assert max(err.values()) <= 1e-12, err
    finally:
        rt.close()


def test_wait_timeout_and_unknown_ticket(data_dir):
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        with pytest.raises(abi.RTError) as e:
            rt.wait(123456, 0.01)
        assert e.value.code == -10
        b = synth.make_batch(20000, L=24, seed=59, cloud=True)
        t, out = rt.submit(_device(b))
        rt.wait(t, 60.0)
        with pytest.raises(abi.RTError) as e:
            rt.poll(t)          # collected tickets are gone
        assert e.value.code == -10
    finally:
        rt.close()


def test_layer_counts_alternating_across_slots(data_dir):
    """Slots that ran different layer counts before must launch any other
    count: kernel attributes are per function, not per slot."""
    rt = abi.Radiation(data_dir, max_layers=48, precision=abi.MIXED, validate=False)
    try:
        seq = [(20000, 36), (20000, 24), (8000, 36), (20000, 48), (8000, 36), (3000, 24)]
        batches = [synth.make_batch(n, L=L, seed=60 + i, cloud=True) for i, (n, L) in enumerate(seq)]
        first = [to_numpy(rt.run(b)) for b in batches]
        tickets = [rt.submit(_device(b)) for b in batches[::-1]]
        for (t, out), b, ref in zip(tickets, batches[::-1], first[::-1]):
            rt.wait(t, 60.0)
            err = compare(b, to_numpy(out), ref, 1e-12)
            assert max(err.values()) <= 1e-12, err
        again = [to_numpy(rt.run(b)) for b in batches]
        for b, x, y in zip(batches, first, again):
            err = compare(b, x, y, 1e-12)
            assert max(err.values()) <= 1e-12, err
    finally:
        rt.close()
