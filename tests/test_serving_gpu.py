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


def _served(rt, bd):
    t, out = rt.submit(bd)
    return t, out


def _wait_done(rt, t, limit_s=60.0):
    import time
    t0 = time.monotonic()
    while rt.poll(t) == 0:
        assert time.monotonic() - t0 < limit_s, "request did not finish"
        time.sleep(0.001)


def test_requests_overlap_on_the_device(data_dir):
    """Four one-job requests submitted back to back run on four slots: the
    device intervals bracketing their kernels (CUDA events) intersect, and
    each result equals the batch run alone."""
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        batches = [synth.make_batch(30000, L=24, seed=70 + i, cloud=True) for i in range(4)]
        alone = [to_numpy(rt.run(b)) for b in batches]
        dev = [_device(b) for b in batches]       # on the device before the first submit
        tick = [_served(rt, d) for d in dev]      # back to back
        infos = []
        for t, _ in tick:
            _wait_done(rt, t)
            infos.append(rt.request_info(t))
        for (t, out), b, ref in zip(tick, batches, alone):
            rt.wait(t, 60.0)
            err = compare(b, to_numpy(out), ref, 1e-12)
            assert max(err.values()) <= 1e-12, err
        iv = sorted((i["device_begin_ms"], i["device_end_ms"]) for i in infos)
        assert all(b >= 0.0 and e > b for b, e in iv), infos
        overlaps = sum(1 for a, b in zip(iv, iv[1:]) if b[0] < a[1])
        assert overlaps >= 1, f"no two requests overlapped on the device: {iv}"
    finally:
        rt.close()


def test_hbm_budget_defers_admission_then_completes(data_dir):
    """With an HBM budget that holds one job's staging but not two, the
    second and third requests wait for the first (their admissions are put
    back, counted in `deferred`) and still complete with the right results."""
    n = 12000   # one served job per request
    probe = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        batches = [synth.make_batch(n, L=24, seed=80 + i, cloud=True) for i in range(3)]
        t, _ = _served(probe, _device(batches[0]))
        probe.wait(t, 60.0)
        one_job = probe.stats()["hbm_used"]       # one serving slot's arena for n columns
        alone = [to_numpy(probe.run(b)) for b in batches]
    finally:
        probe.close()
    assert one_job > 0
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False,
                       hbm_budget=int(one_job * 1.5))
    try:
        dev = [_device(b) for b in batches]
        tick = [_served(rt, d) for d in dev]
        infos = []
        for t, _ in tick:
            _wait_done(rt, t)
            infos.append(rt.request_info(t))
        for (t, out), b, ref in zip(tick, batches, alone):
            rt.wait(t, 60.0)
            err = compare(b, to_numpy(out), ref, 1e-12)
            assert max(err.values()) <= 1e-12, err
        assert sum(i["deferred"] for i in infos) >= 1, infos
        # admitted one at a time: the device intervals do not intersect
        iv = sorted((i["device_begin_ms"], i["device_end_ms"]) for i in infos)
        assert all(b[0] >= a[1] for a, b in zip(iv, iv[1:])), iv
        assert rt.stats()["hbm_used"] <= int(one_job * 1.5)
    finally:
        rt.close()


JOB = 16384   # columns per served job (the library's SERVE_JOB_COLS)


def test_queue_full_is_ebusy(data_dir):
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False, max_queued_jobs=2)
    try:
        big = synth.make_batch(3 * JOB, L=24, seed=90, cloud=True)   # 3 jobs: never fits
        with pytest.raises(abi.RTError) as e:
            rt.submit(_device(big))
        assert e.value.code == -9
        two = _device(synth.make_batch(2 * JOB, L=24, seed=91, cloud=True))   # 2 jobs: fills the queue
        one = _device(synth.make_batch(100, L=24, seed=92, cloud=True))
        t, out = rt.submit(two)
        with pytest.raises(abi.RTError) as e:
            rt.submit(one)                                             # while both jobs are unfinished
        assert e.value.code == -9
        rt.wait(t, 60.0)
        t2, _ = rt.submit(one)                                         # room again
        rt.wait(t2, 60.0)
    finally:
        rt.close()


def test_forced_allocation_failure_is_enomem(data_dir):
    """A one-byte HBM budget: every call that needs staging fails with
    MGCM_RT_ENOMEM, on the synchronous and the served path, and the library
    stays usable for a handle with a normal budget."""
    b = synth.make_batch(500, L=24, seed=93, cloud=True)
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False, hbm_budget=1)
    try:
        for _ in range(2):
            with pytest.raises(abi.RTError) as e:
                rt.run(b)
            assert e.value.code == -5
        t, _ = rt.submit(_device(b))
        with pytest.raises(abi.RTError) as e:
            rt.wait(t, 60.0)
        assert e.value.code == -5
    finally:
        rt.close()
    ok = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        ok.run(b)
    finally:
        ok.close()
