"""Multi-rank path on CPU: two gloo ranks shard the columns, each runs its
shard (oracle as the compute), timings reduce to the max over ranks, and the
gathered outputs equal the single-process result bit for bit."""
import os
import socket

import numpy as np
import pytest

from mgcm_rt import shard


def test_column_shard_partitions():
    for n in (0, 1, 7, 64800, 889920):
        for w in (1, 2, 3, 4, 8):
            r = [shard.column_shard(n, k, w) for k in range(w)]
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            assert max(c1 - c0 for c0, c1 in r) - min(c1 - c0 for c0, c1 in r) <= 1
    with pytest.raises(ValueError):
        shard.column_shard(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, data_dir, q):
    import datetime
    import sys
    import pathlib
    root = pathlib.Path(__file__).resolve().parents[1]
    for p in (root / "legacy-mars-global-climate-model_b200", root / "oracle"):
        sys.path.insert(0, str(p))
    import torch.distributed as dist
    import oracle
    from mgcm_rt import shard as sh, synth
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = 10
        b = synth.make_batch(n, L=24, seed=77, cloud=True)
        c0, c1 = sh.column_shard(n, rank, world)
        mine = {k: (v[c0:c1] if isinstance(v, np.ndarray) and k not in ("sigma", "sol") else v) for k, v in b.items()}
        mine["ncol"] = c1 - c0
        out = oracle.run_batch(oracle.Tables(data_dir), mine, 1)
        t = sh.max_over_ranks(1.0 + rank, dist)
        full = {k: sh.gather_columns(v, dist, n) for k, v in out.items()}
        q.put((rank, t, {k: v for k, v in full.items()} if rank == 0 else None))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather(data_dir, otables):
    import multiprocessing as mp
    import oracle
    from mgcm_rt import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(data_dir), q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    times = {r: t for r, t, _ in res}
    assert times == {0: 2.0, 1: 2.0}          # max over ranks on both
    full = next(f for r, _, f in res if r == 0)
    ref = oracle.run_batch(otables, synth.make_batch(10, L=24, seed=77, cloud=True), 1)
    for k, v in ref.items():
        np.testing.assert_array_equal(full[k], v, err_msg=k)
