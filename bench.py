"""Benchmark of the B200 column radiative transfer (one JSON line on rank 0).

Workload (one step = one radiation call over one batch): 180 x 360 = 64,800
columns x 24 layers, dust + water-ice cloud, seeded synthetic inputs built by
the reference's input recipe (mgcm_rt.synth), real k tables when staged.
Inputs (2.5 GB) are larger than L2 (126 MB), so no flush is needed between steps.

  value  columns/s with inputs resident in HBM (device pointers, C ABI
         mgcm_rt_enqueue), CUDA events on the launching stream, max over ranks
  e2e    the same through mgcm_rt_run with pinned HOST buffers: every step
         copies the batch in and the outputs back inside the timed region
Multi-GPU: columns shard across ranks with no collective on the data path
(weak scaling: each rank runs its own 64,800-column batch).

--impl reference times the reference algorithm on the host cores (the FP64
CPU oracle, a restatement of the reference Fortran, since the reference
cannot be compiled here: no Fortran compiler) on a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
for p in (ROOT / "legacy-mars-global-climate-model_b200", ROOT / "oracle"):
    sys.path.insert(0, str(p))

METRIC = "RT columns/s mixed vs FP64 on 1 B200 at <=1e-3 flux err; p50/p99 request ms"
UNIT = "columns/s"
WORKLOADS = {
    "c1": dict(ncol=64800, L=24, cloud=True,
               name="180x360 = 64,800 columns x 24 layers, dust + water-ice cloud, half night"),
    "c0": dict(ncol=2160, L=24, cloud=False,
               name="36x60 = 2,160 columns x 24 layers, dust only, half night"),
    "c4": dict(ncol=1036800 // 8, L=48, cloud=True,
               name="720x1440 x 48 layers, one eighth (129,600 columns) per call"),
    # profiling case: inputs ~320 MB (> L2) but a small device footprint
    "prof": dict(ncol=8192, L=24, cloud=True,
                 name="8,192 columns x 24 layers, dust + water-ice cloud (ncu case)"),
}


def algorithmic_bytes_per_column(L: int, cloud: bool) -> int:
    """Bytes the C ABI moves per column (FP64): inputs, outputs, DETAU and
    CUMTAUV in and out.  8*(171L+696) with cloud; minus 8*38*(2L+4) without."""
    lev, lev1, nl = 2 * L + 3, 2 * L + 4, L + 1
    n_in = 5 * lev + 2 * lev1 + 36 * lev1 + 4
    if cloud:
        n_in += 2 * lev1 + 36 * lev1
    n_out = 9 * nl + 7
    n_state = 119 * 2 + 119 * 2      # DETAU in/out, CUMTAUV in/out
    return 8 * (n_in + n_out + n_state)


def peaks():
    try:
        j = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = ROOT / "gpurun_out" / f"clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return None
        rows = []
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                "sw_power_cap"), r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


def cpu_baseline(batch, data_dir, budget_s=10.0):
    """Oracle (FP64 restatement of the reference) on all host cores over a
    bounded sample of the workload's columns."""
    import oracle
    t = oracle.Tables(data_dir)
    cores = os.cpu_count() or 1
    def sub(n):
        s = {k: (v[:n] if isinstance(v, np.ndarray) and v.ndim >= 1 and k not in ("sigma", "sol") else v)
             for k, v in batch.items()}
        s["ncol"] = n
        return s
    n0 = min(int(batch["ncol"]), 64 * cores)
    t0 = time.perf_counter()
    oracle.run_batch(t, sub(n0), cores)
    per = (time.perf_counter() - t0) / n0
    n = int(min(batch["ncol"], max(n0, budget_s / max(per, 1e-9))))
    t0 = time.perf_counter()
    oracle.run_batch(t, sub(n), cores)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first {n} columns of the workload, {dt:.1f} s on {cores} threads"}


def run_reference(args, wl):
    from mgcm_rt import data, synth
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    d, kind = data.ensure_data()
    import oracle
    t = oracle.Tables(d)
    cores = os.cpu_count() or 1
    sample = min(wl["ncol"], 16 * cores)
    b = synth.make_batch(sample, L=wl["L"], seed=1000, cloud=wl["cloud"])
    for _ in range(args.warmup):
        oracle.run_batch(t, b, cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.run_batch(t, b, cores)
        times.append(time.perf_counter() - t0)
    v = sample * len(times) / sum(times)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * wl["ncol"] / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, reference input recipe)",
            "config": {"workload": wl["name"], "columns": wl["ncol"], "layers": wl["L"],
                       "k_tables": kind},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{sample} columns per step, {cores} threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, wl)
        return

    import torch
    from mgcm_rt import abi, data, synth

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    d, kind = data.ensure_data()
    prec = abi.MIXED if args.precision == "mixed" else abi.FP64
    rt = abi.Radiation(d, max_layers=wl["L"], precision=prec, device=local, validate=False)
    b = synth.make_batch(wl["ncol"], L=wl["L"], seed=1000 + rank, cloud=wl["cloud"])
    ncol = wl["ncol"]
    stream = torch.cuda.Stream()
    rt.set_stream(stream)

    # ---- device-resident inputs (value)
    bd = {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
          for k, v in b.items()}
    out = abi.alloc_outputs(ncol, wl["L"], device=torch.device("cuda", local))
    for _ in range(args.warmup):
        rt.enqueue(bd, out)
        rt.sync()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    kern_ms = []
    barrier()
    with Clocks(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            rt.enqueue(bd, out)
            rt.sync()
            kern_ms.append(rt.stats()["gpu_ms"])
        e1.record(stream)
        barrier()
    ms = e0.elapsed_time(e1) / args.steps
    st = rt.stats()
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = ncol * world / (ms / 1e3)

    # ---- end to end through the C ABI with pinned host buffers (e2e)
    e2e = None
    if not args.no_e2e:
        hb = {}
        keep = []
        for k, v in b.items():
            if isinstance(v, np.ndarray):
                tpin = torch.empty(v.shape, dtype=torch.float64, pin_memory=True)
                tpin.numpy()[...] = v
                keep.append(tpin)
                hb[k] = tpin.numpy()
            else:
                hb[k] = v
        ho = {k: torch.empty(tuple(v.shape), dtype=torch.float64, pin_memory=True).numpy()
              for k, v in out.items()}
        h2d = sum(v.nbytes for k, v in hb.items() if isinstance(v, np.ndarray))
        d2h = sum(v.nbytes for v in ho.values()) + hb["detau"].nbytes + hb["cumtauv"].nbytes
        for _ in range(args.warmup):
            rt.run(hb, ho, inplace=True)
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            rt.run(hb, ho, inplace=True)
        e1.record(stream)
        barrier()
        ems = e0.elapsed_time(e1) / args.steps
        if dist:
            t = torch.tensor([ems], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": ncol * world / (ems / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": ems}

    if rank == 0:
        bpc = algorithmic_bytes_per_column(wl["L"], wl["cloud"])
        kms = statistics.mean(kern_ms)
        ach = bpc * ncol / (kms / 1e3) / 1e9
        pk, pk_kind = peaks()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == abi.FP64 else "f32+f64",
            "data": "synthetic (seeded, reference input recipe; real k tables)" if kind == "real"
                    else "synthetic (seeded; synthetic k tables)",
            "config": {"workload": wl["name"], "columns_per_gpu": ncol, "layers": wl["L"],
                       "precision": args.precision, "k_tables": kind,
                       "l2": "inputs 2.5 GB per step > 126 MB L2 (no flush needed)",
                       "parallelism": f"column shards x{world}, no collective"},
            "gpu_launches": args.steps * int(st["kernels"]),
            "roofline": {"bound": "hbm", "achieved": ach, "peak": pk, "unit": "GB/s",
                         "frac": ach / pk, "traffic": None,
                         "kernel": "rt_fp64_kernel" if prec == abi.FP64 else "rt_mixed_kernel",
                         "bytes_per_column": bpc, "kernel_ms": kms, "peak_kind": pk_kind},
            "systems_per_step": st["systems"],
            "clocks": clk.summary(),
        }
        if e2e:
            line["e2e"] = e2e
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(b, d)
        print(json.dumps(line), flush=True)
    rt.set_stream(None)
    rt.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
