"""Freeze the algorithmic operation counts of the radiation path into
bench/algorithmic_counts.json.

The counts are those of the CPU oracle (oracle/orc_count.cpp: the oracle
compiled with a counting number type), i.e. of the reference's own operation
order, on samples of the seeded benchmark workloads: +, -, *, /, sqrt, exp,
log (LOG10 and ln), pow and erf each count as one floating-point operation,
and the k-table gathers of OPTCV/OPTCI are counted separately.  TLIMIT skips
and night columns make the counts data-dependent, so they are per-column
means over the sample.  bench.py reads the file for the FP64-pipe figures of
its roofline.

    python bench/make_counts.py          # rewrites bench/algorithmic_counts.json
"""
from __future__ import annotations

import json
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]
for p in (ROOT / "legacy-mars-global-climate-model_b200", ROOT / "oracle"):
    sys.path.insert(0, str(p))

import numpy as np  # noqa: E402

import oracle  # noqa: E402
from mgcm_rt import data, synth  # noqa: E402

FLOP_KINDS = ("add", "mul", "div", "sqrt", "exp", "log", "pow", "erf")


def _sub(b: dict, n: int) -> dict:
    """The first n columns of a batch dict."""
    out = {k: (v[:n] if isinstance(v, np.ndarray) and k not in ("sigma", "sol") else v) for k, v in b.items()}
    out["ncol"] = n
    return out


def _per_column(cnt: dict, ncol: int) -> dict:
    r = {k: cnt[k] / ncol for k in oracle.COUNT_KINDS}
    r["flops"] = sum(cnt[k] for k in FLOP_KINDS) / ncol
    return r


def main() -> None:
    ddir, kind = data.ensure_data()
    tables = oracle.Tables(ddir, variant="count")
    aero = oracle.AeroTables(ddir, variant="count")
    out = {
        "definition": "floating-point operations of the reference operation order (the CPU oracle compiled "
                      "with a counting number type, oracle/orc_count.cpp): +, -, *, /, sqrt, exp, log, pow, "
                      "erf one each (exp/log/pow/erf as single operations); 'gather' = k-table reads of "
                      "OPTCV/OPTCI, counted apart; per-column means over the sample",
        "k_tables": kind,
        "workloads": {},
    }
    samples = {
        # the bench's own seeded batches (bench.py: make_batch(..., seed=1000 + rank))
        "c1": (synth.make_batch(64800, L=24, seed=1000, cloud=True), 2048, 24),
        "c4": (synth.make_batch(20000, L=48, seed=1000, cloud=True), 1024, 48),
    }
    for name, (b, n, L) in samples.items():
        s = _sub(b, n)
        cnt = oracle.op_counts(lambda: oracle.run_batch(tables, s, 1))
        day = float(np.mean(np.asarray(s["acosz"]) >= 1.0e-5))
        out["workloads"][name] = {"layers": L, "sample_columns": n, "day_fraction": day,
                                  "per_column": _per_column(cnt, n)}
    # the device-side input stages of the host-buffer calls
    tb = synth.make_tracer_batch(2048, L=24, seed=1000, active_dust=False, cloudon=True)
    cnt = oracle.op_counts(lambda: oracle.aerosols(aero, tb, 1))
    out["aerosols_c1_tracers"] = {"sample_columns": 2048, "per_column": _per_column(cnt, 2048),
                                  "what": "OPT_CLD ice optics + prescribed dust (mgcm_rt_run_tracers)"}
    st = synth.make_state_batch(2048, L=24, seed=1000, active_dust=False, cloudon=True)
    cnt = oracle.op_counts(lambda: oracle.prep(st, variant="count"))
    out["prep_c1_state"] = {"sample_columns": 2048, "per_column": _per_column(cnt, 2048),
                            "what": "FILLPT + QH2O + DUSTPROFILE/FILLTAUCUM (mgcm_rt_run_state)"}
    path = pathlib.Path(__file__).resolve().parent / "algorithmic_counts.json"
    path.write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
