"""Writes the oracle's outputs for small seeded cases to tests/golden/*.npz.

Each file holds every output array of oracle.run_batch for one case plus a
SHA-256 of the case's inputs (so a change of the input recipe shows up as its
own failure).  Run from the repository root after building the oracle:
    python tests/golden/make_golden.py
"""
import hashlib
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "legacy-mars-global-climate-model_b200"))

import oracle  # noqa: E402
from mgcm_rt import data, synth  # noqa: E402

CASES = {
    "c1_l24_cloud": dict(ncol=8, L=24, seed=7, cloud=True),
    "c0_l36_dust": dict(ncol=6, L=36, seed=8, cloud=False),
}


def inputs_digest(b: dict) -> str:
    h = hashlib.sha256()
    for k in sorted(b):
        v = b[k]
        if isinstance(v, np.ndarray):
            h.update(k.encode())
            h.update(np.ascontiguousarray(v, dtype=np.float64).tobytes())
    return h.hexdigest()


def case(name: str):
    p = CASES[name]
    b = synth.make_batch(p["ncol"], L=p["L"], seed=p["seed"], cloud=p["cloud"])
    return b


def main():
    d, kind = data.ensure_data()
    if kind != "real":
        raise SystemExit("golden vectors need the real k tables (oracle/stage_data.py)")
    t = oracle.Tables(d)
    for name in CASES:
        b = case(name)
        out = oracle.run_batch(t, b)
        np.savez_compressed(pathlib.Path(__file__).parent / f"{name}.npz", digest=inputs_digest(b),
                            **{k: np.asarray(v) for k, v in out.items()})
        print(name, "written")


if __name__ == "__main__":
    main()
