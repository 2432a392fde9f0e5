"""Locations and formats of the radiation data files.

The library reads the same two k-coefficient files the reference reads at
set-up (code/laginterp.f90:59-69): ``CO2H2O_V_12_95_INTEL`` and
``CO2H2O_IR_12_95_INTEL``, each a Fortran unformatted sequential file with
4-byte record markers holding one record of k values, shape
(7 T, 11 P, 10 H2O, NB bands, 17 Gauss) in Fortran order, then one record of
FZERO(NB).  The input generator additionally reads the water-ice Mie tables
``waterCoated_{vis,ir}_JD_12bands.dat`` (code/initcld.f:161-172).

``default_data_dir()`` is ``<repo>/data`` (override with ``MGCM_RT_DATA``).
When the real files are absent, ``ensure_data()`` writes a seeded synthetic
k-table of identical shape and format (log10 k ~ U[-38,-28], Gauss point 17
identically zero, FZEROV = [0,..,0,0.94], FZEROI = 0) into
``<repo>/data/synthetic`` and returns that directory, so every consumer goes
through the same file reader.
"""
from __future__ import annotations

import os
import pathlib
import struct

import numpy as np

KV_FILE = "CO2H2O_V_12_95_INTEL"
KI_FILE = "CO2H2O_IR_12_95_INTEL"
ICE_VIS_FILE = "waterCoated_vis_JD_12bands.dat"
ICE_IR_FILE = "waterCoated_ir_JD_12bands.dat"
REQUIRED = (KV_FILE, KI_FILE)
OPTIONAL = (ICE_VIS_FILE, ICE_IR_FILE)

NT, NP11, NH, NG = 7, 11, 10, 17

_REPO = pathlib.Path(__file__).resolve().parents[2]


def default_data_dir() -> pathlib.Path:
    env = os.environ.get("MGCM_RT_DATA")
    return pathlib.Path(env) if env else _REPO / "data"


def have_real_tables(d: os.PathLike | None = None) -> bool:
    d = pathlib.Path(d) if d else default_data_dir()
    return all((d / f).is_file() for f in REQUIRED)


def _write_record(f, arr: np.ndarray) -> None:
    b = np.ascontiguousarray(arr, dtype="<f8").tobytes()
    f.write(struct.pack("<i", len(b)))
    f.write(b)
    f.write(struct.pack("<i", len(b)))


def read_fortran_records(path: os.PathLike) -> list[np.ndarray]:
    """Read every record of a little-endian, 4-byte-marker sequential file."""
    raw = pathlib.Path(path).read_bytes()
    out, pos = [], 0
    while pos < len(raw):
        (n,) = struct.unpack_from("<i", raw, pos)
        pos += 4
        out.append(np.frombuffer(raw, dtype="<f8", count=n // 8, offset=pos).copy())
        pos += n
        (m,) = struct.unpack_from("<i", raw, pos)
        if m != n:
            raise ValueError(f"{path}: record marker mismatch")
        pos += 4
    return out


def write_synthetic_ktables(d: os.PathLike, seed: int = 20240) -> pathlib.Path:
    """Seeded stand-in for the k tables, same shape and record layout."""
    d = pathlib.Path(d)
    d.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    for name, nb, fz in ((KV_FILE, 7, [0, 0, 0, 0, 0, 0, 0.94]), (KI_FILE, 5, [0] * 5)):
        # Fortran order (nt, np, nh, nw, ng) -> numpy C order reversed
        logk = rng.uniform(-38.0, -28.0, size=(NG, nb, NH, NP11, NT))
        k = 10.0 ** logk
        k[NG - 1] = 0.0
        with open(d / name, "wb") as f:
            _write_record(f, k.ravel())
            _write_record(f, np.asarray(fz, dtype=np.float64))
    (d / "SYNTHETIC").write_text(f"seeded synthetic k tables, seed={seed}\n")
    return d


def ensure_data(d: os.PathLike | None = None) -> tuple[pathlib.Path, str]:
    """Return (directory, kind) with kind 'real' or 'synthetic'."""
    d = pathlib.Path(d) if d else default_data_dir()
    if have_real_tables(d):
        return d, "real"
    syn = d / "synthetic"
    if not have_real_tables(syn):
        write_synthetic_ktables(syn)
    return syn, "synthetic"


def read_ice_tables(d: os.PathLike | None = None):
    """Water-ice coated-sphere Mie tables, read as code/initcld.f:161-172 does.

    Returns dict with qextv/qscatv/gv of shape (15 ratios, 20 bins, 7) and
    qexti/qscati/gi of shape (15, 20, 5), or None when the files are absent.
    """
    d = pathlib.Path(d) if d else default_data_dir()
    fv, fi = d / ICE_VIS_FILE, d / ICE_IR_FILE
    if not (fv.is_file() and fi.is_file()):
        return None
    v = np.array(fv.read_text().split(), dtype=np.float64).reshape(15, 20, 3, 7)
    i = np.array(fi.read_text().split(), dtype=np.float64).reshape(15, 20, 3, 5)
    return {
        "qextv": v[:, :, 0], "qscatv": v[:, :, 1], "gv": v[:, :, 2],
        "qexti": i[:, :, 0], "qscati": i[:, :, 1], "gi": i[:, :, 2],
    }
