"""History-file flux fields of a radiation call (scope: the reference's
`fuptopv ... fdnsurfir`).

COMP3 copies seven per-column fluxes into REAL*4 module arrays after the
radiation (code/comp3.f:703-706,745-747): the visible up/down flux at the top
and at the surface, and the IR up flux at the top, up and down at the
surface.  MHISTV writes them as two unformatted records
(code/mhistv.f:200-201):
    write(11) fuptopv, fdntopv, fupsurfv, fdnsurfv
    write(11) fuptopir, fupsurfir, fdnsurfir
each array REAL*4 (L_J, L_I) in Fortran order.  `history_fields` takes them
from the outputs of any mgcm_rt call (night columns are already zero, as the
reference sets them); `write_flux_records` writes the two records in
gfortran's sequential unformatted layout (4-byte record markers), so a run can
be compared with a history file of the reference.
"""
from __future__ import annotations

import struct

import numpy as np

VIS_FIELDS = ("fuptopv", "fdntopv", "fupsurfv", "fdnsurfv")
IR_FIELDS = ("fuptopir", "fupsurfir", "fdnsurfir")


def _np(a):
    return a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)


def history_fields(out: dict) -> dict:
    """The seven REAL*4 per-column fields from the outputs of one call."""
    up_v, dn_v = _np(out["fluxupv"]), _np(out["fluxdnv"])
    up_i, dn_i = _np(out["fluxupi"]), _np(out["fluxdni"])
    return {
        "fuptopv": up_v[:, 0].astype(np.float32),
        "fdntopv": dn_v[:, 0].astype(np.float32),
        "fupsurfv": up_v[:, -1].astype(np.float32),
        "fdnsurfv": dn_v[:, -1].astype(np.float32),
        "fuptopir": up_i[:, 0].astype(np.float32),
        "fupsurfir": up_i[:, -1].astype(np.float32),
        "fdnsurfir": dn_i[:, -1].astype(np.float32),
    }


def _record(f, payload: bytes) -> None:
    n = struct.pack("<i", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def write_flux_records(f, fields: dict, nj: int, ni: int) -> None:
    """Append the two MHISTV flux records to binary file object `f`.  Columns
    are taken in the order J fastest (column = (J-1) + L_J*(I-1)), which is
    the order of COMP3's loop over J inside I."""
    def arr(name):
        a = np.asarray(fields[name], dtype="<f4")
        if a.size != nj * ni:
            raise ValueError(f"{name}: {a.size} columns, expected {nj}x{ni}")
        return a.reshape(ni, nj).tobytes()      # J fastest = Fortran (L_J, L_I)
    _record(f, b"".join(arr(n) for n in VIS_FIELDS))
    _record(f, b"".join(arr(n) for n in IR_FIELDS))


def read_flux_records(f, nj: int, ni: int) -> dict:
    """Read back the two records written by write_flux_records (or by the
    reference's MHISTV at the same position of its history file)."""
    out = {}
    for names in (VIS_FIELDS, IR_FIELDS):
        n = struct.unpack("<i", f.read(4))[0]
        data = np.frombuffer(f.read(n), dtype="<f4")
        if struct.unpack("<i", f.read(4))[0] != n or data.size != len(names) * nj * ni:
            raise ValueError("not a flux record of this grid")
        for k, name in enumerate(names):
            out[name] = data[k * nj * ni:(k + 1) * nj * ni].copy()
    return out
