"""History-file flux fields (code/comp3.f:703-706,745-747; records of
code/mhistv.f:200-201): values, REAL*4 rounding, night columns, and the
unformatted record layout round trip."""
import io
import struct

import numpy as np

import oracle
from mgcm_rt import history, synth


def test_history_fields_and_records(otables):
    nj, ni = 6, 4
    b = synth.make_batch(nj * ni, L=24, seed=91, cloud=True)
    out = oracle.run_batch(otables, b)
    f = history.history_fields(out)
    assert all(v.dtype == np.float32 and v.shape == (nj * ni,) for v in f.values())
    np.testing.assert_array_equal(f["fuptopv"], out["fluxupv"][:, 0].astype(np.float32))
    np.testing.assert_array_equal(f["fdnsurfir"], out["fluxdni"][:, -1].astype(np.float32))
    night = b["acosz"] < np.float32(1.0e-5)
    assert night.any()
    for k in history.VIS_FIELDS:
        assert np.all(f[k][night] == 0.0)
    buf = io.BytesIO()
    history.write_flux_records(buf, f, nj, ni)
    raw = buf.getvalue()
    n1 = struct.unpack("<i", raw[:4])[0]
    assert n1 == 4 * 4 * nj * ni and raw[4 + n1:8 + n1] == raw[:4]
    n2 = struct.unpack("<i", raw[8 + n1:12 + n1])[0]
    assert n2 == 3 * 4 * nj * ni and len(raw) == 16 + n1 + n2
    # Fortran order: the first REAL*4 of record 1 is fuptopv(1,1), the next fuptopv(2,1)
    first = np.frombuffer(raw[4:12], dtype="<f4")
    np.testing.assert_array_equal(first, f["fuptopv"][:2])
    back = history.read_flux_records(io.BytesIO(raw), nj, ni)
    for k, v in f.items():
        np.testing.assert_array_equal(back[k], v)
