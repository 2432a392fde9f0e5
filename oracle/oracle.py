"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py (the cpu_baseline leg and
the reference arm) import this module, always as the checker.  The product
library never calls it.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
# variant "libm": column exponentials from the host libm instead of the shared
# deterministic exp (measures the reference algorithm's libm sensitivity)
LIBS = {"rt": LIB, "libm": HERE / "_build" / "liboracle_libm.so",
        "count": HERE / "_build" / "liboracle_count.so"}

NTAB_V = 7 * 51 * 10 * 7 * 17
NTAB_I = 7 * 51 * 10 * 5 * 17
NRAW_V = 7 * 11 * 10 * 7 * 17
NRAW_I = 7 * 11 * 10 * 5 * 17

_D = C.POINTER(C.c_double)


class OrcBatch(C.Structure):
    _fields_ = [("ncol", C.c_int), ("L", C.c_int)] + [
        (n, _D) for n in (
            "plev", "tlev", "pmid", "tmid", "qh2o",
            "tauref", "qextrefdst", "taurefcld", "qextrefcld",
            "qxvdst", "qsvdst", "gvdst", "qxidst", "qsidst", "gidst",
            "qxvcld", "qsvcld", "gvcld", "qxicld", "qsicld", "gicld",
            "acosz", "als", "albi", "pcol", "sol", "sigma")
    ] + [("ptrop", C.c_double)] + [
        (n, _D) for n in (
            "detau", "cumtauv",
            "fmnetv", "fluxupv", "fluxdnv", "fmneti", "fluxupi", "fluxdni",
            "suntot", "irtotal", "qrad",
            "nfluxtopv", "nfluxtopi", "diffvt", "dnvflux", "dndiffv", "dnirflux", "fluxsurf")
    ]


def build() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_libs = {}


def lib(variant: str = "rt"):
    _lib = _libs.get(variant)
    if _lib is None:
        path = LIBS[variant]
        if not path.exists():
            build()
        _lib = C.CDLL(str(path))
        _lib.orc_tables_size.restype = C.c_size_t
        _lib.orc_tables_load.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
        _lib.orc_read_ktables.argtypes = [C.c_char_p, C.c_char_p, _D, _D, _D, _D]
        _lib.orc_build_tables.argtypes = [C.c_void_p, _D, _D, _D, _D]
        _lib.orc_run_batch.argtypes = [C.c_void_p, C.POINTER(OrcBatch), C.c_int]
        _lib.orc_tpindex.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _D,
                                     C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), _D]
        _lib.orc_optics_column.argtypes = [C.c_void_p, C.POINTER(OrcBatch), C.c_int] + [_D] * 10
        _lib.orc_dsolflux.argtypes = [C.c_void_p, C.c_int, _D, _D, _D, _D]
        _lib.orc_bins_batch.argtypes = [C.c_void_p, C.POINTER(OrcBatch)] + [C.POINTER(C.c_int)] * 4 + [_D, _D]
        _libs[variant] = _lib
    return _lib


def _p(a):
    return a.ctypes.data_as(_D) if a is not None else None


class Tables:
    """orc_tables built from the two k-coefficient files of a data directory."""

    OFFSETS = None

    def __init__(self, data_dir, variant: str = "rt"):
        self.variant = variant
        L = lib(variant)
        self.buf = np.zeros(L.orc_tables_size() // 8, dtype=np.float64)
        d = pathlib.Path(data_dir)
        rc = L.orc_tables_load(self.buf.ctypes.data, str(d / "CO2H2O_V_12_95_INTEL").encode(),
                               str(d / "CO2H2O_IR_12_95_INTEL").encode())
        if rc != 0:
            raise RuntimeError(f"oracle table load failed ({rc}) from {d}")

    @property
    def ptr(self):
        return self.buf.ctypes.data

    def view(self):
        """Named views into the table struct (layout of orc_tables)."""
        sizes = [("co2v", NTAB_V), ("co2i", NTAB_I), ("fzerov", 7), ("fzeroi", 5),
                 ("pfgasref", 51), ("tgasref", 7), ("pgasref", 11), ("planckir", 5 * 8501),
                 ("wnov", 7), ("dwnv", 7), ("wavev", 7), ("solarf", 7), ("tauray", 7),
                 ("wnoi", 5), ("dwni", 5), ("wavei", 5), ("qextv", 7), ("qscatv", 7), ("gv", 7),
                 ("qexti", 5), ("qscati", 5), ("gi", 5), ("gweight", 17), ("wrefh2o", 10)]
        out, o = {}, 0
        for n, s in sizes:
            out[n] = self.buf[o:o + s]
            o += s
        return out

    def tpindex(self, pw, tw, qh2o):
        lc = np.zeros(4)
        mt, mp, nh = C.c_int(), C.c_int(), C.c_int()
        wr = np.zeros(1)
        lib(self.variant).orc_tpindex(self.ptr, pw, tw, qh2o, _p(lc), C.byref(mt), C.byref(mp),
                          C.byref(nh), _p(wr))
        return mt.value, mp.value, nh.value, float(wr[0]), lc


def _contig(b, k):
    v = b.get(k)
    return None if v is None else np.ascontiguousarray(v, dtype=np.float64)


def make_struct(b: dict, out: dict) -> tuple[OrcBatch, list]:
    keep = []
    s = OrcBatch()
    s.ncol = int(b["ncol"])
    s.L = int(b["L"])
    for n in ("plev", "tlev", "pmid", "tmid", "qh2o", "tauref", "qextrefdst", "taurefcld",
              "qextrefcld", "qxvdst", "qsvdst", "gvdst", "qxidst", "qsidst", "gidst", "qxvcld",
              "qsvcld", "gvcld", "qxicld", "qsicld", "gicld", "acosz", "als", "albi", "pcol",
              "sol", "sigma"):
        a = _contig(b, n)
        keep.append(a)
        setattr(s, n, _p(a))
    s.ptrop = float(b["ptrop"])
    for n in out:
        setattr(s, n, _p(out[n]))
    return s, keep


def alloc_outputs(ncol: int, L: int, detau=None, cumtauv=None) -> dict:
    nl = L + 1
    out = {n: np.zeros((ncol, nl)) for n in (
        "fmnetv", "fluxupv", "fluxdnv", "fmneti", "fluxupi", "fluxdni", "suntot", "irtotal", "qrad")}
    for n in ("nfluxtopv", "nfluxtopi", "diffvt", "dnvflux", "dndiffv", "dnirflux", "fluxsurf"):
        out[n] = np.zeros(ncol)
    out["detau"] = np.array(detau, dtype=np.float64, copy=True) if detau is not None else np.zeros((ncol, 17, 7))
    out["cumtauv"] = (np.array(cumtauv, dtype=np.float64, copy=True) if cumtauv is not None
                      else np.zeros((ncol, 17, 7)))
    return out


def run_batch(tables: Tables, b: dict, nthreads: int = 0) -> dict:
    out = alloc_outputs(int(b["ncol"]), int(b["L"]), b.get("detau"), b.get("cumtauv"))
    s, keep = make_struct(b, out)
    rc = lib(tables.variant).orc_run_batch(tables.ptr, C.byref(s), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle run failed ({rc})")
    return out


def optics_column(tables: Tables, b: dict, col: int) -> dict:
    L = int(b["L"])
    nl, lev = L + 1, 2 * L + 3
    r = {"dtauv": np.zeros((17, 7, nl)), "wbarv": np.zeros((17, 7, nl)), "cosbv": np.zeros((17, 7, nl)),
         "taucumv": np.zeros((17, 7, lev)), "taugsurfv": np.zeros((16, 7)),
         "dtaui": np.zeros((17, 5, nl)), "wbari": np.zeros((17, 5, nl)), "cosbi": np.zeros((17, 5, nl)),
         "taucumi": np.zeros((17, 5, lev)), "taugsurfi": np.zeros((16, 5))}
    out = alloc_outputs(int(b["ncol"]), L)
    s, keep = make_struct(b, out)
    lib(tables.variant).orc_optics_column(tables.ptr, C.byref(s), col, *[_p(r[k]) for k in (
        "dtauv", "wbarv", "cosbv", "taucumv", "taugsurfv", "dtaui", "wbari", "cosbi", "taucumi",
        "taugsurfi")])
    return r


def bins_batch(tables: Tables, b: dict) -> dict:
    """TPINDEX bins and weights and the Planck index of every level of every
    column (orc_bins_batch): mt, mp, nh2o, nplanck, wratio [ncol][LEV],
    lcoef [ncol][LEV][4]; level 1 has zero bins."""
    n, lev = int(b["ncol"]), 2 * int(b["L"]) + 3
    r = {k: np.zeros((n, lev), dtype=np.int32) for k in ("mt", "mp", "nh2o", "nplanck")}
    r["wratio"] = np.zeros((n, lev))
    r["lcoef"] = np.zeros((n, lev, 4))
    out = alloc_outputs(n, int(b["L"]))
    s, keep = make_struct(b, out)
    ip = C.POINTER(C.c_int)
    lib(tables.variant).orc_bins_batch(tables.ptr, C.byref(s), *[r[k].ctypes.data_as(ip) for k in
                                       ("mt", "mp", "nh2o", "nplanck")], _p(r["wratio"]), _p(r["lcoef"]))
    return r


def dsolflux(tables: Tables, sol, acosz, detau) -> np.ndarray:
    acosz = np.ascontiguousarray(acosz, dtype=np.float64)
    detau = np.ascontiguousarray(detau, dtype=np.float64)
    sol = np.ascontiguousarray(sol, dtype=np.float64)
    out = np.zeros(acosz.shape[0])
    lib(tables.variant).orc_dsolflux(tables.ptr, acosz.shape[0], _p(sol), _p(acosz), _p(detau), _p(out))
    return out


# ---- aerosol optics (code/opt_dst.f, code/opt_cld.f, code/ini_optdst.f)
class OrcTracers(C.Structure):
    _fields_ = [("ncol", C.c_int), ("L", C.c_int), ("active_dust", C.c_int), ("cloudon", C.c_int)] + [
        (n, C.c_void_p) for n in ("plev", "tauref_in", "dust_mass", "dust_number", "ice_mass", "ice_core",
                                  "ice_number", "tauref", "qextrefdst", "qxvdst", "qsvdst", "gvdst", "qxidst",
                                  "qsidst", "gidst", "taurefcld", "qextrefcld", "qxvcld", "qsvcld", "gvcld",
                                  "qxicld", "qsicld", "gicld")]


class AeroTables:
    """Dust and water-ice Mie tables and size bins (orc_aero_load)."""

    def __init__(self, data_dir, variant: str = "rt"):
        L = lib(variant)
        L.orc_aero_load.argtypes = [C.c_void_p, C.c_char_p]
        L.orc_aerosols.argtypes = [C.c_void_p, C.POINTER(OrcTracers)]
        L.orc_aerosols_mt.argtypes = [C.c_void_p, C.POINTER(OrcTracers), C.c_int]
        self.variant = variant
        L.orc_aero_size.restype = C.c_size_t
        self._buf = C.create_string_buffer(int(L.orc_aero_size()) + 64)
        rc = L.orc_aero_load(self._buf, str(data_dir).encode())
        if rc != 0:
            raise FileNotFoundError(f"aerosol tables not readable in {data_dir} ({rc})")
        self.ptr = C.cast(self._buf, C.c_void_p)


def aerosols(aero: AeroTables, tb: dict, nthreads: int = 1) -> dict:
    """Tracer batch -> the standard batch dict (per-level aerosol arrays filled
    as COMP3 fills them), ready for run_batch."""
    ncol, L = int(tb["ncol"]), int(tb["L"])
    lev1 = 2 * L + 4
    out = {k: v for k, v in tb.items()}
    keep = []
    def arr(shape):
        a = np.zeros(shape)
        keep.append(a)
        return a
    names_d = ("tauref", "qextrefdst", "qxvdst", "qsvdst", "gvdst", "qxidst", "qsidst", "gidst")
    names_c = ("taurefcld", "qextrefcld", "qxvcld", "qsvcld", "gvcld", "qxicld", "qsicld", "gicld")
    shapes = ((ncol, lev1), (ncol, lev1), (ncol, 7, lev1), (ncol, 7, lev1), (ncol, 7, lev1),
              (ncol, 5, lev1), (ncol, 5, lev1), (ncol, 5, lev1))
    for n, sh in zip(names_d, shapes):
        out[n] = arr(sh)
    cloud = bool(tb.get("cloudon", 0))
    for n, sh in zip(names_c, shapes):
        out[n] = arr(sh) if cloud else None
    s = OrcTracers()
    s.ncol, s.L = ncol, L
    s.active_dust = 1 if tb.get("active_dust", 0) else 0
    s.cloudon = 1 if cloud else 0
    src = {"plev": "plev", "tauref_in": "tauref", "dust_mass": "dust_mass", "dust_number": "dust_number",
           "ice_mass": "ice_mass", "ice_core": "ice_core_mass", "ice_number": "ice_number"}
    for f, k in src.items():
        v = tb.get(k)
        if v is not None:
            v = np.ascontiguousarray(v, dtype=np.float64)
            keep.append(v)
        setattr(s, f, v.ctypes.data if v is not None else None)
    for n in names_d + names_c:
        setattr(s, n, out[n].ctypes.data if out[n] is not None else None)
    lib(aero.variant).orc_aerosols_mt(aero.ptr, C.byref(s), nthreads)
    for k in ("dust_mass", "dust_number", "ice_mass", "ice_core_mass", "ice_number", "active_dust", "cloudon"):
        out.pop(k, None)
    return out


# ---- column prep (code/potemp1.f, fillpt.f90, comp3.f:576-589, dustprofile.f, filltaucum.f)
NPDST = 100


class OrcPrep(C.Structure):
    _fields_ = [("ncol", C.c_int), ("L", C.c_int), ("active_water", C.c_int), ("prescribed_dust", C.c_int),
                ("ptrop", C.c_double), ("psf", C.c_double), ("rptau", C.c_double), ("mwratio", C.c_double)] + [
        (n, C.c_void_p) for n in ("sigma", "pcol", "tstrat", "gt", "t", "vapour", "tautot", "conr",
                                  "plev", "tlev", "pmid", "tmid", "qh2o", "tauref")]


def _prep_lib(variant: str = "rt"):
    L = lib(variant)
    L.orc_prep.argtypes = [C.POINTER(OrcPrep)]
    L.orc_dust_grid.argtypes = [C.c_double, C.c_double, _D]
    L.orc_dust_profile.argtypes = [_D, C.c_double, C.c_double, C.c_double, _D]
    L.orc_jsrchgt.argtypes = [C.c_int, _D, C.c_double]
    L.orc_jsrchgt.restype = C.c_int
    return L


def dust_grid(psf: float, ptrop: float) -> np.ndarray:
    """PRDST(1..NPDST) (code/dustprofile.f:32-37)."""
    out = np.empty(NPDST)
    _prep_lib().orc_dust_grid(psf, ptrop, _p(out))
    return out


def dust_profile(prdst, rptau: float, conr: float, tautot: float) -> np.ndarray:
    """TAUDST(1..NPDST) of one column (code/dustprofile.f:59-114)."""
    pr = np.ascontiguousarray(prdst, dtype=np.float64)
    out = np.empty(NPDST)
    _prep_lib().orc_dust_profile(_p(pr), rptau, conr, tautot, _p(out))
    return out


def jsrchgt(sx, target: float) -> int:
    """JSRCHGT(N, SX, 1, TARGET) (code/jsrchgt.f90), 1-based."""
    a = np.ascontiguousarray(sx, dtype=np.float64)
    return int(_prep_lib().orc_jsrchgt(len(a), _p(a), target))


def prep(st: dict, variant: str = "rt") -> dict:
    """State batch (synth.make_state_batch) -> the tracer batch COMP3 would
    hand to the aerosol optics: PLEV/TLEV/PMID/TMID/QH2O, and TAUREF for
    prescribed dust, filled as the reference fills them."""
    ncol, L = int(st["ncol"]), int(st["L"])
    lev = 2 * L + 3
    prescribed = not st.get("active_dust", 0)
    water = bool(st.get("active_water", 0))
    keep = []
    def inp(k):
        v = st.get(k)
        if v is None:
            return None
        v = np.ascontiguousarray(v, dtype=np.float64)
        keep.append(v)
        return v.ctypes.data
    out = {n: np.zeros((ncol, lev)) for n in ("plev", "tlev", "pmid", "tmid", "qh2o")}
    out["tauref"] = np.zeros((ncol, lev + 1)) if prescribed else None
    s = OrcPrep()
    s.ncol, s.L = ncol, L
    s.active_water = 1 if water else 0
    s.prescribed_dust = 1 if prescribed else 0
    s.ptrop = float(st["ptrop"])
    s.psf = float(st.get("psf", 0.0))
    s.rptau = float(st.get("rptau", 0.0))
    s.mwratio = float(st.get("mwratio", 0.0))
    for k in ("sigma", "pcol", "tstrat", "gt", "t"):
        setattr(s, k, inp(k))
    s.vapour = inp("vapour") if water else None
    s.tautot = inp("tautot") if prescribed else None
    s.conr = inp("conr") if prescribed else None
    for k, v in out.items():
        setattr(s, k, v.ctypes.data if v is not None else None)
    _prep_lib(variant).orc_prep(C.byref(s))
    tb = {k: st[k] for k in ("ncol", "L", "ptrop", "sigma", "sol", "pcol", "acosz", "als", "albi",
                             "detau", "cumtauv", "dust_mass", "dust_number", "ice_mass", "ice_core_mass",
                             "ice_number", "active_dust", "cloudon")}
    tb.update(out)
    return tb


# ---- operation counts (orc_count.cpp: the oracle with a counting number type)
COUNT_KINDS = ("add", "mul", "div", "sqrt", "exp", "log", "pow", "erf", "gather")


def op_counts(fn) -> dict:
    """Run fn() -- a call into the "count" variant of the oracle on one
    thread -- and return the floating-point operations it performed, by
    kind (COUNT_KINDS)."""
    L = lib("count")
    out = (C.c_ulonglong * len(COUNT_KINDS))()
    L.orc_count_reset()
    fn()
    L.orc_count_read(out)
    return dict(zip(COUNT_KINDS, (int(v) for v in out)))
