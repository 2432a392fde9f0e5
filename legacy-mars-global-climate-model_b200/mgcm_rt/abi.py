"""ctypes binding of the C ABI (include/mgcm_rt.h) -- the reference-facing call.

The reference runs, per column, ``OPTCV -> SFLUXV -> OPTCI -> SFLUXI`` and the
heating block of ``COMP3`` (code/comp3.f:637-771).  ``Radiation.run`` takes a
whole batch of columns in the library layout (see ``mgcm_rt.synth``) and
returns the same outputs.  Arrays may be numpy (host) or CUDA torch tensors
(device); the pointer kind is passed to the library, which copies host arrays
itself.  There is no CPU fallback: a missing library raises at import.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

from . import INPUT_COL, INPUT_LEV, OUTPUT_COL, OUTPUT_LAY

LIB_PATH = (pathlib.Path(os.environ["MGCM_RT_LIBRARY"]) if os.environ.get("MGCM_RT_LIBRARY")
            else pathlib.Path(__file__).resolve().parent / "libmgcmrt.so")

FP64, MIXED = 0, 1
STATUS = {0: "OK", -1: "EINVAL", -2: "ENONFINITE", -3: "ETEMP", -4: "ELAYERS", -5: "ENOMEM",
          -6: "EIO", -7: "ECUDA", -8: "ETIMEOUT", -9: "EBUSY", -10: "ENOTFOUND"}

_D = C.POINTER(C.c_double)


class Config(C.Structure):
    _fields_ = [("max_layers", C.c_int), ("precision", C.c_int), ("device", C.c_int),
                ("validate", C.c_int), ("hbm_budget", C.c_size_t), ("solver", C.c_int),
                ("max_queued_jobs", C.c_int)]


class RequestInfo(C.Structure):
    _fields_ = [("done", C.c_int), ("status", C.c_int), ("jobs", C.c_int), ("deferred", C.c_int),
                ("submit_ms", C.c_double), ("done_ms", C.c_double), ("device_begin_ms", C.c_double),
                ("device_end_ms", C.c_double)]


SOLVER_AUTO, SOLVER_THREAD, SOLVER_QUAD, SOLVER_ONCHIP, SOLVER_TMEM, SOLVER_FUSED = 0, 1, 2, 3, 4, 5


_IN_PTRS = ("sigma", "sol", "plev", "tlev", "pmid", "tmid", "qh2o", "tauref", "qextrefdst",
            "qxvdst", "qsvdst", "gvdst", "qxidst", "qsidst", "gidst", "taurefcld", "qextrefcld",
            "qxvcld", "qsvcld", "gvcld", "qxicld", "qsicld", "gicld", "acosz", "als", "albi",
            "pcol", "detau", "cumtauv")
_OUT_PTRS = ("fmnetv", "fluxupv", "fluxdnv", "fmneti", "fluxupi", "fluxdni", "suntot",
             "irtotal", "qrad", "nfluxtopv", "nfluxtopi", "diffvt", "dnvflux", "dndiffv",
             "dnirflux", "fluxsurf")


class BatchIn(C.Structure):
    _fields_ = [("ncol", C.c_int), ("nlayers", C.c_int), ("device_ptrs", C.c_int),
                ("ptrop", C.c_double)] + [(n, C.c_void_p) for n in _IN_PTRS]


class BatchOut(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in _OUT_PTRS]


class Stats(C.Structure):
    _fields_ = [("gpu_ms", C.c_double), ("total_ms", C.c_double), ("columns", C.c_longlong),
                ("systems", C.c_longlong), ("kernels", C.c_int), ("status", C.c_int),
                ("hbm_used", C.c_longlong), ("hbm_budget", C.c_longlong)]


class RTError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where}: {STATUS.get(code, code)} ({lib().mgcm_rt_strerror(code).decode()})")


_TR_PTRS = ("sigma", "sol", "plev", "tlev", "pmid", "tmid", "qh2o", "tauref", "dust_mass", "dust_number",
            "ice_mass", "ice_core_mass", "ice_number", "acosz", "als", "albi", "pcol", "detau", "cumtauv")


class BatchTracers(C.Structure):
    _fields_ = [("ncol", C.c_int), ("nlayers", C.c_int), ("device_ptrs", C.c_int), ("active_dust", C.c_int),
                ("cloudon", C.c_int), ("ptrop", C.c_double)] + [(n, C.c_void_p) for n in _TR_PTRS]


_ST_PTRS = ("sigma", "sol", "pcol", "t", "tstrat", "gt", "vapour", "tautot", "conr", "dust_mass",
            "dust_number", "ice_mass", "ice_core_mass", "ice_number", "acosz", "als", "albi", "detau",
            "cumtauv", "plev", "tlev", "pmid", "tmid", "qh2o", "tauref")
# prepared level arrays a state call can return (the last six of _ST_PTRS)
PREP_FIELDS = ("plev", "tlev", "pmid", "tmid", "qh2o", "tauref")


class BatchState(C.Structure):
    _fields_ = [("ncol", C.c_int), ("nlayers", C.c_int), ("device_ptrs", C.c_int), ("active_dust", C.c_int),
                ("cloudon", C.c_int), ("active_water", C.c_int), ("ptrop", C.c_double), ("psf", C.c_double),
                ("rptau", C.c_double), ("mwratio", C.c_double)] + [(n, C.c_void_p) for n in _ST_PTRS]


class Tune(C.Structure):
    _fields_ = [("chunk_cols", C.c_int), ("solve_ctas_per_sm", C.c_int), ("reduce_rows", C.c_int),
                ("candidates", C.c_int), ("tuning_cols", C.c_int), ("default_ms", C.c_double),
                ("best_ms", C.c_double), ("kernels", C.c_int), ("columns", C.c_int),
                ("threads_per_cta", C.c_int)]


_lib = None


def lib():
    """Load libmgcmrt.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} not built; run __graft_entry__.build()")
        L = C.CDLL(str(LIB_PATH))
        L.mgcm_rt_create.restype = C.c_void_p
        L.mgcm_rt_create.argtypes = [C.POINTER(Config), C.c_char_p, C.POINTER(C.c_int)]
        L.mgcm_rt_run.argtypes = [C.c_void_p, C.POINTER(BatchIn), C.POINTER(BatchOut)]
        L.mgcm_rt_run_multi.argtypes = [C.c_void_p, C.c_int, C.POINTER(BatchIn), C.POINTER(BatchOut)]
        L.mgcm_rt_submit.argtypes = [C.c_void_p, C.POINTER(BatchIn), C.POINTER(BatchOut),
                                     C.POINTER(C.c_longlong)]
        L.mgcm_rt_poll.argtypes = [C.c_void_p, C.c_longlong]
        L.mgcm_rt_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_double]
        L.mgcm_rt_get_request_info.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(RequestInfo)]
        L.mgcm_rt_dsolflux.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 5
        L.mgcm_rt_debug_bins.argtypes = [C.c_void_p, C.POINTER(BatchIn)] + [C.c_void_p] * 6
        L.mgcm_rt_enqueue.argtypes = [C.c_void_p, C.POINTER(BatchIn), C.POINTER(BatchOut)]
        L.mgcm_rt_sync.argtypes = [C.c_void_p]
        L.mgcm_rt_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        L.mgcm_rt_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.mgcm_rt_tables_host.argtypes = [C.c_char_p, _D, _D, _D, _D]
        L.mgcm_rt_destroy.argtypes = [C.c_void_p]
        L.mgcm_rt_strerror.restype = C.c_char_p
        L.mgcm_rt_strerror.argtypes = [C.c_int]
        L.mgcm_rt_version.restype = C.c_char_p
        L.mgcm_rt_run_tracers.argtypes = [C.c_void_p, C.POINTER(BatchTracers), C.POINTER(BatchOut)]
        L.mgcm_rt_run_state.argtypes = [C.c_void_p, C.POINTER(BatchState), C.POINTER(BatchOut)]
        L.mgcm_rt_graph_create.argtypes = [C.c_void_p, C.c_int, C.POINTER(BatchIn), C.POINTER(BatchOut),
                                           C.c_int, C.POINTER(C.c_void_p)]
        L.mgcm_rt_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
        L.mgcm_rt_graph_status.argtypes = [C.c_void_p]
        L.mgcm_rt_graph_info.argtypes = [C.c_void_p, C.POINTER(Tune)]
        L.mgcm_rt_graph_destroy.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a):
    if a is None:
        return None
    if _is_torch(a):
        return a.data_ptr()
    return a.ctypes.data


def _host(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def alloc_outputs(ncol: int, L: int, like=None, device=None):
    """Output dict in the library layout (numpy, or torch on `device`)."""
    nl = L + 1
    if device is not None:
        import torch
        z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=device)  # noqa: E731
    else:
        z = lambda *s: np.zeros(s)  # noqa: E731
    out = {n: z(ncol, nl) for n in OUTPUT_LAY}
    out.update({n: z(ncol) for n in OUTPUT_COL})
    return out


def make_in(b: dict, device_ptrs: bool, keep: list) -> BatchIn:
    s = BatchIn()
    s.ncol = int(b["ncol"])
    s.nlayers = int(b["L"])
    s.device_ptrs = 1 if device_ptrs else 0
    s.ptrop = float(b["ptrop"])
    for n in _IN_PTRS:
        a = b.get(n)
        if a is not None and not device_ptrs:
            a = _host(a)
        if a is not None:
            keep.append(a)
        setattr(s, n, _ptr(a))
    return s


def make_out(o: dict) -> BatchOut:
    s = BatchOut()
    for n in _OUT_PTRS:
        setattr(s, n, _ptr(o[n]))
    return s


class Radiation:
    """A handle on one GPU: tables resident in HBM, runs batches of columns."""

    def __init__(self, data_dir, max_layers: int = 48, precision: int = FP64, device: int = 0,
                 validate: bool = True, hbm_budget: int = 0, solver: int = 0, max_queued_jobs: int = 0):
        cfg = Config(max_layers, precision, device, 1 if validate else 0, hbm_budget, solver, max_queued_jobs)
        st = C.c_int(0)
        self._h = lib().mgcm_rt_create(C.byref(cfg), str(data_dir).encode(), C.byref(st))
        if not self._h:
            raise RTError(st.value, "mgcm_rt_create")
        self.precision = precision
        self.device = device
        self._inflight: dict = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().mgcm_rt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, b: dict, out: dict | None = None, inplace: bool = False) -> dict:
        """Radiation for every column of batch ``b``.

        Host (numpy) inputs give numpy outputs; CUDA tensors give CUDA
        outputs.  DETAU and CUMTAUV are updated in place in ``b`` for device
        inputs (and for host inputs with ``inplace``); otherwise host inputs
        are left untouched and the updated copies are returned."""
        dev = _is_torch(b["plev"]) and b["plev"].is_cuda
        keep: list = []
        if dev:
            bi = make_in(b, True, keep)
            if out is None:
                out = alloc_outputs(int(b["ncol"]), int(b["L"]), device=b["plev"].device)
        else:
            if not inplace:
                b = dict(b)
                b["detau"] = np.array(b["detau"], dtype=np.float64, copy=True)
                b["cumtauv"] = np.array(b["cumtauv"], dtype=np.float64, copy=True)
            bi = make_in(b, False, keep)
            if out is None:
                out = alloc_outputs(int(b["ncol"]), int(b["L"]))
        bo = make_out(out)
        rc = lib().mgcm_rt_run(self._h, C.byref(bi), C.byref(bo))
        if rc != 0:
            raise RTError(rc, "mgcm_rt_run")
        out["detau"] = b["detau"]
        out["cumtauv"] = b["cumtauv"]
        return out

    def enqueue(self, b: dict, out: dict) -> None:
        """Device-resident batch: enqueue on the handle's stream, no wait."""
        keep: list = []
        bi = make_in(b, True, keep)
        bo = make_out(out)
        self._keep = (keep, bi, bo)
        rc = lib().mgcm_rt_enqueue(self._h, C.byref(bi), C.byref(bo))
        if rc != 0:
            raise RTError(rc, "mgcm_rt_enqueue")

    def sync(self) -> None:
        rc = lib().mgcm_rt_sync(self._h)
        if rc != 0:
            raise RTError(rc, "mgcm_rt_sync")

    def set_stream(self, stream) -> None:
        """Use a caller stream (a torch.cuda.Stream or raw handle; None resets)."""
        ptr = None if stream is None else int(getattr(stream, "cuda_stream", stream))
        rc = lib().mgcm_rt_set_stream(self._h, ptr)
        if rc != 0:
            raise RTError(rc, "mgcm_rt_set_stream")

    def run_multi(self, batches: list, outs: list | None = None) -> list:
        dev = _is_torch(batches[0]["plev"]) and batches[0]["plev"].is_cuda
        keep: list = []
        ins = (BatchIn * len(batches))()
        outs_c = (BatchOut * len(batches))()
        if outs is None:
            outs = [alloc_outputs(int(b["ncol"]), int(b["L"]),
                                  device=b["plev"].device if dev else None) for b in batches]
        bs = []
        for i, b in enumerate(batches):
            if not dev:
                b = dict(b)
                b["detau"] = np.array(b["detau"], dtype=np.float64, copy=True)
                b["cumtauv"] = np.array(b["cumtauv"], dtype=np.float64, copy=True)
            bs.append(b)
            ins[i] = make_in(b, dev, keep)
            outs_c[i] = make_out(outs[i])
        rc = lib().mgcm_rt_run_multi(self._h, len(batches), ins, outs_c)
        if rc != 0:
            raise RTError(rc, "mgcm_rt_run_multi")
        for b, o in zip(bs, outs):
            o["detau"] = b["detau"]
            o["cumtauv"] = b["cumtauv"]
        return outs

    # ---- tracer inputs (aerosol optics on the device) -----------------
    def run_tracers(self, t: dict, out: dict | None = None, inplace: bool = False) -> dict:
        """Radiation from tracer mixing ratios (synth.make_tracer_batch layout):
        the device fills the per-level dust/ice optical properties, then runs
        the radiation.  Host or CUDA inputs as in run()."""
        dev = _is_torch(t["plev"]) and t["plev"].is_cuda
        if not dev and not inplace:
            t = dict(t)
            t["detau"] = np.array(t["detau"], dtype=np.float64, copy=True)
            t["cumtauv"] = np.array(t["cumtauv"], dtype=np.float64, copy=True)
        keep: list = []
        s = BatchTracers()
        s.ncol, s.nlayers = int(t["ncol"]), int(t["L"])
        s.device_ptrs = 1 if dev else 0
        s.active_dust = 1 if t.get("active_dust", 0) else 0
        s.cloudon = 1 if t.get("cloudon", 0) else 0
        s.ptrop = float(t["ptrop"])
        for n in _TR_PTRS:
            a = t.get(n)
            if a is not None and not dev:
                a = _host(a)
            if a is not None:
                keep.append(a)
            setattr(s, n, _ptr(a))
        if out is None:
            out = alloc_outputs(s.ncol, s.nlayers, device=t["plev"].device if dev else None)
        bo = make_out(out)
        rc = lib().mgcm_rt_run_tracers(self._h, C.byref(s), C.byref(bo))
        if rc != 0:
            raise RTError(rc, "mgcm_rt_run_tracers")
        out["detau"], out["cumtauv"] = t["detau"], t["cumtauv"]
        return out

    def run_state(self, st: dict, out: dict | None = None, inplace: bool = False,
                  return_levels: bool = False) -> dict:
        """Radiation from the GCM state of each column (synth.make_state_batch
        layout): the device builds PLEV/TLEV/PMID/TMID/QH2O (and TAUREF for
        prescribed dust), then the aerosol optics, then the radiation.  With
        ``return_levels`` the prepared arrays come back in ``out`` under
        PREP_FIELDS.  Host or CUDA inputs as in run()."""
        dev = _is_torch(st["t"]) and st["t"].is_cuda
        if not dev and not inplace:
            st = dict(st)
            st["detau"] = np.array(st["detau"], dtype=np.float64, copy=True)
            st["cumtauv"] = np.array(st["cumtauv"], dtype=np.float64, copy=True)
        ncol, L = int(st["ncol"]), int(st["L"])
        if out is None:
            out = alloc_outputs(ncol, L, device=st["t"].device if dev else None)
        prescribed = not st.get("active_dust", 0)
        if return_levels:
            lev = 2 * L + 3
            for n in PREP_FIELDS:
                if n == "tauref" and not prescribed:
                    continue
                shape = (ncol, lev + 1 if n == "tauref" else lev)
                if dev:
                    import torch
                    out[n] = torch.empty(shape, dtype=torch.float64, device=st["t"].device)
                else:
                    out[n] = np.empty(shape)
        keep: list = []
        s = BatchState()
        s.ncol, s.nlayers = ncol, L
        s.device_ptrs = 1 if dev else 0
        s.active_dust = 0 if prescribed else 1
        s.cloudon = 1 if st.get("cloudon", 0) else 0
        s.active_water = 1 if st.get("active_water", 0) else 0
        s.ptrop = float(st["ptrop"])
        s.psf = float(st.get("psf", 0.0))
        s.rptau = float(st.get("rptau", 0.0))
        s.mwratio = float(st.get("mwratio", 0.0))
        for n in _ST_PTRS:
            a = out.get(n) if n in PREP_FIELDS else st.get(n)
            if a is not None and not dev and n not in PREP_FIELDS:
                a = _host(a)
            if a is not None:
                keep.append(a)
            setattr(s, n, _ptr(a))
        bo = make_out(out)
        rc = lib().mgcm_rt_run_state(self._h, C.byref(s), C.byref(bo))
        if rc != 0:
            raise RTError(rc, "mgcm_rt_run_state")
        out["detau"], out["cumtauv"] = st["detau"], st["cumtauv"]
        return out

    # ---- captured uneven batches --------------------------------------
    def graph(self, batches: list, outs: list | None = None, autotune: bool = True) -> "Graph":
        """Capture device-resident batches (one per grid or ensemble member, up
        to 64) as one CUDA graph; see Graph."""
        for b in batches:
            if not (_is_torch(b["plev"]) and b["plev"].is_cuda):
                raise ValueError("graph batches must be CUDA tensors")
        keep: list = []
        ins = (BatchIn * len(batches))()
        if outs is None:
            outs = [alloc_outputs(int(b["ncol"]), int(b["L"]), device=b["plev"].device) for b in batches]
        outs_c = (BatchOut * len(batches))()
        for i, b in enumerate(batches):
            ins[i] = make_in(b, True, keep)
            outs_c[i] = make_out(outs[i])
        g = C.c_void_p()
        rc = lib().mgcm_rt_graph_create(self._h, len(batches), ins, outs_c, 1 if autotune else 0, C.byref(g))
        if rc != 0:
            raise RTError(rc, "mgcm_rt_graph_create")
        for b, o in zip(batches, outs):
            o["detau"], o["cumtauv"] = b["detau"], b["cumtauv"]
        return Graph(self, g, outs, (keep, ins, outs_c, batches))

    # ---- serving -------------------------------------------------------
    def submit(self, b: dict, out: dict | None = None) -> tuple[int, dict]:
        """Queue batch ``b``; returns (ticket, out).  Arrays must stay alive and
        unmodified until ``wait`` returns; host DETAU/CUMTAUV are updated in
        place."""
        dev = _is_torch(b["plev"]) and b["plev"].is_cuda
        keep: list = []
        bi = make_in(b, dev, keep)
        if out is None:
            out = alloc_outputs(int(b["ncol"]), int(b["L"]),
                                device=b["plev"].device if dev else None)
        bo = make_out(out)
        t = C.c_longlong(0)
        rc = lib().mgcm_rt_submit(self._h, C.byref(bi), C.byref(bo), C.byref(t))
        if rc != 0:
            raise RTError(rc, "mgcm_rt_submit")
        self._inflight[t.value] = (keep, bi, bo, b, out)
        out["detau"], out["cumtauv"] = b["detau"], b["cumtauv"]
        return t.value, out

    def poll(self, ticket: int) -> int:
        """1 finished, 0 pending; raises on an error status."""
        rc = lib().mgcm_rt_poll(self._h, ticket)
        if rc < 0:
            raise RTError(rc, "mgcm_rt_poll")
        return rc

    def request_info(self, ticket: int) -> dict:
        """Timeline of a request not yet released by ``wait`` (host and
        device ms, jobs, HBM-budget deferrals)."""
        r = RequestInfo()
        rc = lib().mgcm_rt_get_request_info(self._h, ticket, C.byref(r))
        if rc != 0:
            raise RTError(rc, "mgcm_rt_get_request_info")
        return {k: getattr(r, k) for k, _ in RequestInfo._fields_}

    def wait(self, ticket: int, timeout_s: float = -1.0) -> None:
        rc = lib().mgcm_rt_wait(self._h, ticket, float(timeout_s))
        if rc == -8:
            raise RTError(rc, "mgcm_rt_wait")
        self._inflight.pop(ticket, None)
        if rc != 0:
            raise RTError(rc, "mgcm_rt_wait")

    def dsolflux(self, sol, acosz, detau, dndiffv):
        dev = _is_torch(acosz)
        if dev:
            import torch
            out = torch.empty_like(acosz)
            args = [sol, acosz, detau, dndiffv]
        else:
            args = [_host(sol), _host(acosz), _host(detau), _host(dndiffv)]
            out = np.zeros(args[1].shape[0])
        rc = lib().mgcm_rt_dsolflux(self._h, int(acosz.shape[0]), 1 if dev else 0,
                                    *[_ptr(a) for a in args], _ptr(out))
        if rc != 0:
            raise RTError(rc, "mgcm_rt_dsolflux")
        return out

    def debug_bins(self, b: dict) -> dict:
        """The integer bins the device stages for batch ``b`` (CUDA tensors):
        per level K = 1..LEV of each column MT, MP, NH2O, WRATIO, LCOEF(1..4)
        of TPINDEX (zeros at K = 1) and the Planck index INT(TLEV*10-499)."""
        import torch
        keep: list = []
        bi = make_in(b, True, keep)
        n, lev = int(b["ncol"]), 2 * int(b["L"]) + 3
        dev = b["plev"].device
        out = {k: torch.zeros(n, lev, dtype=torch.int32, device=dev) for k in ("mt", "mp", "nh2o", "nplanck")}
        out["wratio"] = torch.zeros(n, lev, dtype=torch.float64, device=dev)
        out["lcoef"] = torch.zeros(n, lev, 4, dtype=torch.float64, device=dev)
        rc = lib().mgcm_rt_debug_bins(self._h, C.byref(bi), *[out[k].data_ptr() for k in
                                      ("mt", "mp", "nh2o", "nplanck", "wratio", "lcoef")])
        if rc != 0:
            raise RTError(rc, "mgcm_rt_debug_bins")
        return out

    def stats(self) -> dict:
        s = Stats()
        lib().mgcm_rt_get_stats(self._h, C.byref(s))
        return {f: getattr(s, f) for f, _ in Stats._fields_}


def tables_host(data_dir) -> dict:
    """Set-up tables as the library builds them (no GPU needed)."""
    co2v = np.zeros(7 * 51 * 10 * 7 * 17)
    co2i = np.zeros(7 * 51 * 10 * 5 * 17)
    pl = np.zeros(5 * 8501)
    pf = np.zeros(51)
    rc = lib().mgcm_rt_tables_host(str(data_dir).encode(), co2v.ctypes.data_as(_D),
                                   co2i.ctypes.data_as(_D), pl.ctypes.data_as(_D),
                                   pf.ctypes.data_as(_D))
    if rc != 0:
        raise RTError(rc, "mgcm_rt_tables_host")
    return {"co2v": co2v, "co2i": co2i, "planckir": pl, "pfgasref": pf}


class Graph:
    """A captured set of batches: launch(stream) replays the whole radiation
    call of every batch; results land in .outs (DETAU/CUMTAUV in the batches)."""

    def __init__(self, rt: Radiation, g, outs, keep):
        self._rt, self._g, self.outs, self._keep = rt, g, outs, keep

    def launch(self, stream=None) -> None:
        ptr = None if stream is None else int(getattr(stream, "cuda_stream", stream))
        rc = lib().mgcm_rt_graph_launch(self._g, ptr)
        if rc != 0:
            raise RTError(rc, "mgcm_rt_graph_launch")

    def status(self) -> int:
        return lib().mgcm_rt_graph_status(self._g)

    def info(self) -> dict:
        t = Tune()
        rc = lib().mgcm_rt_graph_info(self._g, C.byref(t))
        if rc != 0:
            raise RTError(rc, "mgcm_rt_graph_info")
        return {k: getattr(t, k) for k, _ in Tune._fields_}

    def close(self) -> None:
        if self._g:
            lib().mgcm_rt_graph_destroy(self._g)
            self._g = None


def exported_symbols() -> list[str]:
    """Names declared in include/mgcm_rt.h."""
    import re
    hdr = pathlib.Path(__file__).resolve().parents[2] / "include" / "mgcm_rt.h"
    txt = hdr.read_text()
    return sorted(set(re.findall(r"\b(mgcm_rt_[a-z_]+)\s*\(", txt)))


__all__ = ["Radiation", "FP64", "MIXED", "RTError", "lib", "tables_host", "alloc_outputs",
           "exported_symbols", "INPUT_LEV", "INPUT_COL"]
