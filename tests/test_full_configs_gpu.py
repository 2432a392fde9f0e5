"""Whole workloads on the GPU against the oracle, through the C ABI.

* 36 x 60 = 2,160 columns x 24 layers, dust only (the reference's default
  grid): FP64 within 1e-12 of the oracle.
* 180 x 360 = 64,800 columns x 24 layers, dust + water ice: FP64 within
  1e-12 of the oracle; MIXED within 1e-3 relative on every flux and 1e-2 K/sol
  on the heating rate (dT/dt = QRAD*OM over one sol of 88,775 s), against the
  oracle, not against the FP64 GPU path.
* The integer bins the device stages (TPINDEX's MT, MP, NH2O and the Planck
  index INT(TLEV*10-499)) equal the oracle's on every level of both
  workloads, of the edge batch, and of a batch whose pressures, temperatures
  and water mixing ratios sit exactly on, and one ulp either side of, every
  bin edge (code/tpindex.f90:72-134, code/sfluxi.f90:54-55,
  code/gfluxi.f90:73-74,86-87).  WRATIO and LCOEF come out bit-identical too.

The FP64 tolerances are those of tests/helpers.compare (flux floor 1e-3 of
the column's flux scale; divergences and QRAD scaled by the column's flux
scale).  The inputs are the bench's seeded workloads (mgcm_rt.synth)."""
import numpy as np
import pytest

import oracle
from helpers import compare, edge_batch, mixed_errors, to_numpy
from mgcm_rt import abi, synth

pytestmark = pytest.mark.gpu
RTOL = 1e-12
FLUX_TOL, HEAT_TOL = 1e-3, 1e-2

WORKLOADS = {"c0": dict(ncol=2160, L=24, cloud=False), "c1": dict(ncol=64800, L=24, cloud=True)}


@pytest.fixture(scope="module")
def batches(otables):
    out = {}
    for name, w in WORKLOADS.items():
        b = synth.make_batch(w["ncol"], L=w["L"], seed=1000, cloud=w["cloud"])
        out[name] = (b, oracle.run_batch(otables, b))
    return out


def _check(b, got, ref):
    err = compare(b, to_numpy(got), ref, RTOL)
    bad = {k: v for k, v in err.items() if not v <= RTOL}
    assert not bad, f"max normalised errors above {RTOL}: {bad}"


@pytest.mark.parametrize("name", ["c0", "c1"])
def test_fp64_whole_workload(data_dir, batches, name):
    b, ref = batches[name]
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=True)
    try:
        _check(b, rt.run(b), ref)
    finally:
        rt.close()


def test_mixed_whole_workload_within_tolerance(data_dir, batches):
    b, ref = batches["c1"]
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.MIXED, validate=True)
    try:
        got = rt.run(b)
    finally:
        rt.close()
    e = mixed_errors(b, got, ref)
    print("MIXED vs oracle, 64,800 x L24:", {k: f"{v:.3g}" for k, v in e.items()})
    assert e["flux_max"] <= FLUX_TOL, e
    assert e["heat_dT_Ksol_max"] <= HEAT_TOL, e
    # DETAU/CUMTAUV (in/out state) within the flux tolerance as well
    for k in ("detau", "cumtauv"):
        d = np.abs(np.asarray(got[k]) - ref[k]) / (np.abs(ref[k]) + 1e-30)
        assert float(d.max()) <= FLUX_TOL, (k, float(d.max()))


def _device(b):
    import torch
    return {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
            for k, v in b.items()}


def _edge_grid_batch(otables):
    """Three columns of 24 layers whose PMID run through every pressure bin
    limit (the exact largest double still in bin n, and the next one up),
    whose TMID sit on and one ulp around the 50 K grid, whose TLEV make
    T*10-499 land on and one ulp around integers, and whose QH2O sit on and
    one ulp around the WREFH2O grid."""
    b = synth.make_batch(6, L=24, seed=41, cloud=True, night_frac=0.0)
    lev = b["plev"].shape[1]

    def mp_of(p):
        return otables.tpindex(p, 200.0, 1e-5)[1]

    def last_in_bin(n):
        # largest p with MP <= n (log10(p) <= PREF(n+1)); bisect on the
        # ordered bit patterns of positive doubles
        lo = int(np.float64(1e-12).view(np.int64))
        hi = int(np.float64(1e6).view(np.int64))
        while hi - lo > 1:
            mid = (lo + hi) // 2
            if mp_of(float(np.int64(mid).view(np.float64))) <= n:
                lo = mid
            else:
                hi = mid
        return float(np.int64(lo).view(np.float64))

    edges = []
    for n in range(1, 50):
        p = last_in_bin(n)
        edges += [p, float(np.nextafter(p, np.inf))]
    ks = list(range(1, lev))          # 0-based levels 1..LEV-1 = K 2..LEV
    for i, p in enumerate(edges):
        c, k = divmod(i, len(ks))
        b["pmid"][c, ks[k]] = p
    tgrid = [50.0, 100.0, 150.0, 200.0, 250.0, 300.0]
    tv = [x for t in tgrid for x in (np.nextafter(t, 0), t, np.nextafter(t, 1e9))]
    for i, t in enumerate(tv):
        b["tmid"][3, 1 + i] = t
    # Planck: T*10-499 an integer (T = n/10) and one ulp around it
    pv = [x for t in (60.0, 149.9, 150.0, 200.1, 273.15, 279.9) for x in (np.nextafter(t, 0), t, np.nextafter(t, 1e9))]
    for i, t in enumerate(pv):
        b["tlev"][4, 1 + i] = t
    w = otables.view()["wrefh2o"]
    qv = [x for q in w for x in (np.nextafter(q, 0), q, np.nextafter(q, 1.0))]
    for i, q in enumerate(qv[: lev - 1]):
        b["qh2o"][5, 1 + i] = q
    return b


def _bins_equal(rt, otables, b):
    got = {k: v.cpu().numpy() for k, v in rt.debug_bins(_device(b)).items()}
    ref = oracle.bins_batch(otables, b)
    for k in ("mt", "mp", "nh2o", "nplanck"):
        diff = np.argwhere(got[k] != ref[k])
        assert diff.size == 0, f"{k}: {len(diff)} levels differ, first (col, level-1) {diff[:5].tolist()}"
    for k in ("wratio", "lcoef"):
        assert np.array_equal(got[k], ref[k]), f"{k} not bit-identical"
    return ref


def test_bins_bit_exact(data_dir, otables, batches):
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=True)
    try:
        for name in ("c0", "c1"):
            _bins_equal(rt, otables, batches[name][0])
        _bins_equal(rt, otables, edge_batch(otables))
        ref = _bins_equal(rt, otables, _edge_grid_batch(otables))
        # the edge batch really straddles the edges: every pressure bin 1..50
        # and every water bin 1..10 occurs
        assert set(np.unique(ref["mp"][:3, 1:])) >= set(range(1, 51))
        assert set(np.unique(ref["nh2o"][5, 1:])) == set(range(1, 11))
    finally:
        rt.close()


def test_bins_reject_host_pointers(data_dir):
    import ctypes as C
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64)
    try:
        b = synth.make_batch(2, L=24, seed=3)
        keep = []
        bi = abi.make_in(b, False, keep)
        z = np.zeros(2 * 51, dtype=np.int32)
        zd = np.zeros(2 * 51 * 4)
        rc = abi.lib().mgcm_rt_debug_bins(rt._h, C.byref(bi), *[z.ctypes.data] * 4, zd.ctypes.data,
                                          zd.ctypes.data)
        assert rc == -1
    finally:
        rt.close()


def _beyond_grid_batch():
    """Four columns whose TMID, PMID and QH2O lie beyond the ends of the
    k-table grids (TREF 50..350 K, the 51 reference pressures, WREFH2O);
    TPINDEX clamps them to the edge bins (code/tpindex.f90:72-134).  TLEV
    stays inside the Planck table."""
    b = synth.make_batch(4, L=24, seed=43, cloud=True, night_frac=0.0)
    b["tmid"][0, 1:] = 5.0
    b["tmid"][1, 1:] = 1000.0
    b["tmid"][2, 1::2] = 49.0
    b["tmid"][2, 2::2] = 351.0
    b["pmid"][0, 1:] = 1.0e-10
    b["pmid"][1, 1:] = 1.0e5
    b["qh2o"][2, 1:] = 0.0
    b["qh2o"][3, 1:] = 5.0
    return b


def test_bins_clamped_beyond_the_tables(data_dir, otables):
    """The k-table indices the device forms stay inside the tables whatever
    the state: MT in 1..6, MP in 1..50, NH2O in 1..10, and equal to the
    oracle's.  They are bounded by construction (every search falls back to
    an edge bin), so no gather can leave the table."""
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=True)
    try:
        b = _beyond_grid_batch()
        ref = _bins_equal(rt, otables, b)
        lv = slice(1, None)   # K = 2..LEV (K = 1 has no tpindex call)
        assert ref["mt"][:, lv].min() >= 1 and ref["mt"][:, lv].max() <= 6
        assert ref["mp"][:, lv].min() >= 1 and ref["mp"][:, lv].max() <= 50
        assert ref["nh2o"][:, lv].min() >= 1 and ref["nh2o"][:, lv].max() <= 10
        # the clamps are reached
        assert set(ref["mt"][0, lv]) == {1} and set(ref["mt"][1, lv]) == {6}
        assert set(ref["mp"][0, lv]) == {1} and set(ref["mp"][1, lv]) == {50}
        assert set(ref["nh2o"][2, lv]) == {1} and set(ref["nh2o"][3, lv]) == {10}
    finally:
        rt.close()


def test_planck_range_reported_without_validation(data_dir, otables):
    """With validation off, a TLEV outside the Planck table still ends the
    call with MGCM_RT_ETEMP: the kernels clamp the index INT(T*10-499) to
    1..8501 and raise a status flag (code/sfluxi.f90:54-55).  The handle
    stays usable, and the next batch matches the oracle."""
    rt = abi.Radiation(data_dir, max_layers=24, precision=abi.FP64, validate=False)
    try:
        b = synth.make_batch(8, L=24, seed=44, cloud=True)
        for t in (30.0, 950.0):
            bad = dict(b)
            bad["tlev"] = b["tlev"].copy()
            bad["tlev"][5, 9] = t
            with pytest.raises(abi.RTError) as e:
                rt.run(bad)
            assert e.value.code == -3
        _check(b, rt.run(b), oracle.run_batch(otables, b))
    finally:
        rt.close()
