"""CPU tests of the oracle (the checker) and of host-side logic; no GPU."""
import ctypes
import math

import numpy as np
import pytest

import oracle
from mgcm_rt import synth

R4 = lambda x: float(np.float32(x))  # noqa: E731


def test_solar_and_gauss_invariants(otables):
    v = otables.view()
    # setspv.f90:118-121: the seven REAL*4 band fluxes (sum 1356 W/m^2 at 1 AU)
    assert v["solarf"].sum() == pytest.approx(1356.1, abs=1e-4)
    assert v["solarf"][0] == R4(12.7)
    # modules.f90:335-345: Gauss split 0.95 / 0.05, point 17 weight 0
    assert v["gweight"][:8].sum() == pytest.approx(0.95, abs=1e-9)
    assert v["gweight"][8:16].sum() == pytest.approx(0.05, abs=1e-9)
    assert v["gweight"][16] == 0.0


def test_planck_table_integrates_to_sigma_t4(otables):
    v = otables.view()
    pl = v["planckir"].reshape(8501, 5)
    dw = v["dwni"]
    for T in (150.0, 200.0, 250.0, 300.0):
        it = int(T * 10.0 - 499)
        flux = math.pi * (pl[it - 1] * dw).sum()
        sigma_t4 = 5.67032e-8 * T ** 4
        # the five IR bands span 10-2222 cm-1: nearly all of B(T) at Mars temperatures
        assert 0.97 < flux / sigma_t4 <= 1.0 + 1e-6


def test_product_tables_bit_identical(data_dir, otables):
    from mgcm_rt import abi
    p = abi.tables_host(data_dir)
    v = otables.view()
    for k in ("co2v", "co2i", "planckir", "pfgasref"):
        assert np.array_equal(p[k], v[k]), k


def _libm_log10():
    m = ctypes.CDLL("libm.so.6")
    m.log10.restype = ctypes.c_double
    m.log10.argtypes = [ctypes.c_double]
    return m.log10


def test_tpindex_pressure_limits_reproduce_log10_bins(otables):
    """The device searches pressure bins by p <= plimit[n] instead of
    log10(p) <= PREF(n).  Rebuild plimit by the same bisection and check it
    reproduces the oracle's MP at and around every bin edge."""
    log10 = _libm_log10()
    pref = otables.view()["pfgasref"]
    lim = []
    for t in pref:
        lo, hi = np.float64(10.0 ** t * 0.5), np.float64(10.0 ** t * 2.0)
        a = lo.view(np.int64).item()
        b = hi.view(np.int64).item()
        while b - a > 1:
            m = (a + b) // 2
            if log10(np.int64(m).view(np.float64).item()) <= t:
                a = m
            else:
                b = m
        lim.append(np.int64(a).view(np.float64).item())
    rng = np.random.default_rng(3)
    ps = list(10.0 ** rng.uniform(-7, 5, 2000))
    for x in lim:
        for d in range(-3, 4):
            ps.append((np.float64(x).view(np.int64) + d).view(np.float64).item())
    for p in ps:
        mp_ref = otables.tpindex(p, 200.0, 1e-5)[1]
        mp = 50
        for n in range(2, 51):
            if p <= lim[n - 1]:
                mp = n - 1
                break
        assert mp == mp_ref, p


def test_tpindex_edges(otables):
    # temperature exactly on the reference grid goes to the lower bin
    assert otables.tpindex(1.0, 100.0, 0.0)[0] == 1
    assert otables.tpindex(1.0, 100.0000001, 0.0)[0] == 2
    assert otables.tpindex(1.0, 20.0, 0.0)[0] == 1
    assert otables.tpindex(1.0, 400.0, 0.0)[0] == 6
    # water: at or above WREFH2O(10) -> NH2O = 10, WRATIO = 0
    mt, mp, nh, wr, _ = otables.tpindex(1.0, 200.0, 0.4)
    assert nh == 10 and wr == 0.0
    mt, mp, nh, wr, _ = otables.tpindex(1.0, 200.0, 0.25)
    assert nh == 8 and wr == pytest.approx(0.5)


def test_night_column_has_no_visible_flux(otables):
    b = synth.make_batch(8, L=24, seed=5, cloud=True, night_frac=1.0)
    o = oracle.run_batch(otables, b, 1)
    for k in ("fmnetv", "fluxupv", "fluxdnv", "suntot"):
        assert not o[k].any()
    assert not o["dnvflux"].any() and not o["diffvt"].any()
    np.testing.assert_array_equal(o["detau"], b["detau"])      # kept for night
    np.testing.assert_array_equal(o["cumtauv"], b["cumtauv"])
    assert (o["fluxupi"] > 0).all()


def test_day_column_energy_bookkeeping(otables):
    b = synth.make_batch(16, L=24, seed=6, cloud=True, night_frac=0.0)
    o = oracle.run_batch(otables, b, 1)
    # incident solar at the top of the model: SOL * mu0 (all of it enters the
    # top "level" minus the tiny stratospheric attenuation)
    inc = b["sol"].sum() * b["acosz"]
    assert np.all(o["fluxdnv"][:, 0] <= inc * (1 + 1e-9))
    assert np.all(o["fluxdnv"][:, 0] > 0.9 * inc)
    # net flux at the top equals minus what the column plus surface absorbs
    assert np.all(o["nfluxtopv"] < 0)
    # the divergences sum to the top net flux difference
    np.testing.assert_allclose(o["suntot"].sum(1), o["fmnetv"][:, -1] - o["nfluxtopv"], rtol=1e-9)


def test_thin_atmosphere_limit(otables):
    """tau -> 0: with no dust, no cloud and a tiny column the visible
    downward flux at the surface approaches the incident beam."""
    b = synth.make_batch(4, L=24, seed=7, cloud=False, night_frac=0.0)
    b["plev"] = b["plev"] * 1e-4
    b["pmid"] = b["pmid"] * 1e-4
    b["pcol"] = b["pcol"] * 1e-4
    b["tauref"][:] = 0.0
    o = oracle.run_batch(otables, b, 1)
    inc = b["sol"].sum() * b["acosz"]
    np.testing.assert_allclose(o["fluxdnv"][:, -1], inc, rtol=2e-3)


def test_oracle_threads_match_serial(otables):
    b = synth.make_batch(40, L=24, seed=8, cloud=True)
    o1 = oracle.run_batch(otables, b, 1)
    o4 = oracle.run_batch(otables, b, 4)
    for k in o1:
        np.testing.assert_array_equal(o1[k], o4[k])


def test_synth_inputs_follow_reference_construction():
    b = synth.make_batch(32, L=24, seed=9, cloud=True)
    L = 24
    lev = 2 * L + 3
    assert b["plev"].shape == (32, lev) and b["qxvdst"].shape == (32, 7, lev + 1)
    # fillpt.f90: PLEV(1)=PLEV(2)=PTROP/2, monotone below; TMID pairs
    assert np.all(b["plev"][:, 0] == b["ptrop"] / 2) and np.all(np.diff(b["plev"][:, 1:], axis=1) >= 0)
    np.testing.assert_array_equal(b["tmid"][:, 2::2][:, :L], b["tmid"][:, 3::2][:, :L])
    # emiss.f90 sigma: sigma(L_LEVELS) = sum DSIG = 1
    assert synth.sigma_grid(24)[-1] == pytest.approx(1.0, abs=1e-6)
    for L2 in (36, 48):
        s = synth.sigma_grid(L2)
        assert s[-1] == pytest.approx(1.0, abs=1e-9) and np.all(np.diff(s[2::2]) > 0)
    # dust: TAUREF sums to about TAUTOT * (column fraction); non-negative
    assert np.all(b["tauref"] >= 0) and np.all(b["tauref"][:, -1] == 0)
    # clouds: TAUREFCLD/QEXTREFCLD present on 2..6 sub-levels per column
    nz = (b["taurefcld"] > 0).sum(1)
    assert np.all((nz >= 2) & (nz <= 6))


def test_dsolflux_oracle_matches_closed_form(otables):
    b = synth.make_batch(6, L=24, seed=10, night_frac=0.0)
    de = np.full((6, 17, 7), 0.3)
    ds = oracle.dsolflux(otables, b["sol"], b["acosz"], de)
    v = otables.view()
    gw, fz = v["gweight"], v["fzerov"]
    w = np.outer(gw[:16].sum() * np.ones(7), 1)[:, 0] * (1 - fz) + fz
    exp = (b["acosz"][:, None] * b["sol"][None, :] * np.exp(-0.3 / b["acosz"][:, None]) * w[None, :]).sum(1)
    np.testing.assert_allclose(ds, exp, rtol=1e-12)


def test_libm_sensitivity_of_reference_ir(data_dir, otables):
    """The reference IR two-stream amplifies one-ulp differences of EXP
    (EP-EM cancellation in thin layers); visible stays at rounding level.
    This bounds what any exp implementation can change."""
    from helpers import compare
    t2 = oracle.Tables(data_dir, variant="libm")
    b = synth.make_batch(64, L=24, seed=2, cloud=True)
    a = oracle.run_batch(otables, b)
    c = oracle.run_batch(t2, b)
    err = compare(b, c, a, 1e-12)
    assert err["fmnetv"] < 1e-11 and err["fluxdnv"] < 1e-11
    assert err["fmneti"] < 1e-4 and err["fluxupi"] < 1e-4
    assert 0 < max(err["fmneti"], err["fluxdni"])


def test_shared_exp_accuracy():
    import ctypes
    L = oracle.lib()
    m = ctypes.CDLL("libm.so.6")
    m.exp.restype = ctypes.c_double
    m.exp.argtypes = [ctypes.c_double]
    L.orc_exp.restype = ctypes.c_double
    L.orc_exp.argtypes = [ctypes.c_double]
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-40, 40, 20000), rng.uniform(-700, 700, 2000),
                         [0.0, -35.0, 35.0, 1e-300, -1e-300]])
    same = 0
    for x in xs:
        a, b = L.orc_exp(float(x)), m.exp(float(x))
        assert abs(a - b) <= math.ulp(b) * 1.0001
        same += a == b
    assert same / len(xs) > 0.99
    assert L.orc_exp(0.0) == 1.0


@pytest.mark.parametrize("name", ["c1_l24_cloud", "c0_l36_dust"])
def test_oracle_reproduces_golden_vectors(otables, name):
    """The oracle and the input recipe reproduce the committed fixtures
    (tests/golden/make_golden.py)."""
    import importlib.util
    import pathlib
    gdir = pathlib.Path(__file__).parent / "golden"
    spec = importlib.util.spec_from_file_location("make_golden", gdir / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    g = np.load(gdir / f"{name}.npz")
    b = mg.case(name)
    assert mg.inputs_digest(b) == str(g["digest"]), "input recipe changed"
    out = oracle.run_batch(otables, b)
    for k, v in out.items():
        np.testing.assert_allclose(np.asarray(v), g[k], rtol=1e-13, atol=1e-300, err_msg=k)


def test_operation_count_build_reproduces_the_oracle(data_dir, otables):
    """oracle/orc_count.cpp (the oracle with a counting number type) computes
    the same bits as the oracle and counts the operations
    bench/algorithmic_counts.json is built from."""
    import json
    import pathlib
    tc = oracle.Tables(data_dir, variant="count")
    b = synth.make_batch(24, L=24, seed=1000, cloud=True)
    ref = oracle.run_batch(otables, b, 1)
    got = {}
    cnt = oracle.op_counts(lambda: got.update(oracle.run_batch(tc, b, 1)))
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    # IR: 5 bands x 16 Gauss points x 50 levels x 8 corners per column;
    # visible: 7 x 16 x 50 x 8 per day column
    day = int(np.sum(np.asarray(b["acosz"]) >= 1.0e-5))
    assert cnt["gather"] == 24 * 5 * 16 * 50 * 8 + day * 7 * 16 * 50 * 8
    assert cnt["div"] > 0 and cnt["exp"] > 0 and cnt["sqrt"] > 0 and cnt["erf"] == 0
    frozen = json.loads((pathlib.Path(__file__).resolve().parents[1] / "bench" /
                         "algorithmic_counts.json").read_text())
    c1 = frozen["workloads"]["c1"]["per_column"]
    # the frozen per-column means are of the same order as this small sample's
    flops = sum(cnt[k] for k in ("add", "mul", "div", "sqrt", "exp", "log", "pow", "erf")) / 24
    assert 0.5 < flops / c1["flops"] < 2.0
