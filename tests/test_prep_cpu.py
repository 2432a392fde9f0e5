"""Column prep of the oracle (PL, FILLPT, QH2O, DUSTPROFILE, FILLTAUCUM)
against independent pure-Python statements of code/potemp1.f:95-106,
code/fillpt.f90:30-72, code/comp3.f:576-589, code/dustprofile.f:32-114,
code/filltaucum.f:39-55 and code/jsrchgt.f90 (libm exp/log/pow: agreement
to 1e-13 relative; the oracle uses the deterministic routines of
include/mgcm_rt_math.h, which the device uses too)."""
import math

import numpy as np
import pytest

import oracle
from mgcm_rt import synth

R4 = lambda x: float(np.float32(x))  # noqa: E731
NPDST = 100


# ---- pure-Python statements of the reference loops (1-based like Fortran)
def py_dust_grid(psf, ptrop):
    ex = float(np.float32(1.0) / (np.float32(NPDST) - np.float32(1.0)))   # REAL*4 exponent
    refpr = (5.0 * psf / ptrop) ** ex
    pr = [0.0] * (NPDST + 1)
    pr[1] = ptrop
    for n in range(2, NPDST + 1):
        pr[n] = refpr * pr[n - 1]
    return pr


def py_dust_profile(pr, rptau, conr, tautot):
    s = 0.0
    n = 2
    while n <= NPDST:
        if pr[n] < rptau:
            pave = 0.5 * (pr[n] + pr[n - 1])
            s = s + math.exp(conr * (1.0 - (rptau / pave))) * (pr[n] - pr[n - 1])
        if pr[n] >= rptau:
            break
        n += 1
    pave = 0.5 * (rptau + pr[n - 1])
    s = s + math.exp(conr * (1.0 - (rptau / pave))) * (rptau - pr[n - 1])
    q0 = tautot / s
    qr = [0.0] * (NPDST + 1)
    for n in range(1, NPDST):
        if rptau > pr[n + 1]:
            pave = 0.5 * (pr[n + 1] + pr[n])
            qr[n] = q0 * math.exp(conr * (1.0 - (rptau / pave)))
        if pr[n] <= rptau <= pr[n + 1]:
            pave = 0.5 * (pr[n] + rptau)
            qr[n] = q0 * (math.exp(conr * (1.0 - (rptau / pave))) * (rptau - pr[n]) + (pr[n + 1] - rptau)) \
                / (pr[n + 1] - pr[n])
        if rptau < pr[n]:
            qr[n] = q0
    td = [0.0] * (NPDST + 1)
    for n in range(2, NPDST + 1):
        td[n] = td[n - 1] + qr[n - 1] * (pr[n] - pr[n - 1])
    return td


def py_jsrchgt(sx, target):
    n = len(sx)
    if target > sx[n - 1]:
        return n + 1
    if target < sx[0]:
        return 1
    jl, jh = 1, n
    while jh - jl > 1:
        jm = (jl + jh) // 2
        if target > sx[jm - 1]:
            jl = jm
        else:
            jh = jm
    if target == sx[jh - 1]:
        jh += 1
    return jh


def py_prep_column(st, c):
    L = int(st["L"])
    lev = 2 * L + 3
    ptrop, p = float(st["ptrop"]), float(st["pcol"][c])
    sig = [0.0] + list(st["sigma"])
    pl = [0.0] * (lev + 1)
    for k in range(3, lev):
        pl[k] = ptrop + sig[k] * p
    pl[lev] = ptrop + p
    plev = [0.0] * (lev + 1)
    plev[1] = plev[2] = ptrop / 2.0
    for k in range(3, lev + 1):
        plev[k] = pl[k]
    tl = [0.0] * (lev + 1)
    for l in range(1, L + 1):
        tl[2 * l + 2] = float(st["t"][c, l - 1])
    tlev = [0.0] * (lev + 1)
    for k in (1, 2, 3):
        tlev[k] = float(st["tstrat"][c])
    for k in range(4, lev, 2):
        tlev[k] = tl[k]
    for k in range(5, lev - 1, 2):
        tlev[k] = tlev[k + 1] + (tlev[k - 1] - tlev[k + 1]) * math.log(plev[k] / plev[k + 1]) \
            / math.log(plev[k - 1] / plev[k + 1])
    tlev[lev] = float(st["gt"][c])
    tmid = [0.0] * (lev + 1)
    pmid = [0.0] * (lev + 1)
    tmid[1] = tmid[2] = tlev[2]
    pmid[1], pmid[2] = plev[1], plev[2]
    for l in range(1, L + 1):
        tmid[2 * l + 1] = tmid[2 * l + 2] = tlev[2 * l + 1]
        pmid[2 * l + 1] = pmid[2 * l + 2] = plev[2 * l + 1]
    tmid[lev], pmid[lev] = tlev[lev], plev[lev]
    qh = [0.0] * (lev + 1)
    for l in range(1, L + 1):
        k = 2 * l + 2
        qh[k] = float(st["mwratio"]) * float(st["vapour"][c, l - 1]) if st["active_water"] else R4(1.0e-7)
        qh[k + 1] = qh[k]
    out = dict(plev=plev[1:], tlev=tlev[1:], pmid=pmid[1:], tmid=tmid[1:], qh2o=qh[1:])
    if not st["active_dust"]:
        pr = py_dust_grid(float(st["psf"]), ptrop)
        td = py_dust_profile(pr, float(st["rptau"]), float(st["conr"][c]), float(st["tautot"][c]))
        tc = [0.0] * (lev + 1)
        tr = [0.0] * (lev + 2)
        for k in range(4, lev + 1):
            pstar = p * sig[k] + ptrop
            pstar1 = max(pstar, pr[1])
            ns = min(py_jsrchgt(pr[1:NPDST], pstar1) - 1, NPDST - 1)
            tc[k] = td[ns] + (pstar1 - pr[ns]) * (td[ns + 1] - td[ns]) / (pr[ns + 1] - pr[ns])
            tr[k] = tc[k] - tc[k - 1]
        out["tauref"] = tr[1:]
    return out


def test_jsrchgt_matches_statement_and_searchsorted():
    rng = np.random.default_rng(5)
    sx = np.sort(rng.uniform(0.0, 10.0, 37))
    targets = list(rng.uniform(-1.0, 11.0, 200)) + list(sx) + [sx[0], sx[-1], -5.0, 50.0]
    for t in targets:
        j = oracle.jsrchgt(sx, t)
        assert j == py_jsrchgt(list(sx), t)
        # first 1-based index with SX(j) > target (N+1 past the end)
        assert j == int(np.searchsorted(sx, t, side="right")) + 1


@pytest.mark.parametrize("psf,ptrop", [(7.01, 0.0008), (6.1, 0.0008), (9.5, 0.002)])
def test_dust_grid(psf, ptrop):
    got = oracle.dust_grid(psf, ptrop)
    ref = np.array(py_dust_grid(psf, ptrop)[1:])
    assert got[0] == ptrop
    assert np.all(np.diff(got) > 0)
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=0)
    # the top of the grid is 5 * PSF (code/dustprofile.f:32) up to the
    # REAL*4 rounding of the exponent 1/99 (about 1e-8 relative at the top)
    assert abs(got[-1] / (5.0 * psf) - 1.0) < 1e-7


@pytest.mark.parametrize("conr", [R4(0.03), 0.007, 0.04, R4(0.5)])
@pytest.mark.parametrize("rptau", [R4(6.1), 0.00085, 100.0])   # 0.00085: loop leaves at n = 2
def test_dust_profile(conr, rptau):
    pr = oracle.dust_grid(7.01, 0.0008)
    got = oracle.dust_profile(pr, rptau, conr, 0.37)
    ref = np.array(py_dust_profile([0.0] + list(pr), rptau, conr, 0.37)[1:])
    assert got[0] == 0.0
    assert np.all(np.diff(got) >= 0)
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-300)
    # linear in TAUTOT (qrdst0 = tautot / sum)
    got2 = oracle.dust_profile(pr, rptau, conr, 0.74)
    np.testing.assert_allclose(got2, 2.0 * got, rtol=1e-14, atol=0)


@pytest.mark.parametrize("L", [24, 36])
@pytest.mark.parametrize("active_dust,active_water,vary", [(False, True, False), (False, False, True),
                                                           (True, True, False)])
def test_prep_matches_statement(L, active_dust, active_water, vary):
    st = synth.make_state_batch(40, L=L, seed=11 + L, active_dust=active_dust, cloudon=False,
                                active_water=active_water, vary_conr=vary)
    tb = oracle.prep(st)
    for c in range(st["ncol"]):
        ref = py_prep_column(st, c)
        for k in ("plev", "pmid", "qh2o"):
            np.testing.assert_array_equal(tb[k][c], ref[k], err_msg=k)
        for k in ("tlev", "tmid"):
            np.testing.assert_allclose(tb[k][c], ref[k], rtol=1e-13, atol=0, err_msg=k)
        if not active_dust:
            tol = 1e-13 * float(st["tautot"][c])
            np.testing.assert_allclose(tb["tauref"][c], ref["tauref"], rtol=1e-12, atol=tol)
    if active_dust:
        assert tb["tauref"] is None


def test_prep_structure():
    """FILLPT's fixed points and the TAUREF bookkeeping of code/comp3.f:618."""
    st = synth.make_state_batch(64, L=24, seed=2, cloudon=False)
    tb = oracle.prep(st)
    lev = 2 * 24 + 3
    np.testing.assert_array_equal(tb["plev"][:, 0], st["ptrop"] / 2.0)
    np.testing.assert_array_equal(tb["plev"][:, lev - 1], st["ptrop"] + st["pcol"])
    np.testing.assert_array_equal(tb["tlev"][:, 2], st["tstrat"])
    np.testing.assert_array_equal(tb["tlev"][:, 3:lev - 1:2], st["t"])
    np.testing.assert_array_equal(tb["tlev"][:, lev - 1], st["gt"])
    np.testing.assert_array_equal(tb["tmid"][:, 2::2][:, :24], tb["tmid"][:, 3::2][:, :24])
    np.testing.assert_array_equal(tb["qh2o"][:, :3], 0.0)
    tr = tb["tauref"]
    np.testing.assert_array_equal(tr[:, :3], 0.0)
    np.testing.assert_array_equal(tr[:, lev], 0.0)
    assert np.all(tr >= 0.0)
    # odd TLEV lie between their even neighbours (log-pressure interpolation)
    lo = np.minimum(tb["tlev"][:, 3:lev - 3:2], tb["tlev"][:, 5:lev - 1:2])
    hi = np.maximum(tb["tlev"][:, 3:lev - 3:2], tb["tlev"][:, 5:lev - 1:2])
    mid = tb["tlev"][:, 4:lev - 2:2]
    assert np.all(mid >= lo - 1e-12) and np.all(mid <= hi + 1e-12)


@pytest.mark.parametrize("L", [1, 2, 99])
def test_prep_layer_count_edges(L):
    """FILLPT's interpolation loop is empty at L = 1 and one level long at
    L = 2; L = 99 is the largest layer count the library accepts."""
    st = synth.make_state_batch(8, L=L, seed=40 + L, active_dust=False, cloudon=False,
                                active_water=True, vary_conr=True)
    tb = oracle.prep(st)
    for c in range(st["ncol"]):
        ref = py_prep_column(st, c)
        for k in ("plev", "pmid", "qh2o"):
            np.testing.assert_array_equal(tb[k][c], ref[k], err_msg=k)
        for k in ("tlev", "tmid"):
            np.testing.assert_allclose(tb[k][c], ref[k], rtol=1e-13, atol=0, err_msg=k)
        tol = 1e-13 * float(st["tautot"][c])
        np.testing.assert_allclose(tb["tauref"][c], ref["tauref"], rtol=1e-12, atol=tol)
