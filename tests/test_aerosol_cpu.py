"""Aerosol optics of the oracle (OPT_DST / OPT_CLD / prescribed dust) against
an independent numpy statement of code/opt_dst.f:55-161 and
code/opt_cld.f:55-188 (libm erf/log/pow; agreement to 1e-12 relative), plus
the table set-up and the deterministic erf/ln/pow of include/mgcm_rt_math.h."""
import ctypes
import math

import numpy as np
import pytest

import oracle
from mgcm_rt import synth

R4 = lambda x: float(np.float32(x))  # noqa: E731


@pytest.fixture(scope="module")
def aero(data_dir):
    return oracle.AeroTables(data_dir)


def _tables(data_dir):
    def read(name, n):
        v = np.array([np.float32(x) for x in (data_dir / name).read_text().split()], dtype=np.float64)
        assert v.size == n
        return v
    cv = read("waterCoated_vis_JD_12bands.dat", 15 * 20 * 3 * 7).reshape(15, 20, 3, 7)
    ci = read("waterCoated_ir_JD_12bands.dat", 15 * 20 * 3 * 5).reshape(15, 20, 3, 5)
    dv = read("Dust_vis_wolff2010_JD_12bands.dat", 20 * 3 * 7).reshape(20, 3, 7)
    di = read("Dust_ir_wolff2010_JD_12bands.dat", 20 * 3 * 5).reshape(20, 3, 5)
    athird = float(np.float32(1.0) / np.float32(3.0))
    rad = np.empty(20)
    radb = np.empty(21)
    rad[0], rad[19] = R4(1e-7), R4(50e-6)
    radb[0], radb[20] = R4(0.0001e-6), R4(1e-2)
    vrat = math.exp(math.log(rad[19] / rad[0]) / 19.0 * 3.0)
    for i in range(19):
        rad[i + 1] = rad[i] * vrat ** athird
        radb[i + 1] = ((2.0 * vrat) / (vrat + 1.0)) ** athird * rad[i]
    return cv, ci, dv, di, radb, athird


def _opt(L, pl, ma, mcor, nb, cld, tabs):
    cv, ci, dv, di, radb, athird = tabs
    lev1 = 2 * L + 4
    qr, tr = np.ones(lev1), np.zeros(lev1)
    xv, sv, gv = np.ones((7, lev1)), np.full((7, lev1), R4(0.99)), np.zeros((7, lev1))
    xi, si, gi = np.ones((5, lev1)), np.full((5, lev1), R4(0.99)), np.zeros((5, lev1))
    dev = R4(0.3087) if cld else R4(0.63676)
    dev2 = 1.0 / (R4(math.sqrt(2.0)) * dev)
    cor = np.array([0.1, 0.2, 0.25, 0.3, 0.35, 0.4, 0.45, 0.5, 0.55, 0.6, 0.65, 0.7, 0.8, 0.9, 0.99],
                   dtype=np.float32)
    for l in range(1, L + 1):
        if not cld:
            if not (ma[l - 1] > R4(1e-8) and nb[l - 1] > 1.0):
                continue
            Mo, No, dens = ma[l - 1], nb[l - 1] + 1.0, 2500.0
            tv, ti = dv, di
        else:
            if not (ma[l - 1] + mcor[l - 1] > R4(1e-7) and nb[l - 1] > 1.0):
                continue
            mtc = np.float32(mcor[l - 1] / 2500.0 / (ma[l - 1] / 917.0 + mcor[l - 1] / 2500.0))
            mtc = np.float32(float(mtc) ** athird)
            irap = 15
            for i in range(1, 16):
                if mtc < cor[i - 1] and i != 1:
                    irap = i - 1
                    break
                if mtc == cor[i - 1]:
                    irap = i
                    break
                if mtc < cor[i - 1] and i == 1:
                    irap = 1
                    break
            Mo, No = ma[l - 1] + mcor[l - 1], nb[l - 1]
            dens = ma[l - 1] / Mo * 917.0 + mcor[l - 1] / Mo * 2500.0
            tv, ti = cv[irap - 1], ci[irap - 1]
        cst = 0.75 / (math.pi * dens)
        Rs = (Mo / No * cst) ** athird * math.exp(-0.5 * dev * dev)
        Ao = No * math.pi * (Rs * Rs)
        Rs = Rs * math.exp(1.5 * dev * dev)
        Rs = 1.0 / min(max(Rs, R4(1e-7)), R4(100e-6) if cld else R4(50e-6))
        e = np.array([math.erf(math.log(r * Rs) * dev2) for r in radb])
        surf = 0.5 * (e[1:] - e[:-1])
        for nn in (1, 2):
            k = 2 * l + 1 + nn
            xv[:, k - 1] = surf @ tv[:, 0]
            sv[:, k - 1] = np.minimum(surf @ tv[:, 1], R4(0.99999) * xv[:, k - 1])
            gv[:, k - 1] = surf @ tv[:, 2]
            xi[:, k - 1] = surf @ ti[:, 0]
            si[:, k - 1] = np.minimum(surf @ ti[:, 1], R4(0.99999) * xi[:, k - 1])
            gi[:, k - 1] = surf @ ti[:, 2]
            qr[k - 1] = xv[5, k - 1]
            tr[k - 1] = Ao * qr[k - 1] * (100.0 * (pl[k - 1] - pl[k - 2]) / 3.72)
    return tr, qr, xv, sv, gv, xi, si, gi


@pytest.mark.parametrize("L", [5, 24])
def test_oracle_aerosols_match_independent_statement(data_dir, aero, L):
    tb = synth.make_tracer_batch(12, L=L, seed=300 + L, active_dust=True, cloudon=True)
    full = oracle.aerosols(aero, tb)
    tabs = _tables(data_dir)
    for c in range(12):
        d = _opt(L, tb["plev"][c], tb["dust_mass"][c], None, tb["dust_number"][c], False, tabs)
        d[0][:3] = 0.0
        d[0][-1] = 0.0
        k = _opt(L, tb["plev"][c], tb["ice_mass"][c], tb["ice_core_mass"][c], tb["ice_number"][c], True, tabs)
        for got, ref in zip([full[n][c] for n in ("tauref", "qextrefdst", "qxvdst", "qsvdst", "gvdst",
                                                  "qxidst", "qsidst", "gidst")], d):
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-300)
        for got, ref in zip([full[n][c] for n in ("taurefcld", "qextrefcld", "qxvcld", "qsvcld", "gvcld",
                                                  "qxicld", "qsicld", "gicld")], k):
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-300)


def test_tracer_batches_exercise_both_branches(data_dir):
    tb = synth.make_tracer_batch(64, L=24, seed=310, active_dust=True, cloudon=True)
    dust_on = (tb["dust_mass"] > np.float32(1e-8)) & (tb["dust_number"] > 1.0)
    ice_on = (tb["ice_mass"] + tb["ice_core_mass"] > np.float32(1e-7)) & (tb["ice_number"] > 1.0)
    assert dust_on.any() and (~dust_on).any()
    assert ice_on.any() and (~ice_on).any()


def test_prescribed_dust_is_band_constants(aero):
    tb = synth.make_tracer_batch(4, L=24, seed=311, active_dust=False, cloudon=False)
    full = oracle.aerosols(aero, tb)
    assert np.all(full["qxvdst"][:, 0, :] == 1.834) and np.all(full["gidst"][:, 4, :] == 0.316)
    assert np.all(full["qextrefdst"] == 2.452)
    np.testing.assert_array_equal(full["tauref"][:, :-1], tb["tauref"][:, :-1])
    assert np.all(full["tauref"][:, -1] == 0.0) and full["taurefcld"] is None


def test_deterministic_erf_ln_pow():
    lib = oracle.lib()
    for name in ("orc_erf", "orc_ln", "orc_pow"):
        getattr(lib, name).restype = ctypes.c_double
    lib.orc_erf.argtypes = lib.orc_ln.argtypes = [ctypes.c_double]
    lib.orc_pow.argtypes = [ctypes.c_double, ctypes.c_double]
    xs = np.concatenate([np.linspace(-7, 7, 14001), [1.5, 6.0, -1.5]])
    assert max(abs(lib.orc_erf(x) - math.erf(x)) for x in xs) < 1e-15
    ys = np.exp(np.linspace(-700, 700, 5001))
    assert max(abs(lib.orc_ln(y) - math.log(y)) / max(abs(math.log(y)), 1.0) for y in ys) < 5e-16
    zs = np.exp(np.linspace(-60, 10, 5001))
    assert max(abs(lib.orc_pow(z, 1 / 3) - z ** (1 / 3)) / z ** (1 / 3) for z in zs) < 5e-15
