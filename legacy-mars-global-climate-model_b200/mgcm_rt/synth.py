"""Seeded synthetic column batches with the reference's input construction.

There is no public dataset for this path; a batch is drawn from a seed with
the distributions of the workload definitions and then pushed through host
restatements of the reference routines that build the radiation inputs:

* sigma grid         code/emiss.f:103-115 with DSIG from code/modules.f90:731-737
* level pressures    code/potemp1.f:95-106, code/fillpt.f90:30-72
* dust profile       code/dustprofile.f:32-114 (Conrath, CONRNU=0.03, RPTAU=6.1)
                     and code/filltaucum.f:39-55
* dust optics        code/ini_optdst.f:44-61 with the Wolff constants of
                     code/setrad.f90:73-105
* water-ice optics   code/opt_cld.f:79-183 on the coated-sphere tables read by
                     code/initcld.f:141-172 (dev_ice = 0.3087)
* water vapour       QH2O = MWRATIO * q, code/comp3.f:576-589, code/input.f:180
* solar              SOL = SOLARF / RSDIST, code/comp3.f:300-304

Distributions: surface pressure U[400,1100] Pa; T0 ~ U[180,280] K at the
surface with a lapse rate U[1,3] K/km on z = (R T0 / g) ln(ps/p), clamped to
[140,280] K; ground temperature T0 + U[-10,10]; dust visible optical depth
lognormal(median 0.3, sigma 0.6) at RPTAU; vapour 0-50 pr-um uniform in the
column; cos(zenith) U[0,1] with a seeded half of the columns at night;
albedo U[0.1,0.4]; emissivity U[0.9,1.0].  Water-ice cloud (optional):
optical depth lognormal(median 0.05, sigma 1.0) spread over 1-3 contiguous
layers, effective radius U[1,5] um, core-ratio index U{1..15}.
"""
from __future__ import annotations

import math

import numpy as np

from . import data as _data

NV, NI, NG = 7, 5, 17

# code/modules.f90:731-737 (24-layer sigma thicknesses)
DSIG24 = np.array([
    0.0001237, 0.0002186, 0.0003877, 0.0006877, 0.0012199, 0.0021622,
    0.0038572, 0.0057287, 0.0094287, 0.0155443, 0.0256262, 0.0422609,
    0.0696418, 0.1148966, 0.1530633, 0.1572269, 0.1352191, 0.1212412,
    0.0718975, 0.0435678, 0.014, 0.008, 0.003, 0.001])

# code/constants_h (modules.f90:118-148)
GRAV, RGAS, CP, KAPA = 3.72, 189.02, 735.94, 0.25684
MWCO2, MWH2O = 4.41e-2, 1.80153e-2          # modules.f90:770-771
PTROP_TUTORIAL = 0.0008                     # tutorial/mars_tutorial:46 (mbar)
PSF_TUTORIAL = 7.010                        # tutorial/mars_tutorial:46
RPTAU, CONRNU, NPDST = 6.1, 0.03, 100       # modules.f90:854,874; L_NPDST
RSDIST_TUTORIAL = 2.4667                    # Ls ~ 5 deg, squared AU distance
SOLARF = np.array([12.7, 24.2, 54.6, 145.9, 354.9, 657.5, 106.3],
                  dtype=np.float32).astype(np.float64)   # setspv.f90:120-121 (REAL*4)

# Wolff dust constants (setrad.f90:73-105) and their derived Q arrays
QEV1 = np.array([1.834, 2.296, 2.672, 2.829, 2.698, 2.452, 2.261])
QSV1 = np.array([1.695, 2.031, 2.583, 2.744, 2.626, 2.225, 1.525])
GV1 = np.array([0.551, 0.640, 0.661, 0.678, 0.690, 0.743, 0.868])
QEI1 = np.array([0.008, 0.262, 0.491, 1.017, 0.444])
QSI1 = np.array([0.001, 0.037, 0.122, 0.351, 0.336])
GI1 = np.array([0.004, 0.030, 0.095, 0.214, 0.316])
NREFV = 6


def sigma_grid(L: int) -> np.ndarray:
    """SIGMA(1..2L+3) as code/emiss.f:103-115 builds it (SIGMA(1)=SIGMA(2)=0).

    L = 24 uses the reference DSIG.  Other L interpolate the cumulative sigma
    of the 24-layer set monotonically in normalised layer index (no reference
    sigma set exists for L = 36/48)."""
    if L == 24:
        dsig = DSIG24.copy()
    else:
        cum24 = np.concatenate([[0.0], np.cumsum(DSIG24)])
        cum24 /= cum24[-1]
        x24 = np.linspace(0.0, 1.0, 25)
        xL = np.linspace(0.0, 1.0, L + 1)
        # monotone (piecewise cubic Hermite, Fritsch-Carlson) in index space
        cumL = _pchip(x24, cum24, xL)
        dsig = np.diff(cumL)
    lev = 2 * L + 3
    sig = np.zeros(lev)
    for k in range(1, L + 1):           # SIGMA(2K+3) = SIGMA(2K+1) + DSIG(K)
        sig[2 * k + 2] = sig[2 * k] + dsig[k - 1]
    for k in range(4, lev, 2):          # SIGMA(K) = 0.5*(SIGMA(K+1)+SIGMA(K-1))
        sig[k - 1] = 0.5 * (sig[k] + sig[k - 2])
    return sig


def _pchip(x, y, xq):
    h = np.diff(x)
    d = np.diff(y) / h
    m = np.zeros_like(y)
    for i in range(1, len(y) - 1):
        if d[i - 1] * d[i] > 0:
            w1, w2 = 2 * h[i] + h[i - 1], h[i] + 2 * h[i - 1]
            m[i] = (w1 + w2) / (w1 / d[i - 1] + w2 / d[i])
    m[0], m[-1] = d[0], d[-1]
    idx = np.clip(np.searchsorted(x, xq, side="right") - 1, 0, len(h) - 1)
    t = (xq - x[idx]) / h[idx]
    h00, h10 = 2 * t**3 - 3 * t**2 + 1, t**3 - 2 * t**2 + t
    h01, h11 = -2 * t**3 + 3 * t**2, t**3 - t**2
    return h00 * y[idx] + h10 * h[idx] * m[idx] + h01 * y[idx + 1] + h11 * h[idx] * m[idx + 1]


def dust_profile_grid(ptrop: float, psf: float = PSF_TUTORIAL):
    """PRDST and the unit-TAUTOT cumulative optical depth TAUDST/TAUTOT on it
    (code/dustprofile.f:32-114 with a spatially constant CONRNU)."""
    refpr = (5.0 * psf / ptrop) ** (1.0 / (float(NPDST) - 1.0))
    prdst = np.empty(NPDST)
    prdst[0] = ptrop
    for n in range(1, NPDST):
        prdst[n] = refpr * prdst[n - 1]
    conr = CONRNU
    s = 0.0
    n = 1
    while n < NPDST:
        if prdst[n] < RPTAU:
            pave = 0.5 * (prdst[n] + prdst[n - 1])
            s += math.exp(conr * (1.0 - RPTAU / pave)) * (prdst[n] - prdst[n - 1])
        if prdst[n] >= RPTAU:
            break
        n += 1
    pave = 0.5 * (RPTAU + prdst[n - 1])
    s += math.exp(conr * (1.0 - RPTAU / pave)) * (RPTAU - prdst[n - 1])
    q0 = 1.0 / s
    qr = np.zeros(NPDST)
    for n in range(NPDST - 1):
        if RPTAU > prdst[n + 1]:
            pave = 0.5 * (prdst[n + 1] + prdst[n])
            qr[n] = q0 * math.exp(conr * (1.0 - RPTAU / pave))
        if prdst[n] <= RPTAU <= prdst[n + 1]:
            pave = 0.5 * (prdst[n] + RPTAU)
            qr[n] = q0 * (math.exp(conr * (1.0 - RPTAU / pave)) * (RPTAU - prdst[n])
                          + (prdst[n + 1] - RPTAU)) / (prdst[n + 1] - prdst[n])
        if RPTAU < prdst[n]:
            qr[n] = q0
    taud = np.zeros(NPDST)
    for n in range(1, NPDST):
        taud[n] = taud[n - 1] + qr[n - 1] * (prdst[n] - prdst[n - 1])
    return prdst, taud


def _ice_bins():
    """radb_rt of code/initcld.f:141-156."""
    nbin = 20
    rad = np.empty(nbin)
    radb = np.empty(nbin + 1)
    rad[0], rad[-1] = 1.0e-7, 50.0e-6
    radb[0], radb[-1] = 0.0001e-6, 1.0e-2
    vrat = math.exp(math.log(rad[-1] / rad[0]) / float(nbin - 1) * 3.0)
    for i in range(nbin - 1):
        rad[i + 1] = rad[i] * vrat ** (1.0 / 3.0)
        radb[i + 1] = ((2.0 * vrat) / (vrat + 1.0)) ** (1.0 / 3.0) * rad[i]
    return radb


def _erf(x):
    return np.vectorize(math.erf)(x)


def make_batch(ncol: int, L: int = 24, seed: int = 0, cloud: bool = False,
               night_frac: float = 0.5, ptrop: float = PTROP_TUTORIAL,
               rsdist: float = RSDIST_TUTORIAL, data_dir=None) -> dict:
    """Build a batch dict of float64 arrays in the library's layout.

    Shapes: level arrays (ncol, 2L+3); level+1 arrays (ncol, 2L+4); band
    arrays (ncol, NB, 2L+4); per-column scalars (ncol,); DETAU and CUMTAUV
    (ncol, 17, 7) seeded with the reference's first-call values (DETAU = 0.1,
    comp3.f:1200-1228; CUMTAUV = 0)."""
    rng = np.random.default_rng(seed)
    lev = 2 * L + 3
    lev1 = lev + 1
    sig = sigma_grid(L)

    ps = rng.uniform(400.0, 1100.0, ncol) / 100.0          # mbar
    p = ps - ptrop                                         # P(J,I)
    t0 = rng.uniform(180.0, 280.0, ncol)
    gam = rng.uniform(1.0, 3.0, ncol)
    gt = t0 + rng.uniform(-10.0, 10.0, ncol)

    # PL (potemp1.f:95-106): PL(K) = PTROP + SIGMA(K) P, PL(2) = PTROP/2
    pl = np.empty((ncol, lev))
    pl[:, 0] = 0.0
    pl[:, 1] = ptrop / 2.0
    pl[:, 2:lev - 1] = ptrop + sig[None, 2:lev - 1] * p[:, None]
    pl[:, lev - 1] = ptrop + p

    def temp_at(pp):
        z = (RGAS * t0[:, None] / GRAV) * np.log(ps[:, None] / pp) / 1000.0
        return np.clip(t0[:, None] - gam[:, None] * z, 140.0, 280.0)

    tl = temp_at(np.maximum(pl, 1e-30))
    tstrat = tl[:, 1]                                      # stratosphere layer

    # fillpt.f90:30-72
    plev = np.empty((ncol, lev))
    plev[:, 0] = ptrop / 2.0
    plev[:, 1] = ptrop / 2.0
    plev[:, 2:] = pl[:, 2:]
    tlev = np.empty((ncol, lev))
    tlev[:, 0:3] = tstrat[:, None]
    for k in range(4, lev, 2):                              # K=4..L_LEVELS-1 step 2
        tlev[:, k - 1] = tl[:, k - 1]
    for k in range(5, lev - 1, 2):                          # K=5..L_LEVELS-2 step 2
        tlev[:, k - 1] = tlev[:, k] + (tlev[:, k - 2] - tlev[:, k]) * \
            np.log(plev[:, k - 1] / plev[:, k]) / np.log(plev[:, k - 2] / plev[:, k])
    tlev[:, lev - 1] = gt
    tmid = np.empty((ncol, lev))
    pmid = np.empty((ncol, lev))
    tmid[:, 0] = tmid[:, 1] = tlev[:, 1]
    pmid[:, 0] = plev[:, 0]
    pmid[:, 1] = plev[:, 1]
    for l in range(1, L + 1):
        tmid[:, 2 * l] = tmid[:, 2 * l + 1] = tlev[:, 2 * l]
        pmid[:, 2 * l] = pmid[:, 2 * l + 1] = plev[:, 2 * l]
    tmid[:, lev - 1] = tlev[:, lev - 1]
    pmid[:, lev - 1] = plev[:, lev - 1]

    # water vapour: QH2O(K) = MWRATIO * q for K = 4..L_LEVELS, 0 above
    wpr = rng.uniform(0.0, 50.0, ncol)                     # pr-um
    q = (wpr * 1.0e-3) / (ps * 100.0 / GRAV)
    qh2o = np.zeros((ncol, lev))
    qh2o[:, 3:] = (q * (MWCO2 / MWH2O))[:, None]

    # dust: Conrath profile scaled to TAUTOT, sampled by filltaucum
    tautot = 0.3 * np.exp(0.6 * rng.standard_normal(ncol))
    prdst, taud1 = dust_profile_grid(ptrop)
    tauref = np.zeros((ncol, lev1))
    taucum = np.zeros((ncol, lev))
    for k in range(4, lev + 1):
        pstar = p * sig[k - 1] + ptrop
        pstar1 = np.maximum(pstar, prdst[0])
        nstar = np.minimum(np.searchsorted(prdst[:NPDST - 1], pstar1, side="right"), NPDST - 1)
        i0 = nstar - 1
        frac = (pstar1 - prdst[i0]) / (prdst[i0 + 1] - prdst[i0])
        taucum[:, k - 1] = tautot * (taud1[i0] + frac * (taud1[i0 + 1] - taud1[i0]))
        tauref[:, k - 1] = taucum[:, k - 1] - taucum[:, k - 2]
    tauref[:, lev] = 0.0                                    # comp3.f:615

    qscv = np.where(QSV1 >= QEV1, np.float32(0.99999) * QEV1, QSV1)
    qsci = np.where(QSI1 >= QEI1, np.float32(0.99999) * QEI1, QSI1)
    qxvdst = np.broadcast_to(QEV1[None, :, None], (ncol, NV, lev1)).copy()
    qsvdst = np.broadcast_to(qscv[None, :, None], (ncol, NV, lev1)).copy()
    gvdst = np.broadcast_to(GV1[None, :, None], (ncol, NV, lev1)).copy()
    qxidst = np.broadcast_to(QEI1[None, :, None], (ncol, NI, lev1)).copy()
    qsidst = np.broadcast_to(qsci[None, :, None], (ncol, NI, lev1)).copy()
    gidst = np.broadcast_to(GI1[None, :, None], (ncol, NI, lev1)).copy()
    qextrefdst = np.full((ncol, lev1), QEV1[NREFV - 1])

    acosz = rng.uniform(0.0, 1.0, ncol)
    night = rng.uniform(0.0, 1.0, ncol) < night_frac
    acosz[night] = 0.0
    als = rng.uniform(0.1, 0.4, ncol)
    albi = 1.0 - rng.uniform(0.9, 1.0, ncol)

    out = dict(
        L=L, ncol=ncol, ptrop=float(ptrop), sigma=sig, sol=SOLARF / rsdist,
        plev=plev, tlev=tlev, pmid=pmid, tmid=tmid, qh2o=qh2o,
        tauref=tauref, qextrefdst=qextrefdst,
        qxvdst=qxvdst, qsvdst=qsvdst, gvdst=gvdst,
        qxidst=qxidst, qsidst=qsidst, gidst=gidst,
        acosz=acosz, als=als, albi=albi, pcol=p,
        detau=np.full((ncol, NG, NV), 0.1), cumtauv=np.zeros((ncol, NG, NV)),
    )
    meta = {"seed": seed, "cloud": bool(cloud), "night_frac": night_frac}
    if cloud:
        ice, kind = _ice_clouds(rng, ncol, L, pl, data_dir)
        out.update(ice)
        meta["ice_optics"] = kind
    out["meta"] = meta
    return out


def _ice_clouds(rng, ncol, L, pl, data_dir):
    """Per-level ice inputs as code/opt_cld.f:55-183 fills them."""
    lev = 2 * L + 3
    lev1 = lev + 1
    tab = _data.read_ice_tables(data_dir)
    qxv = np.ones((ncol, NV, lev1))
    qsv = np.full((ncol, NV, lev1), 0.99)
    gv = np.zeros((ncol, NV, lev1))
    qxi = np.ones((ncol, NI, lev1))
    qsi = np.full((ncol, NI, lev1), 0.99)
    gi = np.zeros((ncol, NI, lev1))
    qextref = np.ones((ncol, lev1))
    tauc = np.zeros((ncol, lev1))

    tau_ice = 0.05 * np.exp(1.0 * rng.standard_normal(ncol))
    nlay = rng.integers(1, 4, ncol)
    lo, hi = max(1, L // 3), max(2, L - 3)
    start = rng.integers(lo, hi, ncol)
    reff = rng.uniform(1.0e-6, 5.0e-6, ncol)
    irap = rng.integers(0, 15, ncol)

    dev = 0.3087
    dev2 = 1.0 / (math.sqrt(2.0) * dev)
    radb = _ice_bins()
    rs = 1.0 / np.clip(reff, 1.0e-7, 100.0e-6)
    e = _erf(np.log(radb[None, :] * rs[:, None]) * dev2)
    surf = 0.5 * (e[:, 1:] - e[:, :-1])                       # (ncol, 20)
    if tab is not None:
        cxv = np.einsum("cb,cbw->cw", surf, tab["qextv"][irap])
        csv = np.einsum("cb,cbw->cw", surf, tab["qscatv"][irap])
        cgv = np.einsum("cb,cbw->cw", surf, tab["gv"][irap])
        cxi = np.einsum("cb,cbw->cw", surf, tab["qexti"][irap])
        csi = np.einsum("cb,cbw->cw", surf, tab["qscati"][irap])
        cgi = np.einsum("cb,cbw->cw", surf, tab["gi"][irap])
    else:   # tables absent: fixed plausible ice properties (labelled in meta)
        cxv = np.full((ncol, NV), 2.1)
        csv = np.full((ncol, NV), 2.09)
        cgv = np.full((ncol, NV), 0.80)
        cxi = np.linspace(0.6, 1.6, NI)[None, :].repeat(ncol, 0)
        csi = 0.5 * cxi
        cgi = np.full((ncol, NI), 0.3)
    csv = np.minimum(csv, np.float32(0.99999) * cxv)
    csi = np.minimum(csi, np.float32(0.99999) * cxi)

    cols = np.arange(ncol)
    mass_tot = np.zeros(ncol)
    for j in range(3):
        on = j < nlay
        layer = np.minimum(start + j, L)
        for nn in (1, 2):
            k = 2 * layer + 1 + nn                               # 1-based level
            m = 100.0 * (pl[cols, k - 1] - pl[cols, k - 2]) / GRAV
            mass_tot += np.where(on, m, 0.0)
    for j in range(3):
        on = j < nlay
        layer = np.minimum(start + j, L)
        for nn in (1, 2):
            k = 2 * layer + 1 + nn
            c = cols[on]
            kk = k[on] - 1
            qxv[c, :, kk] = cxv[on]
            qsv[c, :, kk] = csv[on]
            gv[c, :, kk] = cgv[on]
            qxi[c, :, kk] = cxi[on]
            qsi[c, :, kk] = csi[on]
            gi[c, :, kk] = cgi[on]
            qextref[c, kk] = cxv[on, NREFV - 1]
            m = 100.0 * (pl[c, kk] - pl[c, kk - 1]) / GRAV
            tauc[c, kk] = tau_ice[on] * m / mass_tot[on]
    return (dict(taurefcld=tauc, qextrefcld=qextref, qxvcld=qxv, qsvcld=qsv, gvcld=gv,
                 qxicld=qxi, qsicld=qsi, gicld=gi),
            "tables" if tab is not None else "fixed-properties")


def make_tracer_batch(ncol: int, L: int = 24, seed: int = 0, active_dust: bool = True,
                      cloudon: bool = True, night_frac: float = 0.5, data_dir=None):
    """Inputs of mgcm_rt_run_tracers: the column state of make_batch (dust
    off, its Conrath TAUREF kept for prescribed dust) plus per-layer tracer
    mixing ratios as COMP3's QTRACE holds them (code/comp3.f:592-630):
      dust  mass Ma [kg/kg] and number Nb [1/kg] sized so that OPT_DST gives
            roughly the Conrath profile's optical depth (effective radius
            U[0.8, 2.0] um per column); layers of negligible dust fall below
            OPT_DST's thresholds;
      ice   1-3 contiguous layers with ice mass, core (dust) mass and number
            (radius U[1, 5] um, optical depth lognormal(0.05, 1), core mass
            fraction U[0, 0.5])."""
    b = make_batch(ncol, L=L, seed=seed, cloud=False, night_frac=night_frac, data_dir=data_dir)
    rng = np.random.default_rng(seed + 7919)
    lev = 2 * L + 3
    pl = b["plev"]
    mass = np.empty((ncol, L))   # kg/m^2 of the layer's first radiation level pair
    for l in range(1, L + 1):
        k = 2 * l + 2
        mass[:, l - 1] = 100.0 * (pl[:, k - 1] - pl[:, k - 3]) / GRAV
    t = {k: v for k, v in b.items() if k not in (
        "qextrefdst", "qxvdst", "qsvdst", "gvdst", "qxidst", "qsidst", "gidst")}
    t["active_dust"] = 1 if active_dust else 0
    t["cloudon"] = 1 if cloudon else 0
    if active_dust:
        r = rng.uniform(0.8e-6, 2.0e-6, ncol)[:, None]
        tau = np.empty((ncol, L))
        for l in range(1, L + 1):
            tau[:, l - 1] = b["tauref"][:, 2 * l + 1] + b["tauref"][:, 2 * l + 2]
        no = tau / (math.pi * r * r * 2.5 * np.maximum(mass, 1e-12))
        ma = no * (4.0 / 3.0) * math.pi * r ** 3 * 2500.0
        t["dust_number"] = no
        t["dust_mass"] = ma
    else:
        t["dust_number"] = None
        t["dust_mass"] = None
    if cloudon:
        ima = np.zeros((ncol, L))
        icor = np.zeros((ncol, L))
        inb = np.zeros((ncol, L))
        tau_ice = 0.05 * np.exp(rng.standard_normal(ncol))
        nlay = rng.integers(1, 4, ncol)
        start = rng.integers(max(1, L // 3), max(2, L - 3), ncol)
        r = rng.uniform(1.0e-6, 5.0e-6, ncol)
        fcor = rng.uniform(0.0, 0.5, ncol)
        for j in range(3):
            on = j < nlay
            l = np.minimum(start + j, L)
            c = np.arange(ncol)[on]
            m = mass[c, l[on] - 1]
            n = tau_ice[on] / nlay[on] / (math.pi * r[on] ** 2 * 2.0 * np.maximum(m, 1e-12))
            mtot = n * (4.0 / 3.0) * math.pi * r[on] ** 3 * 917.0
            inb[c, l[on] - 1] = n
            icor[c, l[on] - 1] = fcor[on] * mtot
            ima[c, l[on] - 1] = (1.0 - fcor[on]) * mtot
        t["ice_mass"], t["ice_core_mass"], t["ice_number"] = ima, icor, inb
    else:
        t["ice_mass"] = t["ice_core_mass"] = t["ice_number"] = None
    t["meta"] = dict(b["meta"], tracers=True)
    return t


def make_state_batch(ncol: int, L: int = 24, seed: int = 0, active_dust: bool = False,
                     cloudon: bool = True, active_water: bool = True, vary_conr: bool = False,
                     night_frac: float = 0.5, data_dir=None):
    """Inputs of mgcm_rt_run_state: the GCM state of each column, before
    COMP3 assembles the radiation arrays.  The columns of make_tracer_batch
    (same seed) supply P(J,I), the tracers and the surface; from them:
      t        TL(2l+2), the layer temperatures (the lapse-rate profile at
               the layer mid-pressures), [ncol][L]
      tstrat   the stratosphere temperature TL(2); gt the ground temperature
      vapour   the water-vapour mass mixing ratio, uniform in the column
      tautot   dust visible optical depth at RPTAU, lognormal(median 0.3,
               sigma 0.6) (prescribed dust)
      conr     the Conrath parameter: CONRNU (REAL*4 0.03,
               code/modules.f90:874) or, with vary_conr, U[0.007, 0.04] (the
               range of the latitude-varying form, code/dustprofile.f:43-53)
    psf = 7.010 mbar (the tutorial namelist), RPTAU the module's REAL*4 6.1
    (code/modules.f90:854), MWRATIO = MWCO2/MWH2O (code/input.f:180)."""
    b = make_tracer_batch(ncol, L=L, seed=seed, active_dust=active_dust, cloudon=cloudon,
                          night_frac=night_frac, data_dir=data_dir)
    rng = np.random.default_rng(seed + 104729)
    lev = 2 * L + 3
    tlev = b["tlev"]
    st = {k: b[k] for k in ("ncol", "L", "ptrop", "sigma", "sol", "pcol", "acosz", "als", "albi",
                            "detau", "cumtauv", "dust_mass", "dust_number", "ice_mass",
                            "ice_core_mass", "ice_number", "active_dust", "cloudon")}
    st["t"] = np.ascontiguousarray(tlev[:, 3:lev - 1:2])      # K = 4, 6, .., 2L+2
    st["tstrat"] = tlev[:, 0].copy()
    st["gt"] = tlev[:, lev - 1].copy()
    mwratio = MWCO2 / MWH2O
    st["active_water"] = 1 if active_water else 0
    st["mwratio"] = mwratio
    st["vapour"] = np.repeat((b["qh2o"][:, 3] / mwratio)[:, None], L, axis=1) if active_water else None
    st["psf"] = PSF_TUTORIAL
    st["rptau"] = float(np.float32(RPTAU))
    if not active_dust:
        st["tautot"] = 0.3 * np.exp(0.6 * rng.standard_normal(ncol))
        st["conr"] = (rng.uniform(0.007, 0.04, ncol) if vary_conr
                      else np.full(ncol, float(np.float32(CONRNU))))
    else:
        st["tautot"] = st["conr"] = None
    st["meta"] = dict(b["meta"], state=True, vary_conr=bool(vary_conr))
    return st
