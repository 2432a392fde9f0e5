"""Comparison helpers for the parity tests."""
import numpy as np

from mgcm_rt import OUTPUT_COL, OUTPUT_LAY, synth

FLUX_LAY = ("fmnetv", "fluxupv", "fluxdnv", "fmneti", "fluxupi", "fluxdni")
DIV_LAY = ("suntot", "irtotal")
CP, GRAV, KAPA = 735.94, 3.72, 0.25684


def flux_scale(ref):
    """Per-column flux magnitude: largest |flux| of the column (W/m^2)."""
    s = np.zeros(ref["fluxupi"].shape[0])
    for k in FLUX_LAY:
        s = np.maximum(s, np.abs(ref[k]).max(axis=1))
    return s


def heating_scale(b, ref):
    """Per-layer K/s that one W/m^2 of flux-divergence error makes in QRAD."""
    plev = np.asarray(b["plev"])
    L = int(b["L"])
    nl = L + 1
    lev = 2 * L + 3
    ym = np.empty((plev.shape[0], nl))
    om = np.empty_like(ym)
    for l in range(1, nl + 1):
        k = 2 * l
        ym[:, l - 1] = (float(b["ptrop"]) * 100.0 / GRAV if k == 2
                        else (plev[:, k] - plev[:, k - 2]) * 100.0 / GRAV)
        om[:, l - 1] = (plev[:, k - 1] / plev[:, lev - 1]) ** KAPA
    return 1.0 / (CP * ym * om)


def compare(b, got, ref, rtol):
    """Max error per output, normalised:
    fluxes:    |d| / (|ref| + rtol-floor at the column's flux scale)
    SUNTOT/IRTOTAL, scalars: |d| / column flux scale
    QRAD:      |d| / (column flux scale * heating scale)
    Returns dict name -> max normalised error (pass when <= rtol)."""
    fs = flux_scale(ref)[:, None]
    hs = heating_scale(b, ref)
    err = {}
    for k in FLUX_LAY:
        d = np.abs(np.asarray(got[k]) - ref[k])
        err[k] = float((d / (np.abs(ref[k]) + fs * 1e-3 + 1e-300)).max()) if d.size else 0.0
    for k in DIV_LAY:
        d = np.abs(np.asarray(got[k]) - ref[k])
        err[k] = float((d / (fs + 1e-300)).max()) if d.size else 0.0
    d = np.abs(np.asarray(got["qrad"]) - ref["qrad"])
    err["qrad"] = float((d / (fs * hs + 1e-300)).max()) if d.size else 0.0
    for k in OUTPUT_COL:
        d = np.abs(np.asarray(got[k]) - ref[k])
        err[k] = float((d / (fs[:, 0] + 1e-300)).max()) if d.size else 0.0
    for k in ("detau", "cumtauv"):
        d = np.abs(np.asarray(got[k]) - ref[k])
        err[k] = float((d / (np.abs(ref[k]) + 1e-300)).max()) if d.size else 0.0
    return err


def to_numpy(o):
    out = {}
    for k, v in o.items():
        out[k] = v.detach().cpu().numpy() if hasattr(v, "detach") else np.asarray(v)
    return out


def mixed_errors(b, got, ref):
    """Accuracy summary of a mixed-precision run against FP64:
    max relative flux error (floor 1e-3 of the column flux scale) and the
    heating-rate error in K/sol, both as dT/dt = QRAD*OM (temperature) and
    as QRAD itself (potential temperature)."""
    got = to_numpy(got)
    fs = flux_scale(ref)[:, None]
    out = {}
    for k in FLUX_LAY:
        d = np.abs(got[k] - ref[k]) / (np.abs(ref[k]) + 1e-3 * fs)
        out[k] = float(d.max()) if d.size else 0.0
    out["flux_max"] = max(out[k] for k in FLUX_LAY)
    plev = np.asarray(b["plev"])
    L = int(b["L"])
    lev = 2 * L + 3
    om = np.stack([(plev[:, 2 * l - 1] / plev[:, lev - 1]) ** KAPA for l in range(1, L + 2)], 1)
    dth = np.abs(got["qrad"] - ref["qrad"]) * 88775.0
    out["heat_dT_Ksol_max"] = float((dth * om).max()) if dth.size else 0.0
    out["heat_dT_Ksol_rms"] = float(np.sqrt(((dth * om) ** 2).mean())) if dth.size else 0.0
    out["heat_dtheta_Ksol_max"] = float(dth.max()) if dth.size else 0.0
    return out


def edge_batch(otables):
    """Columns whose inputs sit on bin edges: pressures at the tpindex
    limits, temperatures on the 50 K grid and at the Planck table ends,
    humidity at and beyond the water grid ends, the day threshold."""
    b = synth.make_batch(12, L=24, seed=12, cloud=True, night_frac=0.0)
    pref = otables.view()["pfgasref"]
    lev = b["plev"].shape[1]
    # pressures: put PMID of some levels exactly at 10**PREF and one ulp off
    for c, n in enumerate((20, 25, 30, 33)):
        p = 10.0 ** pref[n]
        for k in range(4, lev, 7):
            b["pmid"][c, k] = np.nextafter(p, 0) if k % 2 else p
    # temperatures exactly on the 50 K grid
    b["tmid"][4, 3:] = 200.0
    b["tmid"][5, 3:] = 150.0
    # Planck ends: T = 50.0 exactly (index 1) on an even level
    b["tlev"][6, 1] = 50.0
    b["tlev"][6, 3] = 50.0
    # water at and above WREFH2O(10), and exactly on interior grid points
    b["qh2o"][7, 3:] = 0.4
    b["qh2o"][8, 3:] = 0.7
    b["qh2o"][9, 3:] = 1.0e-3
    # day threshold: exactly the REAL*4 1.0e-5 (day) and just below (night)
    b["acosz"][10] = float(np.float32(1.0e-5))
    b["acosz"][11] = np.nextafter(float(np.float32(1.0e-5)), 0)
    return b
