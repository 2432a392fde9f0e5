// Per-system work of the FP64 radiation path and the ordered per-column
// reduction, shared by the fused kernel and the three-kernel pipeline.
#pragma once
#include "rt_stage.cuh"

namespace mgcm {
namespace fp64 {

constexpr double MAXEXP = 35.0;
constexpr double TAUMAX = 35.0;
constexpr double UBARI = 0.5;
constexpr double PI_D = 3.1415926535897932;
constexpr double TLIMITS = 1.0e-3;
constexpr double TLIMITI = 5.0e-3;

// Resident CTAs per SM (128 threads) asked of the solve kernels.  Both ask
// for 7 (72 registers), so the grid the two solves of a part share -- 7 CTAs
// per SM, from the IR solve's occupancy -- is one wave of either kernel.
// Measured on the 64,800-column call: 11.68 -> 11.52 ms MIXED, 12.00 ->
// 11.83 ms FP64, against 8 (64 registers) for the IR solve and 6 (80) for
// the visible ones.
#ifndef MGCM_IR_SOLVE_MINB
#define MGCM_IR_SOLVE_MINB 7
#endif
#ifndef MGCM_VIS_SOLVE_MINB
#define MGCM_VIS_SOLVE_MINB 7   // the FP64 and the MIXED visible solve
#endif

struct Lay {   // per-layer two-stream coefficients
    double gama, e1, e2, e3, e4, cp, cm, cpm1, cmm1;
};

// Per-system arrays (1-based layer index).  Pass A fills a0..a4; the visible
// pass C writes the layer's two-stream coefficients over the pass-A slots it
// has consumed (plus c5) -- the IR passes C and D recompute theirs from the
// pass-A slots instead -- and both write the DSOLVER rows' AS/DS for the
// back-substitution.
struct SysLocal {
    double a0[D_MAXNL + 1], a1[D_MAXNL + 1], a2[D_MAXNL + 1], a3[D_MAXNL + 2], a4[D_MAXNL + 1];
    double c5[D_MAXNL + 1];
    double as[2 * D_MAXNL + 1], ds[2 * D_MAXNL + 1];
};

// One step of the DTRIDGL upward elimination for row i given row i+1's AS/DS.
__device__ __forceinline__ void elim(double af, double bf, double cf, double df, double as1,
                                     double ds1, double &as, double &ds) {
    const double x = 1.0 / (bf - cf * as1);
    as = af * x;
    ds = (df - cf * ds1) * x;
}

// Rows 2n+1 (odd) and 2n (even) of DSOLVER for layers lo = n, hi = n+1,
// eliminated in DTRIDGL's order: as/ds carry row 2n+2 in and row 2n out;
// row 2n+1 is returned in as_odd/ds_odd.
__device__ __forceinline__ void rows_of_pair(const Lay &lo, const Lay &hi, double &as, double &ds,
                                             double &as_odd, double &ds_odd) {
    {
        const double af = 2.0 * (1.0 - lo.gama * lo.gama);
        const double bf = (lo.e1 - lo.e3) * (1.0 + hi.gama);
        const double cf = (lo.e1 + lo.e3) * (hi.gama - 1.0);
        const double df = lo.e3 * (hi.cpm1 - lo.cp) + lo.e1 * (lo.cm - hi.cmm1);
        elim(af, bf, cf, df, as, ds, as, ds);
        as_odd = as;
        ds_odd = ds;
    }
    {
        const double af = (lo.e1 + lo.e3) * (hi.gama - 1.0);
        const double bf = (lo.e2 + lo.e4) * (hi.gama - 1.0);
        const double cf = 2.0 * (1.0 - hi.gama * hi.gama);
        const double df = (hi.gama - 1.0) * (hi.cpm1 - lo.cp) + (1.0 - hi.gama) * (lo.cm - hi.cmm1);
        elim(af, bf, cf, df, as, ds, as, ds);
    }
}

// The same with every row stored for the back-substitution.
__device__ __forceinline__ void elim_pair(const Lay &lo, const Lay &hi, int n, SysLocal &w,
                                          double &as, double &ds) {
    double ao, dd;
    rows_of_pair(lo, hi, as, ds, ao, dd);
    w.as[2 * n + 1] = ao;
    w.ds[2 * n + 1] = dd;
    w.as[2 * n] = as;
    w.ds[2 * n] = ds;
}

// Row 2NL (surface) of DSOLVER.
__device__ __forceinline__ void bottom_row_v(const Lay &b, double bsurf, double rsf, double &as,
                                             double &ds) {
    const double af = b.e1 - rsf * b.e3;
    const double bf = b.e2 - rsf * b.e4;
    const double df = bsurf - b.cp + rsf * b.cm;
    as = af / bf;
    ds = df / bf;
}

// Row 1 (top) of DSOLVER given row 2.
__device__ __forceinline__ void top_row_v(const Lay &t, double btop, double as2, double ds2, double &as1,
                                          double &ds1) {
    const double af = 0.0, bf = t.gama + 1.0, cf = t.gama - 1.0, df = btop - t.cmm1;
    elim(af, bf, cf, df, as2, ds2, as1, ds1);
}

__device__ __forceinline__ void bottom_row(const Lay &b, int nl, double bsurf, double rsf,
                                           SysLocal &w, double &as, double &ds) {
    bottom_row_v(b, bsurf, rsf, as, ds);
    w.as[2 * nl] = as;
    w.ds[2 * nl] = ds;
}

__device__ __forceinline__ void top_row(const Lay &t, double btop, SysLocal &w, double as2,
                                        double ds2) {
    top_row_v(t, btop, as2, ds2, w.as[1], w.ds[1]);
}

// XK(2n-1), XK(2n) -> XK1, XK2 with the underflow test of dsolver.f90:91-101.
// The test divides; when |XK2| >= 2e-30 |XA + 1e-20| (the usual case) the
// quotient is above the REAL*4 1E-30 whatever its rounding, so the division
// is skipped.  Zero, infinite and NaN operands fail that comparison and take
// the reference's division.
__device__ __forceinline__ void unmix(double xa, double xb, double &xk1, double &xk2) {
    xk1 = xa + xb;
    xk2 = xa - xb;
    const double d = xa + R4(1.e-20);
    if (xk2 != 0.0 && !(fabs(xk2) >= 2.0e-30 * fabs(d)) && fabs(xk2 / d) < R4(1.E-30)) xk2 = 0.0;
}

// Table strides of the k-table corners: MP+1 and MT+1 (elements).
constexpr int KT_DP = D_NH * D_NGK, KT_DT = D_NP * D_NH * D_NGK;

// 8-corner gather and interpolation (optcv.f90:279-301): returns TAUGAS.
// tb points at the band's table plus the Gauss point; the level's corner
// offset and NH2O step come staged (ColSmem::kofs, kdh).
// The level's record, four 16-byte loads.
struct KLv {
    double2 lk01, lk23, wu;
    int2 kd;
};
__device__ __forceinline__ KLv klev_load(const ColSmem &s, int k) {
    const double2 *q = reinterpret_cast<const double2 *>(s.klev + k);
    KLv r;
    r.lk01 = q[0];
    r.lk23 = q[1];
    r.wu = q[2];
    r.kd = *reinterpret_cast<const int2 *>(q + 3);
    return r;
}

__device__ __forceinline__ double taugas_at(const ColSmem &s, int k, const double *__restrict__ tb) {
    const KLv kl = klev_load(s, k);
    const double *p = tb + kl.kd.x;
    const int dh = kl.kd.y;
    const double wr = kl.wu.x;
    auto corner = [&](int off) {
        const double c0 = __ldg(p + off), c1 = __ldg(p + off + dh);
        return c0 + wr * (c1 - c0);
    };
    const double k1 = corner(0), k2 = corner(KT_DP);
    const double k3 = corner(KT_DT + KT_DP), k4 = corner(KT_DT);
    const double ans = kl.lk01.x * k1 + kl.lk01.y * k2 + kl.lk23.x * k3 + kl.lk23.y * k4;
    return kl.wu.y * ans;
}


// TAUGAS at level k from the FP32 table of Cmk*k (mixed precision).
__device__ __forceinline__ float taugas_f(const ColSmem &s, int k, const float *__restrict__ tb) {
    const KLv kl = klev_load(s, k);
    const float *p = tb + kl.kd.x;
    const int dh = kl.kd.y;
    const float wr = (float)kl.wu.x;
    auto corner = [&](int off) {
        const float c0 = __ldg(p + off), c1 = __ldg(p + off + dh);
        return c0 + wr * (c1 - c0);
    };
    const float k1 = corner(0), k2 = corner(KT_DP);
    const float k3 = corner(KT_DT + KT_DP), k4 = corner(KT_DT);
    const float ans = (float)kl.lk01.x * k1 + (float)kl.lk01.y * k2 +
                      (float)kl.lk23.x * k3 + (float)kl.lk23.y * k4;
    return (float)s.dpr[k] * ans;
}

// ---------------------------------------------------------------- visible
// MODE 0: whole system (fused kernel); 1: screen only (optics, TLIMIT
// decision, DETAU and CUMTAUV); 2: solve a system the screen kept.
// F32: opacities from the FP32 table of Cmk*k (mixed precision); everything
// after the per-level optical depth stays FP64.  The midpoint fluxes of layer
// n go to fmp[(n-1) rs] and fmm[(n-1) rs].
template <int MODE, bool F32 = false>
__device__ void solve_vis(const SegDev &sg, int c, int nw, int ng, int sidx, ColSmem &s,
                          const RtConst &K, const double *__restrict__ kv, SysLocal &w,
                          unsigned int &nsolved, double *fmp, double *fmm, double *sc0,
                          double *sc1, double *sc2, const float *__restrict__ kvf = nullptr,
                          size_t rs = 1) {
    const int L = sg.L, NL = L + 1;
    const double fz0 = K.fzerov[nw - 1];
    const bool band_skip = ng < D_NG && fz0 >= R4(0.99);
    const double *tb = kv + (size_t)(nw - 1) * D_NT * D_NP * D_NH * D_NGK + (ng - 1);
    const float *tbf = F32 ? kvf + (size_t)(nw - 1) * D_NT * D_NP * D_NH * D_NGK + (ng - 1) : nullptr;
    double taugsurf = 0.0;
    auto dtauk = [&](int k) -> double {
        if (ng < D_NG) {
            const double tg = F32 ? (double)taugas_f(s, k, tbf) : taugas_at(s, k, tb);
            taugsurf += tg;
            return tg + s.trayaer[k * D_NV + nw - 1];
        }
        return s.trayaer[k * D_NV + nw - 1];
    };
    // pass A: levels 2..LEV, TCIN prefix sums, delta-Eddington stream.
    // a0 = W0, a2 = scaled DTAU, a3 = TAU (1..NL+1), a4 = TAUCUM(2l+1); the
    // scaled COSBAR of a layer is staged in the column block (cbs_v)
    const double tc2 = 0.0 + dtauk(2);
    double tc = tc2, tau = 0.0, fprev = 0.0, tcE1 = 0.0, tcLev = 0.0;
    for (int l = 1; l <= NL; ++l) {
        const int k = 2 * l + 1;
        const double da = dtauk(k);
        const double tcA = tc + da;
        double dt, tcB;
        if (l <= L) {
            const double db = dtauk(k + 1);
            tcB = tcA + db;
            dt = da + db;
        } else {
            tcB = tcA;
            dt = da;
        }
        const double wb = s.wnum_v[l * D_NV + nw - 1] / dt;
        const double cb = s.cosb_v[l * D_NV + nw - 1];
        const double f = 1.0 - wb * (cb * cb);
        if (l == 1) {
            tau = 0.0 * f;
            tcE1 = tc2 * f;
            if (MODE != 1) w.a4[1] = tcE1 + (tcA - tc2) * f;
        } else if (l < NL) {
            if (MODE != 1) w.a4[l] = tau + (tcA - tc) * fprev;
        }
        if (MODE != 1) w.a0[l] = wb * (1.0 - cb * cb) / f;
        const double dtl = dt * f;
        if (MODE != 1) {
            w.a2[l] = dtl;
            w.a3[l] = tau;
        }
        tau = tau + dtl;
        fprev = f;
        tc = tcB;
        tcLev = tcB;
    }
    if (MODE != 1) w.a3[NL + 1] = tau;
    const double detau = tau;
    if (MODE != 2) {
        double *detau_o = sg.detau + (size_t)c * 119;
        sg.cumtauv[(size_t)c * 119 + (nw - 1) + 7 * (ng - 1)] = tcLev;
        if (band_skip) {
            s.skip[sidx] = 2;
            return;
        }
        detau_o[(nw - 1) + 7 * (ng - 1)] = detau;
        if (ng < D_NG && taugsurf < TLIMITS) {
            s.skip[sidx] = 1;
            return;
        }
        s.skip[sidx] = 0;
        ++nsolved;
        if (MODE == 1) return;
    }

    // pass C: coefficients bottom-up, rows eliminated as generated.
    const double u0 = sg.acosz[c], rsf = sg.als[c], f0pi = sg.sol[nw - 1];
    const double rcp_u0 = 1.0 / u0, rcp_u02 = 1.0 / (u0 * u0);
    const double s3 = (double)sqrtf(3.0f), s3h = (double)(sqrtf(3.0f) * 0.5f);
    const double bsurf = rsf * u0 * sg.sol[nw - 1] * mgcm_rt_exp(-dmin(detau / u0, MAXEXP));
    const double btop = 0.0;
    // LAMDA, GAMA, AM overwrite W0, a1 (unused by pass A), DTAU of the same layer; AP -> c5
    double *LAM = w.a0, *GAM = w.a1, *AM = w.a2, *AP = w.c5;
    auto coef = [&](int l, double w0, double cb, double dtl, double et_top, double et_bot) {
        Lay y;
        const double g1 = s3h * (2.0 - w0 * (1.0 + cb));
        const double g2 = (s3 * w0 * 0.5) * (1.0 - cb);
        const double g3 = 0.5 * (1.0 - s3 * cb * u0);
        const double lam = sqrt(g1 * g1 - g2 * g2);
        y.gama = (g1 - lam) / g2;
        const double g4 = 1.0 - g3;
        double denom = lam * lam - rcp_u02;
        if (denom == 0.0) denom = R4(1.E-10);
        const double am = f0pi * w0 * (g4 * (g1 + rcp_u0) + g2 * g3) / denom;
        const double ap = f0pi * w0 * (g3 * (g1 - rcp_u0) + g2 * g4) / denom;
        LAM[l] = lam;
        GAM[l] = y.gama;
        AM[l] = am;
        AP[l] = ap;
        y.cpm1 = ap * et_top;
        y.cmm1 = am * et_top;
        y.cp = ap * et_bot;
        y.cm = am * et_bot;
        const double ep = mgcm_rt_exp(dmin(TAUMAX, lam * dtl));
        const double em = 1.0 / ep;
        y.e1 = ep + y.gama * em;
        y.e2 = ep - y.gama * em;
        y.e3 = y.gama * ep + em;
        y.e4 = y.gama * ep - em;
        return y;
    };
    double et_bot = mgcm_rt_exp(-dmin(w.a3[NL + 1] / u0, MAXEXP));
    double et_top = mgcm_rt_exp(-dmin(w.a3[NL] / u0, MAXEXP));
    // layer NL-1's inputs are fetched one step ahead
    const double *cbs = s.cbs_v + nw - 1;   // layer l at cbs[l * D_NV]
    double pw0 = w.a0[NL - 1], pcb = cbs[(NL - 1) * D_NV], pdt = w.a2[NL - 1], pa3 = w.a3[NL - 1];
    Lay hi = coef(NL, w.a0[NL], cbs[NL * D_NV], w.a2[NL], et_top, et_bot);
    double as, ds;
    bottom_row(hi, NL, bsurf, rsf, w, as, ds);
    for (int n = NL - 1; n >= 1; --n) {
        const double w0 = pw0, cb = pcb, dtl = pdt, a3n = pa3;
        if (n > 1) {
            pw0 = w.a0[n - 1];
            pcb = cbs[(n - 1) * D_NV];
            pdt = w.a2[n - 1];
            pa3 = w.a3[n - 1];
        }
        et_bot = et_top;
        et_top = mgcm_rt_exp(-dmin(a3n / u0, MAXEXP));
        const Lay lo = coef(n, w0, cb, dtl, et_top, et_bot);
        elim_pair(lo, hi, n, w, as, ds);
        hi = lo;
    }
    top_row(hi, btop, w, as, ds);

    // pass D: back-substitution, unmixing, midpoint fluxes (layer n+1's
    // values fetched one step ahead).
    double xprev = 0.0;
    double nas1 = w.as[1], nds1 = w.ds[1], nas2 = w.as[2], nds2 = w.ds[2];
    double nlam = LAM[1], ngam = GAM[1], nam = AM[1], nap = AP[1], na3 = w.a3[1], na4 = w.a4[1];
    for (int n = 1; n <= NL; ++n) {
        const double as1 = nas1, ds1 = nds1, as2 = nas2, ds2 = nds2;
        const double lam = nlam, gama = ngam, am = nam, ap = nap, a3n = na3, a4n = na4;
        if (n < NL) {
            nas1 = w.as[2 * n + 1];
            nds1 = w.ds[2 * n + 1];
            nas2 = w.as[2 * n + 2];
            nds2 = w.ds[2 * n + 2];
            nlam = LAM[n + 1];
            ngam = GAM[n + 1];
            nam = AM[n + 1];
            nap = AP[n + 1];
            na3 = w.a3[n + 1];
            na4 = w.a4[n + 1];
        }
        const double xa = n == 1 ? ds1 : ds1 - as1 * xprev;
        const double xb = ds2 - as2 * xa;
        xprev = xb;
        double xk1, xk2;
        unmix(xa, xb, xk1, xk2);
        if (n == 1) {
            const double ep = 1.0, em = 1.0;
            const double fup = xk1 * ep + gama * xk2 * em + ap;
            double fdn = xk1 * ep * gama + xk2 * em + am;
            fdn = fdn + u0 * f0pi * mgcm_rt_exp(-dmin(0.0 / u0, MAXEXP));
            *sc0 = fup;
            *sc1 = fdn;
        }
        if (n < NL) {
            const double tcE = n == 1 ? tcE1 : a3n;
            const double ep = mgcm_rt_exp(dmin(TAUMAX, lam * (a4n - tcE)));
            const double em = 1.0 / ep;
            const double et = mgcm_rt_exp(-dmin(a4n / u0, MAXEXP));
            const double cpmid = ap * et, cmmid = am * et;
            fmp[(size_t)(n - 1) * rs] = xk1 * ep + gama * xk2 * em + cpmid;
            double m = xk1 * ep * gama + xk2 * em + cmmid;
            fmm[(size_t)(n - 1) * rs] = m + u0 * f0pi * et;
        } else {
            const double tb = w.a3[NL + 1];
            const double ep = mgcm_rt_exp(dmin(TAUMAX, lam * (tb - a3n)));
            const double em = 1.0 / ep;
            const double taumid = dmin(tb, TAUMAX);
            const double et = mgcm_rt_exp(-dmin(taumid / u0, MAXEXP));
            const double cpmid = ap * et, cmmid = am * et;
            fmp[(size_t)(n - 1) * rs] = xk1 * ep + gama * xk2 * em + cpmid;
            const double m = xk1 * ep * gama + xk2 * em + cmmid;
            *sc2 = m;
            fmm[(size_t)(n - 1) * rs] = m + u0 * f0pi * et;
        }
    }
}

// ---------------------------------------------------------------- infrared
#ifndef MGCM_IR_SCREEN_UNROLL
#define MGCM_IR_SCREEN_UNROLL 2
#endif
constexpr int IR_SCREEN_UNROLL = MGCM_IR_SCREEN_UNROLL;

// The midpoint fluxes of layer n go to fmp[(n-1) rs] and fmm[(n-1) rs].
template <int MODE>
__device__ void solve_ir(const SegDev &sg, int c, int nw, int ng, int sidx, ColSmem &s,
                         const RtConst &K, const double *__restrict__ ki, SysLocal &w,
                         unsigned int &nsolved, double *fmp, double *fmm, double *sc0, size_t rs = 1) {
    const int L = sg.L, NL = L + 1, LEV = 2 * L + 3;
    const double fz0 = K.fzeroi[nw - 1];
    if (ng < D_NG && fz0 >= R4(0.99)) {
        if (MODE != 2) s.skip[sidx] = 2;
        return;
    }
    const double *tb = ki + (size_t)(nw - 1) * D_NT * D_NP * D_NH * D_NGK + (ng - 1);
    double taugsurf = 0.0;
    auto dtauk = [&](int k) -> double {
        const double ta = s.taer_i[k * D_NI + nw - 1], tcl = s.tcld_i[k * D_NI + nw - 1];
        if (ng < D_NG) {
            const double tg = taugas_at(s, k, tb);
            taugsurf += tg;
            return tg + ta + tcl;
        }
        return ta + tcl;
    };
    if (MODE == 1) {
        // The screen needs TAUGSURF only: the gas optical depths of levels
        // 2..LEV summed in order (code/optci.f90:143-167).  The gathers of
        // IR_SCREEN_UNROLL levels are issued before they are summed, so a
        // warp has that many levels' table reads in flight.
        double taug = 0.0;
        if (ng < D_NG) {
            int k = 2;
            for (; k + IR_SCREEN_UNROLL - 1 <= LEV; k += IR_SCREEN_UNROLL) {
                double tg[IR_SCREEN_UNROLL];
#pragma unroll
                for (int u = 0; u < IR_SCREEN_UNROLL; ++u) tg[u] = taugas_at(s, k + u, tb);
#pragma unroll
                for (int u = 0; u < IR_SCREEN_UNROLL; ++u) taug += tg[u];
            }
            for (; k <= LEV; ++k) taug += taugas_at(s, k, tb);
            if (taug < TLIMITI) {
                s.skip[sidx] = 1;
                return;
            }
        }
        s.skip[sidx] = 0;
        ++nsolved;
        return;
    }
    // pass A. a0 = WBARI, a1 = COSBI, a2 = DTAUI, a4 = TAUCUMI(2l+1)-TAUCUMI(2l)
    const double tiny = R4(1.0E-9);
    double tc = 0.0 + dtauk(2);
    for (int l = 1; l <= NL; ++l) {
        const int k = 2 * l + 1;
        const double da = dtauk(k);
        const double tcA = tc + da;
        double dt, tcB;
        if (k + 1 <= LEV) {
            const double db = dtauk(k + 1);
            tcB = tcA + db;
            dt = da + db + 1.0e-50;
        } else {
            tcB = tcA;
            dt = da + 0.0 + 1.0e-50;
        }
        double wb;
        if (dt > tiny) {
            wb = s.wnum_i[l * D_NI + nw - 1] / dt;
        } else {
            wb = 0.0;
            dt = tiny;
        }
        if (MODE != 1) {
            w.a0[l] = wb;
            w.a2[l] = dt;
            if (l < NL) w.a4[l] = tcA - tc;
        }
        tc = tcB;
    }
    if (MODE != 2) {
        if (ng < D_NG && taugsurf < TLIMITI) {
            s.skip[sidx] = 1;
            return;
        }
        s.skip[sidx] = 0;
        ++nsolved;
        if (MODE == 1) return;
    }
    const double *plev = sg.plev + (size_t)c * LEV;
    const double rsf = sg.albi[c];
    const double tautop = w.a2[1] * plev[2 - 1] / (plev[4 - 1] - plev[2 - 1]);
    const double btop = (1.0 - mgcm_rt_exp(-tautop / UBARI)) * s.pltop_i[nw - 1];
    const double bsurf = s.bsurf_i[nw - 1];
    // LAMDA, GAMA, B1, TERM of layer l (code/gfluxi.f90:69-93).  Pass C
    // and pass D both evaluate them from the pass-A slots (WBARI, DTAUI),
    // which stay intact: recomputing costs less than a round trip of four
    // more per-layer arrays through local memory (measured on the c1 call:
    // 15.8 -> 15.4 ms).  The visible solve keeps its stored coefficients:
    // there the recomputation measured slower.
    auto lay4 = [&](int l, double w0, double dt, double &lam, double &gama, double &b1, double &term) {
        const double cb = s.cosb_i[l * D_NI + nw - 1];
        const double alpha = sqrt((1.0 - w0) / (1.0 - w0 * cb));
        lam = alpha * (1.0 - w0 * cb) / UBARI;
        b1 = s.pdif_i[l * D_NI + nw - 1] / dt;
        gama = (1.0 - alpha) / (1.0 + alpha);
        term = UBARI / (1.0 - w0 * cb);
    };
    auto coef = [&](int l, double w0, double dt) {
        Lay y;
        double lam, b1, term;
        lay4(l, w0, dt, lam, y.gama, b1, term);
        const double b0 = s.b0_i[l * D_NI + nw - 1];
        y.cp = b0 + b1 * dt + b1 * term;
        y.cm = b0 + b1 * dt - b1 * term;
        y.cpm1 = b0 + b1 * term;
        y.cmm1 = b0 - b1 * term;
        const double ep = mgcm_rt_exp(dmin(lam * dt, TAUMAX));
        const double em = 1.0 / ep;
        y.e1 = ep + y.gama * em;
        y.e2 = ep - y.gama * em;
        y.e3 = y.gama * ep + em;
        y.e4 = y.gama * ep - em;
        return y;
    };
    double pw0 = w.a0[NL - 1], pdt = w.a2[NL - 1];
    Lay hi = coef(NL, w.a0[NL], w.a2[NL]);
    double as, ds;
    bottom_row(hi, NL, bsurf, rsf, w, as, ds);
    for (int n = NL - 1; n >= 1; --n) {
        const double w0 = pw0, dt = pdt;
        if (n > 1) {
            pw0 = w.a0[n - 1];
            pdt = w.a2[n - 1];
        }
        const Lay lo = coef(n, w0, dt);
        elim_pair(lo, hi, n, w, as, ds);
        hi = lo;
    }
    top_row(hi, btop, w, as, ds);

    double xprev = 0.0;
    double nas1 = w.as[1], nds1 = w.ds[1], nas2 = w.as[2], nds2 = w.ds[2];
    double nw0 = w.a0[1], ndt = w.a2[1];
    double ndtk = 1 < NL ? w.a4[1] : w.a2[1];
    for (int n = 1; n <= NL; ++n) {
        const double as1 = nas1, ds1 = nds1, as2 = nas2, ds2 = nds2;
        const double dtk = ndtk, w0n = nw0, dtn = ndt;
        if (n < NL) {
            nas1 = w.as[2 * n + 1];
            nds1 = w.ds[2 * n + 1];
            nas2 = w.as[2 * n + 2];
            nds2 = w.ds[2 * n + 2];
            nw0 = w.a0[n + 1];
            ndt = w.a2[n + 1];
            ndtk = n + 1 < NL ? w.a4[n + 1] : w.a2[n + 1];
        }
        double lam, gama, b1, term;
        lay4(n, w0n, dtn, lam, gama, b1, term);
        const double xa = n == 1 ? ds1 : ds1 - as1 * xprev;
        const double xb = ds2 - as2 * xa;
        xprev = xb;
        double xk1, xk2;
        unmix(xa, xb, xk1, xk2);
        const double b0 = s.b0_i[n * D_NI + nw - 1];
        const double ep = mgcm_rt_exp(dmin(lam * dtk, TAUMAX));
        const double em = 1.0 / ep;
        const double cpmid = b0 + b1 * dtk + b1 * term;
        const double cmmid = b0 + b1 * dtk - b1 * term;
        const double p = xk1 * ep + gama * xk2 * em + cpmid;
        const double m = xk1 * ep * gama + xk2 * em + cmmid;
        fmp[(size_t)(n - 1) * rs] = p * PI_D;
        fmm[(size_t)(n - 1) * rs] = m * PI_D;
        if (n == 1) {
            const double ep1 = 1.0, em1 = 1.0;
            const double cpm = b0 + b1 * term, cmm = b0 - b1 * term;
            const double fup = xk1 * ep1 + gama * xk2 * em1 + cpm;
            const double fdn = xk1 * ep1 * gama + xk2 * em1 + cmm;
            *sc0 = (fup - fdn) * PI_D;
        }
    }
}

// Ordered sums over (band, Gauss) of one output (code/sfluxv.f90:60-164,
// code/sfluxi.f90:57-145).  q: 0 net, 1 up, 2 down (layer l), 3 top net, 4 DIFFV.
__device__ inline double reduce_family(const ColSmem &s, const RtConst &K, bool vis, int q, int l,
                                int NL) {
    const int nb = vis ? D_NV : D_NI, base = vis ? 0 : NSYS_V;
    const double *fz = vis ? K.fzerov : K.fzeroi;
    double acc = 0.0;
    for (int nw = 1; nw <= nb; ++nw) {
        double fzero = fz[nw - 1];
        const double dw = vis ? 1.0 : K.dwni[nw - 1];
        auto val = [&](int sidx) -> double {
            switch (q) {
                case 0: return s.fmp[(size_t)sidx * NL + l - 1] - s.fmm[(size_t)sidx * NL + l - 1];
                case 1: return s.fmp[(size_t)sidx * NL + l - 1];
                case 2: return s.fmm[(size_t)sidx * NL + l - 1];
                case 3: return vis ? s.sc0[sidx] - s.sc1[sidx] : s.sc0[sidx];
                default: return s.sc2[sidx];
            }
        };
        if (!(fzero >= R4(0.99))) {
            for (int ng = 1; ng <= D_NG - 1; ++ng) {
                const int sidx = base + (nw - 1) * D_NG + ng - 1;
                if (s.skip[sidx] == 1) {
                    fzero = fzero + (1.0 - fz[nw - 1]) * K.gweight[ng - 1];
                    continue;
                }
                if (vis) acc = acc + val(sidx) * K.gweight[ng - 1] * (1.0 - fz[nw - 1]);
                else acc = acc + val(sidx) * dw * K.gweight[ng - 1] * (1.0 - fz[nw - 1]);
            }
        }
        const int s17 = base + (nw - 1) * D_NG + D_NG - 1;
        if (vis) acc = acc + val(s17) * fzero;
        else acc = acc + val(s17) * dw * fzero;
    }
    return acc;
}


// Per-row multipliers of the compact layout for one family of a column: the
// kept systems in ascending order get m1,m2,m3 so that the reference's term
// is ((val*m1)*m2)*m3 -- visible (val*GWEIGHT)*(1-FZEROV) or val*FZERO for
// Gauss point 17; IR ((val*DWNI)*GWEIGHT)*(1-FZEROI) or (val*DWNI)*FZERO
// (code/sfluxv.f90:102-162, code/sfluxi.f90:95-143).  Unused factors are
// exactly 1.0, which leaves the product bit-identical.  Returns the rows.
__device__ inline int family_multipliers(const unsigned char *skip, const RtConst &K, bool vis,
                                  double *m1, double *m2, double *m3) {
    const int nb = vis ? D_NV : D_NI, base = vis ? 0 : NSYS_V;
    const double *fz = vis ? K.fzerov : K.fzeroi;
    int pos = 0;
    for (int nw = 1; nw <= nb; ++nw) {
        double fzero = fz[nw - 1];
        const double dw = vis ? 1.0 : K.dwni[nw - 1];
        if (!(fzero >= R4(0.99))) {
            for (int ng = 1; ng <= D_NG - 1; ++ng) {
                const int sidx = base + (nw - 1) * D_NG + ng - 1;
                if (skip[sidx] != 0) {
                    fzero = fzero + (1.0 - fz[nw - 1]) * K.gweight[ng - 1];
                    continue;
                }
                if (vis) {
                    m1[pos] = K.gweight[ng - 1];
                    m2[pos] = 1.0 - fz[nw - 1];
                    m3[pos] = 1.0;
                } else {
                    m1[pos] = dw;
                    m2[pos] = K.gweight[ng - 1];
                    m3[pos] = 1.0 - fz[nw - 1];
                }
                ++pos;
            }
        }
        if (vis) {
            m1[pos] = fzero;
            m2[pos] = 1.0;
        } else {
            m1[pos] = dw;
            m2[pos] = fzero;
        }
        m3[pos] = 1.0;
        ++pos;
    }
    return pos;
}

// Ordered sum of one output over the family's kept rows (q: 0 net, 1 up,
// 2 down at layer l; 3 top net; 4 DIFFV).
__device__ __forceinline__ double reduce_rows(const double *fl, const double *sc, int mnl, int rows,
                                              const double *m1, const double *m2,
                                              const double *m3, bool vis, int q, int l) {
    double acc = 0.0;
    const size_t stride = (size_t)2 * mnl;
    if (q < 3) {
        const double *p = fl + (l - 1);
        for (int r = 0; r < rows; ++r, p += stride) {
            const double v = q == 0 ? p[0] - p[mnl] : (q == 1 ? p[0] : p[mnl]);
            acc = acc + v * m1[r] * m2[r] * m3[r];
        }
    } else {
        for (int r = 0; r < rows; ++r) {
            const double v = q == 3 ? (vis ? sc[r * 4] - sc[r * 4 + 1] : sc[r * 4]) : sc[r * 4 + 2];
            acc = acc + v * m1[r] * m2[r] * m3[r];
        }
    }
    return acc;
}

// Ordered band/Gauss sums of one column, then SUNTOT, IRTOTAL and QRAD
// (code/comp3.f:677-681,735-747,765-771).  Called by all threads of a CTA.
template <class Red>
__device__ void reduce_and_heat(const SegDev &sg, int c, Red red, double *fmnet_v, double *fmnet_i,
                                double *misc, bool day) {
    const int L = sg.L, NL = L + 1, LEV = 2 * L + 3;
    const int t = threadIdx.x;
    // ordered reductions: visible 3*NL+2 items, IR 3*NL+1 items
    const int nv_items = 3 * NL + 2, ni_items = 3 * NL + 1;
    for (int it = t; it < nv_items + ni_items; it += blockDim.x) {
        const bool vis = it < nv_items;
        const int j = vis ? it : it - nv_items;
        int q, l = 1;
        if (j < 3 * NL) { q = j / NL; l = j % NL + 1; }
        else q = 3 + (j - 3 * NL);
        double v = 0.0;
        if (!vis || day) v = red(vis, q, l);
        const size_t o = (size_t)c * NL + l - 1;
        if (vis) {
            if (q == 0) { sg.fmnetv[o] = v; fmnet_v[l] = v; }
            else if (q == 1) sg.fluxupv[o] = v;
            else if (q == 2) {
                sg.fluxdnv[o] = v;
                if (l == NL) { sg.dnvflux[c] = v; sg.fluxsurf[c] = (1.0 - sg.als[c]) * v; }
            } else if (q == 3) { sg.nfluxtopv[c] = v; misc[0] = v; }
            else { sg.diffvt[c] = v; sg.dndiffv[c] = v; }
        } else {
            if (q == 0) { sg.fmneti[o] = v; fmnet_i[l] = v; }
            else if (q == 1) sg.fluxupi[o] = v;
            else if (q == 2) { sg.fluxdni[o] = v; if (l == NL) sg.dnirflux[c] = v; }
            else { sg.nfluxtopi[c] = v; misc[1] = v; }
        }
    }
    __syncthreads();
    // divergences and heating rates
    const double *plev = sg.plev + (size_t)c * LEV;
    for (int l = 1 + t; l <= NL; l += blockDim.x) {
        const double sun = day ? (l == 1 ? fmnet_v[1] - misc[0] : fmnet_v[l] - fmnet_v[l - 1]) : 0.0;
        const double irt = l == 1 ? fmnet_i[1] - misc[1] : fmnet_i[l] - fmnet_i[l - 1];
        const int k = 2 * l;
        const double ptrop = sg.ptrop, p = sg.pcol[c];
        const double ym = k == 2 ? ptrop * 100.0 / 3.72 : (plev[k + 1 - 1] - plev[k - 1 - 1]) * 100.0 / 3.72;
        const double om = pow(plev[k - 1] / plev[LEV - 1], 0.25684);
        const double pnlte = sg.sigma[k - 1] * (p - ptrop) + ptrop;
        const double sunlte = sun * 2.2e4 * pnlte / (1.0 + 2.2e4 * pnlte);
        const size_t o = (size_t)c * NL + l - 1;
        sg.suntot[o] = sun;
        sg.irtotal[o] = irt;
        sg.qrad[o] = (sunlte + irt) / (735.94 * ym * om);
    }
}

}  // namespace fp64
}  // namespace mgcm
