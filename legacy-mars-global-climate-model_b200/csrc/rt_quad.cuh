// Four-lane solvers: one (band, Gauss) system per quad of lanes, 8 systems
// per warp, every per-layer value held in registers.
//
// Lane q of a quad owns the contiguous layers q*Rr+1 .. (q+1)*Rr
// (Rr = ceil(NL/4) <= R).  The per-layer work -- the 8-corner gathers, the
// delta-Eddington scaling, the two-stream coefficients, exponentials and
// midpoint terms -- runs on all four lanes at once.  The parts that are
// serial in the reference pass through the lanes in order, the carry moving
// by quad shuffles:
//   A2  TAUCUM / TAU prefix sums, top-down      (code/optcv.f90:128-176,
//       code/getdetau.f90:29-56)
//   C2  DTRIDGL elimination, bottom-up          (code/dtridgl.f90:25-32)
//   D2  back-substitution and unmixing, top-down (code/dtridgl.f90:34-38,
//       code/dsolver.f90:91-103)
// Every formula keeps the operation order of the one-thread-per-system form
// in rt_fp64_sys.cuh, so results are bit-identical to it.  All lanes of a
// warp run the same steps; a quad without a live system repeats one and
// stores nothing, so the full-mask shuffles always meet.
#pragma once
#include "rt_fp64_sys.cuh"

namespace mgcm {
namespace fp64 {

// Broadcast within the quad from quad lane `src`.
__device__ __forceinline__ double qsh(double v, int src) {
    return __shfl_sync(0xffffffffu, v, (threadIdx.x & 28) + src);
}

// ---------------------------------------------------------------- visible
template <int R, bool F32>
__device__ __forceinline__ void quad_vis(const SegDev &sg, int c, int nw, int ng, const ColSmem &s,
                                         const RtConst &K, const double *__restrict__ kv,
                                         const float *__restrict__ kvf, bool live, double *fmp,
                                         double *fmm, double *scr, size_t rs = 1) {
    const int q = threadIdx.x & 3;
    const int L = sg.L, NL = L + 1;
    const int Rr = (NL + 3) / 4;
    const int lfirst = q * Rr + 1, llast = min((q + 1) * Rr, NL);
    const double *tb = kv + (size_t)(nw - 1) * D_NT * D_NP * D_NH * D_NGK + (ng - 1);
    const float *tbf = F32 ? kvf + (size_t)(nw - 1) * D_NT * D_NP * D_NH * D_NGK + (ng - 1) : nullptr;
    const bool gas = ng < D_NG;
    auto dtauk = [&](int k) -> double {
        const double tr = s.trayaer[k * D_NV + nw - 1];
        if (gas) {
            const double tg = F32 ? (double)taugas_f(s, k, tbf) : taugas_at(s, k, tb);
            return tg + tr;
        }
        return tr;
    };
    auto own = [&](int j) { return j < Rr && lfirst + j <= NL; };

    // A1: per-layer optics
    double da[R], db[R], fv[R], w0v[R], cbv[R], dtl[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        da[j] = db[j] = fv[j] = w0v[j] = cbv[j] = dtl[j] = 0.0;
        if (own(j)) {
            const int l = lfirst + j, k = 2 * l + 1;
            da[j] = dtauk(k);
            double dt;
            if (l <= L) {
                db[j] = dtauk(k + 1);
                dt = da[j] + db[j];
            } else {
                dt = da[j];
            }
            const double wb = s.wnum_v[l * D_NV + nw - 1] / dt;
            const double cb = s.cosb_v[l * D_NV + nw - 1];
            const double f = 1.0 - wb * (cb * cb);
            fv[j] = f;
            w0v[j] = wb * (1.0 - cb * cb) / f;
            cbv[j] = s.cbs_v[l * D_NV + nw - 1];
            dtl[j] = dt * f;
        }
    }
    // A2: prefix sums through the lanes
    const double tc2 = 0.0 + dtauk(2);
    double tc = tc2, tau = 0.0, fprev = 0.0, tcE1 = 0.0, tau_end = 0.0;
    double a3[R], a4[R];
#pragma unroll
    for (int j = 0; j < R; ++j) a3[j] = a4[j] = 0.0;
#pragma unroll 1
    for (int step = 0; step < 4; ++step) {
        if (q == step) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                if (!own(j)) continue;
                const int l = lfirst + j;
                const double tcA = tc + da[j];
                const double tcB = l <= L ? tcA + db[j] : tcA;
                if (l == 1) {
                    tau = 0.0 * fv[j];
                    tcE1 = tc2 * fv[j];
                    a4[j] = tcE1 + (tcA - tc2) * fv[j];
                } else if (l < NL) {
                    a4[j] = tau + (tcA - tc) * fprev;
                }
                a3[j] = tau;
                tau = tau + dtl[j];
                fprev = fv[j];
                tc = tcB;
            }
            tau_end = tau;
        }
        tc = qsh(tc, step);
        tau = qsh(tau, step);
        fprev = qsh(fprev, step);
    }
    const double detau = tau;   // TAU(NL+1)

    // C1: two-stream coefficients per layer
    const double u0 = sg.acosz[c], rsf = sg.als[c], f0pi = sg.sol[nw - 1];
    const double rcp_u0 = 1.0 / u0, rcp_u02 = 1.0 / (u0 * u0);
    const double s3 = (double)sqrtf(3.0f), s3h = (double)(sqrtf(3.0f) * 0.5f);
    double lam[R], gam[R], am[R], ap[R], ep[R], em[R], ett[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        lam[j] = gam[j] = am[j] = ap[j] = ett[j] = 0.0;
        ep[j] = em[j] = 1.0;
        if (!own(j)) continue;
        const double w0 = w0v[j], cb = cbv[j];
        const double g1 = s3h * (2.0 - w0 * (1.0 + cb));
        const double g2 = (s3 * w0 * 0.5) * (1.0 - cb);
        const double g3 = 0.5 * (1.0 - s3 * cb * u0);
        const double lm = sqrt(g1 * g1 - g2 * g2);
        gam[j] = (g1 - lm) / g2;
        const double g4 = 1.0 - g3;
        double denom = lm * lm - rcp_u02;
        if (denom == 0.0) denom = R4(1.E-10);
        am[j] = f0pi * w0 * (g4 * (g1 + rcp_u0) + g2 * g3) / denom;
        ap[j] = f0pi * w0 * (g3 * (g1 - rcp_u0) + g2 * g4) / denom;
        lam[j] = lm;
        ett[j] = mgcm_rt_exp(-dmin(a3[j] / u0, MAXEXP));
        ep[j] = mgcm_rt_exp(dmin(TAUMAX, lm * dtl[j]));
        em[j] = 1.0 / ep[j];
    }
    const double et_end = mgcm_rt_exp(-dmin(tau_end / u0, MAXEXP));   // below the lane's last layer
    auto lay = [&](int j, double et_bot) {
        Lay y;
        y.gama = gam[j];
        y.cpm1 = ap[j] * ett[j];
        y.cmm1 = am[j] * ett[j];
        y.cp = ap[j] * et_bot;
        y.cm = am[j] * et_bot;
        y.e1 = ep[j] + y.gama * em[j];
        y.e2 = ep[j] - y.gama * em[j];
        y.e3 = y.gama * ep[j] + em[j];
        y.e4 = y.gama * ep[j] - em[j];
        return y;
    };

    // C2: elimination bottom-up through the lanes.  Carry: AS/DS of row
    // 2l' and GAMA, CPM1, CMM1 of layer l' (the layer below the next one).
    double asl[R], dsl[R], ash[R], dsh[R];
    double as = 0.0, ds = 0.0, hg = 0.0, hcpm1 = 0.0, hcmm1 = 0.0;
#pragma unroll
    for (int j = 0; j < R; ++j) asl[j] = dsl[j] = ash[j] = dsh[j] = 0.0;
#pragma unroll 1
    for (int step = 3; step >= 0; --step) {
        if (q == step) {
#pragma unroll
            for (int j = R - 1; j >= 0; --j) {
                if (!own(j)) continue;
                const int l = lfirst + j;
                const double et_bot = (l == llast || j + 1 >= R) ? et_end : ett[j + 1 < R ? j + 1 : j];
                const Lay lo = lay(j, et_bot);
                if (l == NL) {
                    bottom_row_v(lo, rsf * u0 * f0pi * mgcm_rt_exp(-dmin(detau / u0, MAXEXP)), rsf, as, ds);
                    asl[j] = as;
                    dsl[j] = ds;
                } else {
                    Lay hi;
                    hi.gama = hg;
                    hi.cpm1 = hcpm1;
                    hi.cmm1 = hcmm1;
                    hi.e1 = hi.e2 = hi.e3 = hi.e4 = hi.cp = hi.cm = 0.0;
                    rows_of_pair(lo, hi, as, ds, ash[j], dsh[j]);
                    asl[j] = as;
                    dsl[j] = ds;
                }
                hg = lo.gama;
                hcpm1 = lo.cpm1;
                hcmm1 = lo.cmm1;
            }
        }
        as = qsh(as, step);
        ds = qsh(ds, step);
        hg = qsh(hg, step);
        hcpm1 = qsh(hcpm1, step);
        hcmm1 = qsh(hcmm1, step);
    }
    // row 1 (layer 1 is the carried "hi"; BTOP = 0)
    double as1, ds1;
    {
        Lay t;
        t.gama = hg;
        t.cmm1 = hcmm1;
        t.cpm1 = hcpm1;
        t.e1 = t.e2 = t.e3 = t.e4 = t.cp = t.cm = 0.0;
        top_row_v(t, 0.0, as, ds, as1, ds1);
    }

    // D1: midpoint transmissions per layer (reuse ep/em/ett)
#pragma unroll
    for (int j = 0; j < R; ++j) {
        if (!own(j)) continue;
        const int l = lfirst + j;
        if (l < NL) {
            const double tcE = l == 1 ? tcE1 : a3[j];
            ep[j] = mgcm_rt_exp(dmin(TAUMAX, lam[j] * (a4[j] - tcE)));
            em[j] = 1.0 / ep[j];
            ett[j] = mgcm_rt_exp(-dmin(a4[j] / u0, MAXEXP));
        } else {
            ep[j] = mgcm_rt_exp(dmin(TAUMAX, lam[j] * (detau - a3[j])));
            em[j] = 1.0 / ep[j];
            const double taumid = dmin(detau, TAUMAX);
            ett[j] = mgcm_rt_exp(-dmin(taumid / u0, MAXEXP));
        }
    }
    // D2: back-substitution top-down through the lanes, midpoint fluxes
    double xa = ds1;
#pragma unroll 1
    for (int step = 0; step < 4; ++step) {
        if (q == step) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                if (!own(j)) continue;
                const int l = lfirst + j;
                const double xb = dsl[j] - asl[j] * xa;
                double xk1, xk2;
                unmix(xa, xb, xk1, xk2);
                const double gama = gam[j];
                if (l == 1 && live) {
                    const double e1 = 1.0, e2 = 1.0;
                    const double fup = xk1 * e1 + gama * xk2 * e2 + ap[j];
                    double fdn = xk1 * e1 * gama + xk2 * e2 + am[j];
                    fdn = fdn + u0 * f0pi * mgcm_rt_exp(-dmin(0.0 / u0, MAXEXP));
                    scr[0] = fup;
                    scr[rs] = fdn;
                }
                const double cpmid = ap[j] * ett[j], cmmid = am[j] * ett[j];
                const double p = xk1 * ep[j] + gama * xk2 * em[j] + cpmid;
                const double m = xk1 * ep[j] * gama + xk2 * em[j] + cmmid;
                if (live) {
                    fmp[(size_t)(l - 1) * rs] = p;
                    fmm[(size_t)(l - 1) * rs] = m + u0 * f0pi * ett[j];
                    if (l == NL) scr[2 * rs] = m;
                }
                if (l < NL) xa = dsh[j] - ash[j] * xb;
            }
        }
        xa = qsh(xa, step);
    }
}

// ---------------------------------------------------------------- infrared
template <int R>
__device__ __forceinline__ void quad_ir(const SegDev &sg, int c, int nw, int ng, const ColSmem &s,
                                        const RtConst &K, const double *__restrict__ ki, bool live,
                                        double *fmp, double *fmm, double *scr, size_t rs = 1) {
    const int q = threadIdx.x & 3;
    const int L = sg.L, NL = L + 1, LEV = 2 * L + 3;
    const int Rr = (NL + 3) / 4;
    const int lfirst = q * Rr + 1, llast = min((q + 1) * Rr, NL);
    const double *tb = ki + (size_t)(nw - 1) * D_NT * D_NP * D_NH * D_NGK + (ng - 1);
    const bool gas = ng < D_NG;
    auto dtauk = [&](int k) -> double {
        const double ta = s.taer_i[k * D_NI + nw - 1], tcl = s.tcld_i[k * D_NI + nw - 1];
        if (gas) {
            const double tg = taugas_at(s, k, tb);
            return tg + ta + tcl;
        }
        return ta + tcl;
    };
    auto own = [&](int j) { return j < Rr && lfirst + j <= NL; };
    const double tiny = R4(1.0E-9);

    // A1: per-layer optical depths and single-scattering albedo
    double da[R], db[R], w0v[R], dtv[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        da[j] = db[j] = w0v[j] = dtv[j] = 0.0;
        if (!own(j)) continue;
        const int l = lfirst + j, k = 2 * l + 1;
        da[j] = dtauk(k);
        double dt;
        if (k + 1 <= LEV) {
            db[j] = dtauk(k + 1);
            dt = da[j] + db[j] + 1.0e-50;
        } else {
            dt = da[j] + 0.0 + 1.0e-50;
        }
        double wb;
        if (dt > tiny) {
            wb = s.wnum_i[l * D_NI + nw - 1] / dt;
        } else {
            wb = 0.0;
            dt = tiny;
        }
        w0v[j] = wb;
        dtv[j] = dt;
    }
    // A2: TAUCUMI prefix through the lanes (only the in-layer increments are kept)
    double tc = 0.0 + dtauk(2);
    double a4[R];
#pragma unroll
    for (int j = 0; j < R; ++j) a4[j] = 0.0;
#pragma unroll 1
    for (int step = 0; step < 4; ++step) {
        if (q == step) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                if (!own(j)) continue;
                const int l = lfirst + j, k = 2 * l + 1;
                const double tcA = tc + da[j];
                const double tcB = k + 1 <= LEV ? tcA + db[j] : tcA;
                if (l < NL) a4[j] = tcA - tc;
                tc = tcB;
            }
        }
        tc = qsh(tc, step);
    }

    // C1: coefficients and source terms per layer
    const double *plev = sg.plev + (size_t)c * LEV;
    const double rsf = sg.albi[c];
    const double tautop = qsh(dtv[0], 0) * plev[2 - 1] / (plev[4 - 1] - plev[2 - 1]);
    const double btop = (1.0 - mgcm_rt_exp(-tautop / UBARI)) * s.pltop_i[nw - 1];
    const double bsurf = s.bsurf_i[nw - 1];
    double lam[R], gam[R], b1v[R], term[R], ep[R], em[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        lam[j] = gam[j] = b1v[j] = term[j] = 0.0;
        ep[j] = em[j] = 1.0;
        if (!own(j)) continue;
        const int l = lfirst + j;
        const double w0 = w0v[j], cb = s.cosb_i[l * D_NI + nw - 1], dt = dtv[j];
        const double alpha = sqrt((1.0 - w0) / (1.0 - w0 * cb));
        lam[j] = alpha * (1.0 - w0 * cb) / UBARI;
        b1v[j] = s.pdif_i[l * D_NI + nw - 1] / dt;
        gam[j] = (1.0 - alpha) / (1.0 + alpha);
        term[j] = UBARI / (1.0 - w0 * cb);
        ep[j] = mgcm_rt_exp(dmin(lam[j] * dt, TAUMAX));
        em[j] = 1.0 / ep[j];
    }
    auto lay = [&](int j) {
        Lay y;
        const int l = lfirst + j;
        const double b0 = s.b0_i[l * D_NI + nw - 1], b1 = b1v[j], dt = dtv[j], tm = term[j];
        y.gama = gam[j];
        y.cp = b0 + b1 * dt + b1 * tm;
        y.cm = b0 + b1 * dt - b1 * tm;
        y.cpm1 = b0 + b1 * tm;
        y.cmm1 = b0 - b1 * tm;
        y.e1 = ep[j] + y.gama * em[j];
        y.e2 = ep[j] - y.gama * em[j];
        y.e3 = y.gama * ep[j] + em[j];
        y.e4 = y.gama * ep[j] - em[j];
        return y;
    };

    // C2: elimination bottom-up through the lanes
    double asl[R], dsl[R], ash[R], dsh[R];
    double as = 0.0, ds = 0.0, hg = 0.0, hcpm1 = 0.0, hcmm1 = 0.0;
#pragma unroll
    for (int j = 0; j < R; ++j) asl[j] = dsl[j] = ash[j] = dsh[j] = 0.0;
#pragma unroll 1
    for (int step = 3; step >= 0; --step) {
        if (q == step) {
#pragma unroll
            for (int j = R - 1; j >= 0; --j) {
                if (!own(j)) continue;
                const int l = lfirst + j;
                const Lay lo = lay(j);
                if (l == NL) {
                    bottom_row_v(lo, bsurf, rsf, as, ds);
                } else {
                    Lay hi;
                    hi.gama = hg;
                    hi.cpm1 = hcpm1;
                    hi.cmm1 = hcmm1;
                    hi.e1 = hi.e2 = hi.e3 = hi.e4 = hi.cp = hi.cm = 0.0;
                    rows_of_pair(lo, hi, as, ds, ash[j], dsh[j]);
                }
                asl[j] = as;
                dsl[j] = ds;
                hg = lo.gama;
                hcpm1 = lo.cpm1;
                hcmm1 = lo.cmm1;
            }
        }
        as = qsh(as, step);
        ds = qsh(ds, step);
        hg = qsh(hg, step);
        hcpm1 = qsh(hcpm1, step);
        hcmm1 = qsh(hcmm1, step);
    }
    double as1, ds1;
    {
        Lay t;
        t.gama = hg;
        t.cmm1 = hcmm1;
        t.cpm1 = hcpm1;
        t.e1 = t.e2 = t.e3 = t.e4 = t.cp = t.cm = 0.0;
        top_row_v(t, btop, as, ds, as1, ds1);
    }

    // D1: midpoint transmissions and source terms (reuse ep/em/lam/term)
#pragma unroll
    for (int j = 0; j < R; ++j) {
        if (!own(j)) continue;
        const int l = lfirst + j;
        const double dtk = l < NL ? a4[j] : dtv[j];
        ep[j] = mgcm_rt_exp(dmin(lam[j] * dtk, TAUMAX));
        em[j] = 1.0 / ep[j];
        const double b0 = s.b0_i[l * D_NI + nw - 1], b1 = b1v[j];
        lam[j] = b0 + b1 * dtk + b1 * term[j];   // CPMID
        a4[j] = b0 + b1 * dtk - b1 * term[j];    // CMMID
    }
    // D2: back-substitution top-down through the lanes, midpoint fluxes
    double xa = ds1;
#pragma unroll 1
    for (int step = 0; step < 4; ++step) {
        if (q == step) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                if (!own(j)) continue;
                const int l = lfirst + j;
                const double xb = dsl[j] - asl[j] * xa;
                double xk1, xk2;
                unmix(xa, xb, xk1, xk2);
                const double gama = gam[j];
                const double p = xk1 * ep[j] + gama * xk2 * em[j] + lam[j];
                const double m = xk1 * ep[j] * gama + xk2 * em[j] + a4[j];
                if (live) {
                    fmp[(size_t)(l - 1) * rs] = p * PI_D;
                    fmm[(size_t)(l - 1) * rs] = m * PI_D;
                    if (l == 1) {
                        const double b0 = s.b0_i[l * D_NI + nw - 1], b1 = b1v[j];
                        const double e1 = 1.0, e2 = 1.0;
                        const double cpm = b0 + b1 * term[j], cmm = b0 - b1 * term[j];
                        const double fup = xk1 * e1 + gama * xk2 * e2 + cpm;
                        const double fdn = xk1 * e1 * gama + xk2 * e2 + cmm;
                        scr[0] = (fup - fdn) * PI_D;
                    }
                }
                if (l < NL) xa = dsh[j] - ash[j] * xb;
            }
        }
        xa = qsh(xa, step);
    }
    (void)llast;
}

}  // namespace fp64
}  // namespace mgcm
