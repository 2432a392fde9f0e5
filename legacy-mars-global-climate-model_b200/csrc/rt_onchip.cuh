// Two-stream solves of kept systems with every per-system array on chip.
//
// The one-thread-per-system solves of rt_fp64_sys.cuh keep a system's
// per-layer values (the pass-A optics and the 2NL DSOLVER rows, 7NL + 1
// doubles: 1.4 KB at L = 24) in local memory; with tens of warps per SM that
// working set is larger than L2 and round-trips DRAM.  Here the same values
// live in a per-thread slice of the CTA's shared memory laid out
// [value][thread] (consecutive threads on consecutive 8-byte words: no bank
// conflicts), optionally extended by the SM's tensor memory (rt_tmem.cuh).
// The arithmetic is the one of rt_fp64_sys.cuh statement for statement, so
// results are bit-identical to it.
//
// Value slots of one system with NL layers (1-based layer l, row r):
//   IR       W(l) = WBARI           slot l-1
//            DT(l) = DTAUI           slot NL + l-1
//            TK(l) = TAUCUM(2l+1)-TAUCUM(2l), l < NL   slot 2NL + l-1
//   visible  W0(l)                   slot l-1
//            DTL(l) scaled DTAU      slot NL + l-1
//            TAU(l), l = 1..NL+1     slot 2NL + l-1
//            TCM(l) = TAUCUM(2l+1)   slot 3NL+1 + l-1
//   rows     AS(r), DS(r), r = 1..2NL, after the optics slots
// (code/gfluxi.f90:69-194, code/gfluxv.f90:76-280, code/dsolver.f90:54-103,
//  code/dtridgl.f90:25-38).
#pragma once
#include "rt_fp64_sys.cuh"
#include "rt_tmem.cuh"

namespace mgcm {
namespace onchip {

using namespace fp64;

// Slots a system needs: optics + rows.
__host__ __device__ constexpr int ir_slots(int nl) { return 3 * nl + 4 * nl; }
__host__ __device__ constexpr int vis_slots(int nl) { return 4 * nl + 1 + 4 * nl; }

// A thread's slice of shared memory: value v at base[v * T + t].
template <int T>
struct SmemSlots {
    double *base;
    int t;
    __device__ __forceinline__ double get(int v) const { return base[v * T + t]; }
    __device__ __forceinline__ void put(int v, double x) const { base[v * T + t] = x; }
};

// Tensor memory first, shared memory beyond: value v < vt at two TMEM
// columns of the thread's lane (taddr + 2v), the rest at sbase[(v - vt) * T
// + t].  Every get/put is executed by all 32 threads of the warp with the
// same v (the solves' loops are warp-uniform when the warp's systems share
// one layer count).
template <int T>
struct HybridSlots {
    double *sbase;
    int t;
    uint32_t taddr;
    int vt;
    __device__ __forceinline__ double get(int v) const {
        return v < vt ? tmem_get(taddr + 2u * (uint32_t)v) : sbase[(v - vt) * T + t];
    }
    __device__ __forceinline__ void put(int v, double x) const {
        if (v < vt) tmem_put(taddr + 2u * (uint32_t)v, x);
        else sbase[(v - vt) * T + t] = x;
    }
};

// ---------------------------------------------------------------- infrared
template <class S>
__device__ void solve_ir_oc(const SegDev &sg, int c, int nw, int ng, const ColSmem &s, const double *__restrict__ ki,
                            const S &st, double *fmp, double *fmm, double *sc0, size_t rs) {
    const int L = sg.L, NL = L + 1, LEV = 2 * L + 3;
    const int oW = 0, oDT = NL, oTK = 2 * NL, oAS = 3 * NL, oDS = 5 * NL;   // AS(r) at oAS + r-1
    const double *tb = ki + (size_t)(nw - 1) * D_NT * D_NP * D_NH * D_NGK + (ng - 1);
    auto dtauk = [&](int k) -> double {
        const double ta = s.taer_i[k * D_NI + nw - 1], tcl = s.tcld_i[k * D_NI + nw - 1];
        if (ng < D_NG) return taugas_at(s, k, tb) + ta + tcl;
        return ta + tcl;
    };
    // pass A (code/optci.f90:143-236)
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
        st.put(oW + l - 1, wb);
        st.put(oDT + l - 1, dt);
        if (l < NL) st.put(oTK + l - 1, tcA - tc);
        tc = tcB;
    }
    const double *plev = sg.plev + (size_t)c * LEV;
    const double rsf = sg.albi[c];
    const double dt1 = st.get(oDT);
    const double tautop = dt1 * plev[2 - 1] / (plev[4 - 1] - plev[2 - 1]);
    const double btop = (1.0 - mgcm_rt_exp(-tautop / UBARI)) * s.pltop_i[nw - 1];
    const double bsurf = s.bsurf_i[nw - 1];
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
    // pass C: rows bottom-up, eliminated as generated
    double pw0 = st.get(oW + NL - 2), pdt = st.get(oDT + NL - 2);   // NL >= 2
    Lay hi = coef(NL, st.get(oW + NL - 1), st.get(oDT + NL - 1));
    double as, ds;
    bottom_row_v(hi, bsurf, rsf, as, ds);
    st.put(oAS + 2 * NL - 1, as);
    st.put(oDS + 2 * NL - 1, ds);
    for (int n = NL - 1; n >= 1; --n) {
        const double w0 = pw0, dt = pdt;
        if (n > 1) {
            pw0 = st.get(oW + n - 2);
            pdt = st.get(oDT + n - 2);
        }
        const Lay lo = coef(n, w0, dt);
        double ao, dd;
        rows_of_pair(lo, hi, as, ds, ao, dd);
        st.put(oAS + 2 * n, ao);      // row 2n+1
        st.put(oDS + 2 * n, dd);
        st.put(oAS + 2 * n - 1, as);  // row 2n
        st.put(oDS + 2 * n - 1, ds);
        hi = lo;
    }
    {
        double a1, d1;
        top_row_v(hi, btop, as, ds, a1, d1);
        st.put(oAS, a1);
        st.put(oDS, d1);
    }
    // pass D: back-substitution, unmixing, midpoint fluxes
    double xprev = 0.0;
    double nas1 = st.get(oAS), nds1 = st.get(oDS), nas2 = st.get(oAS + 1), nds2 = st.get(oDS + 1);
    double nw0 = st.get(oW), ndt = st.get(oDT);
    double ndtk = 1 < NL ? st.get(oTK) : ndt;
    for (int n = 1; n <= NL; ++n) {
        const double as1 = nas1, ds1 = nds1, as2 = nas2, ds2 = nds2;
        const double dtk = ndtk, w0n = nw0, dtn = ndt;
        if (n < NL) {
            nas1 = st.get(oAS + 2 * n);
            nds1 = st.get(oDS + 2 * n);
            nas2 = st.get(oAS + 2 * n + 1);
            nds2 = st.get(oDS + 2 * n + 1);
            nw0 = st.get(oW + n);
            ndt = st.get(oDT + n);
            ndtk = n + 1 < NL ? st.get(oTK + n) : ndt;
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

// ---------------------------------------------------------------- visible
// F32: gas opacities from the FP32 table of Cmk*k (MIXED); the rest FP64.
template <class S, bool F32>
__device__ void solve_vis_oc(const SegDev &sg, int c, int nw, int ng, const ColSmem &s, const RtConst &K,
                             const double *__restrict__ kv, const float *__restrict__ kvf, const S &st,
                             double *fmp, double *fmm, double *sc0, double *sc1, double *sc2, size_t rs) {
    const int L = sg.L, NL = L + 1;
    const int oW = 0, oDL = NL, oTAU = 2 * NL, oTCM = 3 * NL + 1, oAS = 4 * NL + 1, oDS = 6 * NL + 1;
    const double *tb = kv + (size_t)(nw - 1) * D_NT * D_NP * D_NH * D_NGK + (ng - 1);
    const float *tbf = F32 ? kvf + (size_t)(nw - 1) * D_NT * D_NP * D_NH * D_NGK + (ng - 1) : nullptr;
    auto dtauk = [&](int k) -> double {
        if (ng < D_NG) {
            const double tg = F32 ? (double)taugas_f(s, k, tbf) : taugas_at(s, k, tb);
            return tg + s.trayaer[k * D_NV + nw - 1];
        }
        return s.trayaer[k * D_NV + nw - 1];
    };
    // pass A (code/optcv.f90:128-274, code/gfluxv.f90:76-103)
    const double tc2 = 0.0 + dtauk(2);
    double tc = tc2, tau = 0.0, fprev = 0.0, tcE1 = 0.0;
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
            st.put(oTCM, tcE1 + (tcA - tc2) * f);
        } else if (l < NL) {
            st.put(oTCM + l - 1, tau + (tcA - tc) * fprev);
        }
        st.put(oW + l - 1, wb * (1.0 - cb * cb) / f);
        const double dtl = dt * f;
        st.put(oDL + l - 1, dtl);
        st.put(oTAU + l - 1, tau);
        tau = tau + dtl;
        fprev = f;
        tc = tcB;
    }
    st.put(oTAU + NL, tau);
    const double detau = tau;
    // pass C (code/gfluxv.f90:108-165)
    const double u0 = sg.acosz[c], rsf = sg.als[c], f0pi = sg.sol[nw - 1];
    const double rcp_u0 = 1.0 / u0, rcp_u02 = 1.0 / (u0 * u0);
    const double s3 = (double)sqrtf(3.0f), s3h = (double)(sqrtf(3.0f) * 0.5f);
    const double bsurf = rsf * u0 * sg.sol[nw - 1] * mgcm_rt_exp(-dmin(detau / u0, MAXEXP));
    const double btop = 0.0;
    // LAMDA, GAMA, AM, AP of a layer from W0, the scaled COSBAR (staged per
    // layer and band) and U0; pass C and pass D both evaluate them
    struct Co { double lam, gama, am, ap; };
    const double *cbs = s.cbs_v + nw - 1;   // layer l at cbs[l * D_NV]
    auto co4 = [&](double w0, double cb) {
        Co r;
        const double g1 = s3h * (2.0 - w0 * (1.0 + cb));
        const double g2 = (s3 * w0 * 0.5) * (1.0 - cb);
        const double g3 = 0.5 * (1.0 - s3 * cb * u0);
        r.lam = sqrt(g1 * g1 - g2 * g2);
        r.gama = (g1 - r.lam) / g2;
        const double g4 = 1.0 - g3;
        double denom = r.lam * r.lam - rcp_u02;
        if (denom == 0.0) denom = R4(1.E-10);
        r.am = f0pi * w0 * (g4 * (g1 + rcp_u0) + g2 * g3) / denom;
        r.ap = f0pi * w0 * (g3 * (g1 - rcp_u0) + g2 * g4) / denom;
        return r;
    };
    auto coef = [&](const Co &q, double dtl, double et_top, double et_bot) {
        Lay y;
        y.gama = q.gama;
        y.cpm1 = q.ap * et_top;
        y.cmm1 = q.am * et_top;
        y.cp = q.ap * et_bot;
        y.cm = q.am * et_bot;
        const double ep = mgcm_rt_exp(dmin(TAUMAX, q.lam * dtl));
        const double em = 1.0 / ep;
        y.e1 = ep + y.gama * em;
        y.e2 = ep - y.gama * em;
        y.e3 = y.gama * ep + em;
        y.e4 = y.gama * ep - em;
        return y;
    };
    double et_bot = mgcm_rt_exp(-dmin(st.get(oTAU + NL) / u0, MAXEXP));
    double et_top = mgcm_rt_exp(-dmin(st.get(oTAU + NL - 1) / u0, MAXEXP));
    const int nm = NL >= 2 ? NL - 2 : 0;
    double pw0 = st.get(oW + nm), pcb = cbs[(NL - 1) * D_NV], pdt = st.get(oDL + nm), pa3 = st.get(oTAU + nm);
    Lay hi = coef(co4(st.get(oW + NL - 1), cbs[NL * D_NV]), st.get(oDL + NL - 1), et_top, et_bot);
    double as, ds;
    bottom_row_v(hi, bsurf, rsf, as, ds);
    st.put(oAS + 2 * NL - 1, as);
    st.put(oDS + 2 * NL - 1, ds);
    for (int n = NL - 1; n >= 1; --n) {
        const double w0 = pw0, cb = pcb, dtl = pdt, a3n = pa3;
        if (n > 1) {
            pw0 = st.get(oW + n - 2);
            pcb = cbs[(n - 1) * D_NV];
            pdt = st.get(oDL + n - 2);
            pa3 = st.get(oTAU + n - 2);
        }
        et_bot = et_top;
        et_top = mgcm_rt_exp(-dmin(a3n / u0, MAXEXP));
        const Lay lo = coef(co4(w0, cb), dtl, et_top, et_bot);
        double ao, dd;
        rows_of_pair(lo, hi, as, ds, ao, dd);
        st.put(oAS + 2 * n, ao);
        st.put(oDS + 2 * n, dd);
        st.put(oAS + 2 * n - 1, as);
        st.put(oDS + 2 * n - 1, ds);
        hi = lo;
    }
    {
        double a1, d1;
        top_row_v(hi, btop, as, ds, a1, d1);
        st.put(oAS, a1);
        st.put(oDS, d1);
    }
    // pass D (code/gfluxv.f90:170-280)
    double xprev = 0.0;
    double nas1 = st.get(oAS), nds1 = st.get(oDS), nas2 = st.get(oAS + 1), nds2 = st.get(oDS + 1);
    double nw0 = st.get(oW), na3 = st.get(oTAU), na4 = st.get(oTCM);
    double ncb = cbs[1 * D_NV];
    const double tbot = st.get(oTAU + NL);
    for (int n = 1; n <= NL; ++n) {
        const double as1 = nas1, ds1 = nds1, as2 = nas2, ds2 = nds2;
        const double w0n = nw0, cbn = ncb, a3n = na3, a4n = na4;
        if (n < NL) {
            nas1 = st.get(oAS + 2 * n);
            nds1 = st.get(oDS + 2 * n);
            nas2 = st.get(oAS + 2 * n + 1);
            nds2 = st.get(oDS + 2 * n + 1);
            nw0 = st.get(oW + n);
            ncb = cbs[(n + 1) * D_NV];
            na3 = st.get(oTAU + n);
            na4 = n + 1 < NL ? st.get(oTCM + n) : 0.0;
        }
        const Co q = co4(w0n, cbn);
        const double lam = q.lam, gama = q.gama, am = q.am, ap = q.ap;
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
            const double ep = mgcm_rt_exp(dmin(TAUMAX, lam * (tbot - a3n)));
            const double em = 1.0 / ep;
            const double taumid = dmin(tbot, TAUMAX);
            const double et = mgcm_rt_exp(-dmin(taumid / u0, MAXEXP));
            const double cpmid = ap * et, cmmid = am * et;
            fmp[(size_t)(n - 1) * rs] = xk1 * ep + gama * xk2 * em + cpmid;
            const double m = xk1 * ep * gama + xk2 * em + cmmid;
            *sc2 = m;
            fmm[(size_t)(n - 1) * rs] = m + u0 * f0pi * et;
        }
    }
}

}  // namespace onchip
}  // namespace mgcm
