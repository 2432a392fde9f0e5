// Aerosol optics on the device: the per-level dust and water-ice optical
// properties that COMP3 prepares for OPTCV/OPTCI, from tracer mixing ratios
// (code/comp3.f:592-630):
//   active dust  OPT_DST  code/opt_dst.f:55-161
//   prescribed   INI_OPTDST band constants (code/ini_optdst.f:29-51,
//                code/setrad.f90:132-155) with TAUREF given (FILLTAUCUM)
//   water ice    OPT_CLD  code/opt_cld.f:55-188
// Per layer: a lognormal size distribution from the mass and number mixing
// ratios, bin weights from DERF differences over the 20 radiative-transfer
// bins, band sums of the REAL*4 Mie tables for the layer's two levels, and
// TAUREF.  Built with --fmad=false; powers, logs, exps and DERF come from
// include/mgcm_rt_math.h, so the results equal the CPU oracle's bit for bit.
//
// One warp per column.  A lane per layer applies the routines' thresholds
// and computes the size parameters of the layers that pass them; a lane per
// level writes every other level (prescribed dust, or the defaults, and
// levels 1-3 and L_LEVELS+1 always); then each layer with aerosol is
// computed across the warp: 21 lanes evaluate the DERF bin edges at once and
// 12 lanes form the band sums (the per-layer chain of 21 DERFs was the cost
// of a thread-per-layer form).  Every level is written exactly once.
#include "rt_aerosol.cuh"
#include "../../include/mgcm_rt_math.h"

namespace mgcm {

namespace {

__device__ __forceinline__ double r4(double x) { return (double)(float)x; }

// Size parameters of one layer's lognormal distribution (OPT_DST / OPT_CLD):
// whether the layer passes the routine's thresholds, the core-ratio row of
// the ice tables, 1/Rs and the cross-section factor Ao.
struct LayerMie {
    double rs_inv, ao;
    int irap;
};

template <bool CLD>
__device__ bool layer_mie(const AeroConst &K, double ma, double mcor, double nb, LayerMie &m) {
    const double PIc = 3.1415926535897932;
    const double athird = (double)(1.0f / 3.0f);
    const double dpden_dt = r4(2.5E+3), dpden_ice = r4(917.);
    bool do_it;
    int irap = AERO_NRATIO;
    double Mo = 0.0, No = 0.0, dens = 0.0;
    if (!CLD) {
        do_it = ma > r4(1.e-8) && nb > 1.0;
        Mo = ma;
        No = nb + 1.0;
        dens = dpden_dt;
    } else {
        do_it = ma + mcor > r4(1.e-7) && nb > 1.0;
        if (do_it) {
            float mtc = (float)(mcor / dpden_dt / (ma / dpden_ice + mcor / dpden_dt));
            mtc = (float)mgcm_rt_pow((double)mtc, athird);
            for (int i = 1; i <= AERO_NRATIO; ++i) {
                const float cr = K.cor_ratio[i - 1];
                if (mtc < cr && i != 1) {
                    irap = i - 1;
                    break;
                } else if (mtc == cr) {
                    irap = i;
                    break;
                } else if (mtc < cr && i == 1) {
                    irap = 1;
                    break;
                }
            }
            Mo = ma + mcor;
            No = nb;
            dens = ma / Mo * dpden_ice + mcor / Mo * dpden_dt;
        }
    }
    if (!do_it) return false;
    const double dev = CLD ? r4(0.3087) : r4(0.63676);
    const double cst = 0.75 / (PIc * dens);
    double Rs = mgcm_rt_pow(Mo / No * cst, athird) * mgcm_rt_exp(-0.5 * (dev * dev));
    m.ao = No * PIc * (Rs * Rs);
    Rs = Rs * mgcm_rt_exp(1.5 * (dev * dev));
    Rs = fmin(fmax(Rs, r4(1.e-7)), CLD ? r4(100.e-6) : r4(50.e-6));
    m.rs_inv = 1.0 / Rs;
    m.irap = irap;
    return true;
}

// The optical properties of one layer that passed the thresholds, spread
// over the warp: lanes 0..20 evaluate the 21 DERF bin edges, lanes 0..6 /
// 7..11 form the visible / IR band sums over the 20 bins in the routine's
// order, for both of the layer's levels (k0 = 2l+2, k0+1; their sums are
// the same numbers), then QEXTREF and TAUREF per level.
template <bool CLD>
__device__ void layer_optics(int lane, const AeroConst &K, const double *__restrict__ mie, int L, int l,
                             const double *pl, const LayerMie &m, double *tauref, double *qextref,
                             double *qxv, double *qsv, double *gv, double *qxi, double *qsi, double *gi) {
    const unsigned full = 0xffffffffu;
    const int lev1 = 2 * L + 4;
    const double GRAVc = 3.72;
    const double dev = CLD ? r4(0.3087) : r4(0.63676);
    const double dev2 = 1.0 / ((double)sqrtf(2.0f) * dev);
    double e = 0.0;
    if (lane <= AERO_NBIN) e = mgcm_rt_erf(mgcm_rt_ln(K.radb[lane] * m.rs_inv) * dev2);
    const double ehi = __shfl_down_sync(full, e, 1);
    const double surf = 0.5 * (ehi - e);   // bin `lane` (lanes 0..19)
    // mie layout: dust [3][bin][7] vis, [3][bin][5] IR; ice [3][ratio][bin][7], [3][ratio][bin][5]
    const bool vis = lane < AERO_NV, ir = lane >= AERO_NV && lane < AERO_NV + AERO_NI;
    const int iw = vis ? lane : lane - AERO_NV, nb = vis ? AERO_NV : AERO_NI;
    const double *tab;
    size_t sq;
    if (vis) {
        tab = CLD ? mie + AERO_DST_SIZE + (size_t)(m.irap - 1) * AERO_NBIN * AERO_NV : mie;
        sq = CLD ? (size_t)AERO_NRATIO * AERO_NBIN * AERO_NV : (size_t)AERO_NBIN * AERO_NV;
    } else {
        tab = CLD ? mie + AERO_DST_SIZE + 3 * AERO_NRATIO * AERO_NBIN * AERO_NV +
                        (size_t)(m.irap - 1) * AERO_NBIN * AERO_NI
                  : mie + 3 * AERO_NBIN * AERO_NV;
        sq = CLD ? (size_t)AERO_NRATIO * AERO_NBIN * AERO_NI : (size_t)AERO_NBIN * AERO_NI;
    }
    double x = 0.0, sc = 0.0, g = 0.0;
    for (int i = 0; i < AERO_NBIN; ++i) {
        const double sf = __shfl_sync(full, surf, i);
        if (vis || ir) {
            x = x + sf * __ldg(tab + i * nb + iw);
            sc = sc + sf * __ldg(tab + sq + i * nb + iw);
            g = g + sf * __ldg(tab + 2 * sq + i * nb + iw);
        }
    }
    const int k0 = 2 * l + 2;
    if (vis || ir) {
        const double scl = fmin(sc, r4(0.99999) * x);
        double *X = vis ? qxv : qxi, *S = vis ? qsv : qsi, *G = vis ? gv : gi;
        for (int k = k0; k <= k0 + 1; ++k) {
            X[iw * lev1 + k - 1] = x;
            S[iw * lev1 + k - 1] = scl;
            G[iw * lev1 + k - 1] = g;
        }
    }
    const double q6 = __shfl_sync(full, x, 5);   // QXV of L_NREFV = 6
    if (lane < 2) {
        const int k = k0 + lane;
        qextref[k - 1] = q6;
        const double mass = 100.0 * (pl[k - 1] - pl[k - 2]) / GRAVc;
        tauref[k - 1] = m.ao * qextref[k - 1] * mass;
    }
}

// Prescribed dust on level k (1-based): band constants, TAUREF as given.
__device__ void prescribed_level(const AeroConst &K, int lev1, int k, const double *tin, double *tauref,
                                 double *qextref, double *qxv, double *qsv, double *gv, double *qxi,
                                 double *qsi, double *gi) {
    qextref[k - 1] = K.qextv[5];
    tauref[k - 1] = k == lev1 ? 0.0 : tin[k - 1];
    for (int i = 0; i < AERO_NV; ++i) {
        qxv[i * lev1 + k - 1] = K.qextv[i];
        qsv[i * lev1 + k - 1] = K.qscatv[i];
        gv[i * lev1 + k - 1] = K.gv[i];
    }
    for (int i = 0; i < AERO_NI; ++i) {
        qxi[i * lev1 + k - 1] = K.qexti[i];
        qsi[i * lev1 + k - 1] = K.qscati[i];
        gi[i * lev1 + k - 1] = K.gi[i];
    }
}

__device__ void default_level(int lev1, int k, double *tauref, double *qextref, double *qxv, double *qsv,
                              double *gv, double *qxi, double *qsi, double *gi) {
    qextref[k - 1] = 1.0;
    tauref[k - 1] = 0.0;
    for (int i = 0; i < AERO_NV; ++i) {
        qxv[i * lev1 + k - 1] = 1.0;
        qsv[i * lev1 + k - 1] = 1.0 * r4(0.99);
        gv[i * lev1 + k - 1] = 0.0;
    }
    for (int i = 0; i < AERO_NI; ++i) {
        qxi[i * lev1 + k - 1] = 1.0;
        qsi[i * lev1 + k - 1] = 1.0 * r4(0.99);
        gi[i * lev1 + k - 1] = 0.0;
    }
}

}  // namespace

constexpr int AERO_MAXL = 99;   // MGCM_RT_MAX_LAYERS

__global__ void __launch_bounds__(32 * AERO_WARPS, 8)   // 64 registers
rt_aerosol(const AeroSeg a, const AeroConst K, const double *__restrict__ mie) {
    __shared__ LayerMie lm[AERO_WARPS][2][AERO_MAXL];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int L = a.L, lev = 2 * L + 3, lev1 = lev + 1;
    for (long long cc = (long long)blockIdx.x * AERO_WARPS + wid; cc < a.ncol;
         cc += (long long)gridDim.x * AERO_WARPS) {
        const size_t c = (size_t)cc;
        const double *pl = a.plev + c * lev;
        // dust arrays (absent for prescribed dust read as band constants)
        double *tr = nullptr, *qr = nullptr, *xv = nullptr, *sv = nullptr, *gv = nullptr;
        double *xi = nullptr, *si = nullptr, *gi = nullptr;
        if (a.tauref) {
            tr = a.tauref + c * lev1;
            qr = a.qextrefdst + c * lev1;
            xv = a.qxvdst + c * AERO_NV * lev1;
            sv = a.qsvdst + c * AERO_NV * lev1;
            gv = a.gvdst + c * AERO_NV * lev1;
            xi = a.qxidst + c * AERO_NI * lev1;
            si = a.qsidst + c * AERO_NI * lev1;
            gi = a.gidst + c * AERO_NI * lev1;
        }
        double *tc = nullptr, *qc = nullptr, *cxv = nullptr, *csv = nullptr, *cgv = nullptr;
        double *cxi = nullptr, *csi = nullptr, *cgi = nullptr;
        if (a.cloudon) {
            tc = a.taurefcld + c * lev1;
            qc = a.qextrefcld + c * lev1;
            cxv = a.qxvcld + c * AERO_NV * lev1;
            csv = a.qsvcld + c * AERO_NV * lev1;
            cgv = a.gvcld + c * AERO_NV * lev1;
            cxi = a.qxicld + c * AERO_NI * lev1;
            csi = a.qsicld + c * AERO_NI * lev1;
            cgi = a.gicld + c * AERO_NI * lev1;
        }
        // the layers that pass OPT_DST's / OPT_CLD's thresholds, a lane per layer
        unsigned dmask[4] = {0u, 0u, 0u, 0u}, cmask[4] = {0u, 0u, 0u, 0u};
        for (int base = 0; base < L; base += 32) {
            const int l = base + lane + 1;
            bool d_on = false, c_on = false;
            if (l <= L) {
                LayerMie m;
                if (a.active_dust && layer_mie<false>(K, a.dust_mass[c * L + l - 1], 0.0,
                                                      a.dust_number[c * L + l - 1], m)) {
                    lm[wid][0][l - 1] = m;
                    d_on = true;
                }
                if (a.cloudon && layer_mie<true>(K, a.ice_mass[c * L + l - 1], a.ice_core[c * L + l - 1],
                                                 a.ice_number[c * L + l - 1], m)) {
                    lm[wid][1][l - 1] = m;
                    c_on = true;
                }
            }
            dmask[base >> 5] = __ballot_sync(full, d_on);
            cmask[base >> 5] = __ballot_sync(full, c_on);
        }
        __syncwarp();
        // every other level: prescribed dust or the routines' defaults (levels
        // 1-3 and L_LEVELS+1 always), a lane per level
        const double *tin = a.tauref_in ? a.tauref_in + c * lev1 : nullptr;
        for (int k = lane + 1; k <= lev1; k += 32) {
            const int l = (k >= 4 && k <= lev) ? (k - 2) / 2 : 0;
            const bool d_act = l && ((dmask[(l - 1) >> 5] >> ((l - 1) & 31)) & 1u);
            const bool c_act = l && ((cmask[(l - 1) >> 5] >> ((l - 1) & 31)) & 1u);
            if (!a.active_dust) {
                if (tr) prescribed_level(K, lev1, k, tin, tr, qr, xv, sv, gv, xi, si, gi);
            } else if (!d_act) {
                default_level(lev1, k, tr, qr, xv, sv, gv, xi, si, gi);
            }
            if (a.cloudon && !c_act) default_level(lev1, k, tc, qc, cxv, csv, cgv, cxi, csi, cgi);
        }
        // the layers with aerosol, one at a time across the warp
        for (int w = 0; w < 4; ++w) {
            for (unsigned bits = dmask[w]; bits; bits &= bits - 1u) {
                const int l = 32 * w + __ffs(bits);
                layer_optics<false>(lane, K, mie, L, l, pl, lm[wid][0][l - 1], tr, qr, xv, sv, gv, xi, si, gi);
            }
            for (unsigned bits = cmask[w]; bits; bits &= bits - 1u) {
                const int l = 32 * w + __ffs(bits);
                layer_optics<true>(lane, K, mie, L, l, pl, lm[wid][1][l - 1], tc, qc, cxv, csv, cgv, cxi, csi,
                                   cgi);
            }
        }
        __syncwarp();   // lm is rewritten for the next column
    }
}

}  // namespace mgcm
