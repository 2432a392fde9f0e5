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
// One thread per (column, layer) owns levels 2l+2 and 2l+3; one thread per
// column owns levels 1-3 and L_LEVELS+1 (defaults).  Every level is written
// exactly once.
#include "rt_aerosol.cuh"
#include "../../include/mgcm_rt_math.h"

namespace mgcm {

namespace {

__device__ __forceinline__ double r4(double x) { return (double)(float)x; }

// OPT_DST / OPT_CLD for one layer's two levels (k0 = 2l+2, 1-based).
template <bool CLD>
__device__ void aero_layer(const AeroConst &K, const double *__restrict__ mie, int L, int l,
                           const double *pl, double ma, double mcor, double nb, double *tauref,
                           double *qextref, double *qxv, double *qsv, double *gv, double *qxi,
                           double *qsi, double *gi) {
    const int lev1 = 2 * L + 4;
    const double PIc = 3.1415926535897932, GRAVc = 3.72;
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
    const int k0 = 2 * l + 2;
    if (!do_it) {   // the routine's defaults
        for (int k = k0; k <= k0 + 1; ++k) {
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
        return;
    }
    const double dev = CLD ? r4(0.3087) : r4(0.63676);
    const double dev2 = 1.0 / ((double)sqrtf(2.0f) * dev);
    const double cst = 0.75 / (PIc * dens);
    double Rs = mgcm_rt_pow(Mo / No * cst, athird) * mgcm_rt_exp(-0.5 * (dev * dev));
    const double Ao = No * PIc * (Rs * Rs);
    Rs = Rs * mgcm_rt_exp(1.5 * (dev * dev));
    Rs = fmin(fmax(Rs, r4(1.e-7)), CLD ? r4(100.e-6) : r4(50.e-6));
    Rs = 1.0 / Rs;
    double surf[AERO_NBIN];
    double elo = mgcm_rt_erf(mgcm_rt_ln(K.radb[0] * Rs) * dev2);
    for (int i = 0; i < AERO_NBIN; ++i) {
        const double ehi = mgcm_rt_erf(mgcm_rt_ln(K.radb[i + 1] * Rs) * dev2);
        surf[i] = 0.5 * (ehi - elo);
        elo = ehi;
    }
    // mie layout: dust [3][bin][7] vis, [3][bin][5] IR; ice [3][ratio][bin][7], [3][ratio][bin][5]
    const double *tv = CLD ? mie + AERO_DST_SIZE + (size_t)(irap - 1) * AERO_NBIN * AERO_NV : mie;
    const double *ti = CLD ? mie + AERO_DST_SIZE + 3 * AERO_NRATIO * AERO_NBIN * AERO_NV +
                                 (size_t)(irap - 1) * AERO_NBIN * AERO_NI
                           : mie + 3 * AERO_NBIN * AERO_NV;
    const size_t sv = CLD ? (size_t)AERO_NRATIO * AERO_NBIN * AERO_NV : (size_t)AERO_NBIN * AERO_NV;
    const size_t si = CLD ? (size_t)AERO_NRATIO * AERO_NBIN * AERO_NI : (size_t)AERO_NBIN * AERO_NI;
    for (int k = k0; k <= k0 + 1; ++k) {
        for (int iw = 0; iw < AERO_NV; ++iw) {
            double x = 0.0, sc = 0.0, g = 0.0;
            for (int i = 0; i < AERO_NBIN; ++i) {
                x = x + surf[i] * __ldg(tv + i * AERO_NV + iw);
                sc = sc + surf[i] * __ldg(tv + sv + i * AERO_NV + iw);
                g = g + surf[i] * __ldg(tv + 2 * sv + i * AERO_NV + iw);
            }
            qxv[iw * lev1 + k - 1] = x;
            qsv[iw * lev1 + k - 1] = fmin(sc, r4(0.99999) * x);
            gv[iw * lev1 + k - 1] = g;
        }
        for (int iw = 0; iw < AERO_NI; ++iw) {
            double x = 0.0, sc = 0.0, g = 0.0;
            for (int i = 0; i < AERO_NBIN; ++i) {
                x = x + surf[i] * __ldg(ti + i * AERO_NI + iw);
                sc = sc + surf[i] * __ldg(ti + si + i * AERO_NI + iw);
                g = g + surf[i] * __ldg(ti + 2 * si + i * AERO_NI + iw);
            }
            qxi[iw * lev1 + k - 1] = x;
            qsi[iw * lev1 + k - 1] = fmin(sc, r4(0.99999) * x);
            gi[iw * lev1 + k - 1] = g;
        }
        qextref[k - 1] = qxv[5 * lev1 + k - 1];   // L_NREFV = 6
        const double mass = 100.0 * (pl[k - 1] - pl[k - 2]) / GRAVc;
        tauref[k - 1] = Ao * qextref[k - 1] * mass;
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

__global__ void __launch_bounds__(128)
rt_aerosol(const AeroSeg a, const AeroConst K, const double *__restrict__ mie) {
    const int L = a.L, lev = 2 * L + 3, lev1 = lev + 1;
    const long long items = (long long)a.ncol * (L + 1);
    for (long long it = blockIdx.x * (long long)blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(it / (L + 1)), l = (int)(it % (L + 1));   // l = 0: levels 1-3, LEV1
        const double *pl = a.plev + (size_t)c * lev;
        double *tr = a.tauref + (size_t)c * lev1, *qr = a.qextrefdst + (size_t)c * lev1;
        double *xv = a.qxvdst + (size_t)c * AERO_NV * lev1, *sv = a.qsvdst + (size_t)c * AERO_NV * lev1;
        double *gv = a.gvdst + (size_t)c * AERO_NV * lev1, *xi = a.qxidst + (size_t)c * AERO_NI * lev1;
        double *si = a.qsidst + (size_t)c * AERO_NI * lev1, *gi = a.gidst + (size_t)c * AERO_NI * lev1;
        if (l == 0) {
            for (int k : {1, 2, 3, lev1}) {
                if (a.active_dust) default_level(lev1, k, tr, qr, xv, sv, gv, xi, si, gi);
                else prescribed_level(K, lev1, k, a.tauref_in + (size_t)c * lev1, tr, qr, xv, sv, gv, xi, si, gi);
            }
        } else if (a.active_dust) {
            aero_layer<false>(K, mie, L, l, pl, a.dust_mass[(size_t)c * L + l - 1], 0.0,
                              a.dust_number[(size_t)c * L + l - 1], tr, qr, xv, sv, gv, xi, si, gi);
        } else {
            for (int k = 2 * l + 2; k <= 2 * l + 3; ++k)
                prescribed_level(K, lev1, k, a.tauref_in + (size_t)c * lev1, tr, qr, xv, sv, gv, xi, si, gi);
        }
        if (a.cloudon) {
            double *tc = a.taurefcld + (size_t)c * lev1, *qc = a.qextrefcld + (size_t)c * lev1;
            double *cxv = a.qxvcld + (size_t)c * AERO_NV * lev1, *csv = a.qsvcld + (size_t)c * AERO_NV * lev1;
            double *cgv = a.gvcld + (size_t)c * AERO_NV * lev1, *cxi = a.qxicld + (size_t)c * AERO_NI * lev1;
            double *csi = a.qsicld + (size_t)c * AERO_NI * lev1, *cgi = a.gicld + (size_t)c * AERO_NI * lev1;
            if (l == 0) {
                for (int k : {1, 2, 3, lev1}) default_level(lev1, k, tc, qc, cxv, csv, cgv, cxi, csi, cgi);
            } else {
                aero_layer<true>(K, mie, L, l, pl, a.ice_mass[(size_t)c * L + l - 1],
                                 a.ice_core[(size_t)c * L + l - 1], a.ice_number[(size_t)c * L + l - 1], tc,
                                 qc, cxv, csv, cgv, cxi, csi, cgi);
            }
        }
    }
}

}  // namespace mgcm
