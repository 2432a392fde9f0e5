/*
 * mgcm_rt_oracle.c -- CPU oracle (TEST INFRASTRUCTURE, never shipped in the
 * product library) for the Legacy Mars GCM column radiative transfer.
 *
 * A line-by-line FP64 restatement of the reference Fortran.  Every routine
 * cites the reference file:line it follows.  Rules kept from the reference
 * build (code/Makefile:7-10, gfortran -O3 without -fdefault-real-8):
 *   - unsuffixed literals such as 0.9999, 1.0E-9, SQRT(3.0) are REAL*4; they
 *     are rounded to float and then promoted (R4() below);
 *   - Fortran evaluates a*b*c as (a*b)*c and a+b+c as (a+b)+c;
 *   - no FMA contraction (x86-64 baseline has none; this file is compiled
 *     with -ffp-contract=off);
 *   - x**2 is x*x, x**4 is (x*x)*(x*x), x**5 is (x*x)*(x*(x*x)) (gfortran's
 *     addition-chain expansion of constant integer powers);
 *   - real-to-integer assignment truncates toward zero.
 *
 * Exponentials inside a column use the deterministic routine of
 * include/mgcm_rt_math.h (build with -DORC_LIBM_EXP for the host libm).
 */
#include "mgcm_rt_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

#define R4(x) ((double)(float)(x))

/* Table-gather hook for the operation-count build (oracle/orc_count.cpp);
 * nothing in the normal builds. */
#ifndef ORC_GATHERS
#define ORC_GATHERS(n) ((void)0)
#endif

/* Per-column exponentials use the shared deterministic exp so the oracle and
 * the FP64 device path agree bit-for-bit (see include/mgcm_rt_math.h for why
 * the reference IR solver needs this).  Built with -DORC_LIBM_EXP the oracle
 * calls the host libm exp instead, which measures the libm sensitivity of the
 * reference algorithm.  Table set-up (Planck integrals) always uses libm. */
#include "../include/mgcm_rt_math.h"
#ifdef ORC_LIBM_EXP
#define cexp_(x) exp(x)
#else
#define cexp_(x) mgcm_rt_exp(x)
#endif

/* constants_h (code/modules.f90:118-148) */
static const double PI = 3.1415926535897932;
static const double GRAV = 3.72;
static const double CPHEAT = 735.94;
static const double SCALEP = 100.0;
static const double KAPA = 0.25684;
static const double CMK = 3.51e22;
/* radinc_h / radcommon_h (code/modules.f90:221-239,335-365) */
static const double MAXEXP = 35.0;
static const double TAUMAX = 35.0; /* L_TAUMAX = 35 (integer) */
static const double UBARI = 0.5;
static const double TLIMITS = 1.0e-3;
static const double TLIMITI = 5.0e-3;
#define NREFV 6 /* L_NREFV, 1-based */

static const double GWEIGHT_TAB[ORC_NGAUSS] = {
    4.8083554740e-02, 1.0563099137e-01, 1.4901065679e-01, 1.7227479710e-01,
    1.7227479710e-01, 1.4901065679e-01, 1.0563099137e-01, 4.8083554740e-02,
    2.5307134073e-03, 5.5595258613e-03, 7.8426661469e-03, 9.0670945845e-03,
    9.0670945845e-03, 7.8426661469e-03, 5.5595258613e-03, 2.5307134073e-03, 0.0};

static const double WREFH2O_TAB[ORC_REFH2O] = {1.0e-7, 1.0e-6, 1.0e-5, 1.0e-4, 1.0e-3,
                                               1.0e-2, 1.0e-1, 2.0e-1, 3.0e-1, 4.0e-1};

size_t orc_tables_size(void) { return sizeof(orc_tables); }
size_t orc_aero_size(void) { return sizeof(orc_aero); }

/* ------------------------------------------------------------------ */
/* Set-up                                                               */
/* ------------------------------------------------------------------ */

static int read_record(FILE *f, double *dst, size_t n) {
    int32_t m1 = 0, m2 = 0;
    if (fread(&m1, 4, 1, f) != 1) return -1;
    if ((size_t)m1 != n * sizeof(double)) return -2;
    if (fread(dst, sizeof(double), n, f) != n) return -3;
    if (fread(&m2, 4, 1, f) != 1 || m2 != m1) return -4;
    return 0;
}

/* laginterp.f90:59-69: one record of k values, one record of FZERO. */
int orc_read_ktables(const char *vis_path, const char *ir_path, double *co2v8, double *fzerov,
                     double *co2i8, double *fzeroi) {
    const size_t nv = (size_t)ORC_NTREF * ORC_NPREF * ORC_REFH2O * ORC_NSPECTV * ORC_NGAUSS;
    const size_t ni = (size_t)ORC_NTREF * ORC_NPREF * ORC_REFH2O * ORC_NSPECTI * ORC_NGAUSS;
    FILE *f = fopen(vis_path, "rb");
    if (!f) return -10;
    int rc = read_record(f, co2v8, nv);
    if (!rc) rc = read_record(f, fzerov, ORC_NSPECTV);
    fclose(f);
    if (rc) return rc - 10;
    f = fopen(ir_path, "rb");
    if (!f) return -20;
    rc = read_record(f, co2i8, ni);
    if (!rc) rc = read_record(f, fzeroi, ORC_NSPECTI);
    fclose(f);
    if (rc) return rc - 20;
    return 0;
}

/* lagrange.f90:11-33 */
static double lagrange(double x, const double xi[4], const double yi[4]) {
    double fm1 = x - xi[0], fm2 = x - xi[1], fm3 = x - xi[2], fm4 = x - xi[3];
    return fm2 * fm3 * fm4 * yi[0] / ((xi[0] - xi[1]) * (xi[0] - xi[2]) * (xi[0] - xi[3])) +
           fm1 * fm3 * fm4 * yi[1] / ((xi[1] - xi[0]) * (xi[1] - xi[2]) * (xi[1] - xi[3])) +
           fm1 * fm2 * fm4 * yi[2] / ((xi[2] - xi[0]) * (xi[2] - xi[1]) * (xi[2] - xi[3])) +
           fm1 * fm2 * fm3 * yi[3] / ((xi[3] - xi[0]) * (xi[3] - xi[1]) * (xi[3] - xi[2]));
}

/* laginterp.f90:102-236 for one band family (nb bands). raw8 is CO2(nt,np11,nh,nw,ng)
 * already converted to log10; out is CO2(nt,np51,nh,nw,ng). */
static void lag_family(const double *raw8, double *out, int nb, const double *pref,
                       const double *pint) {
#define RAW(nt, np, nh, nw, ng) \
    raw8[(nt - 1) + ORC_NTREF * ((np - 1) + ORC_NPREF * ((nh - 1) + ORC_REFH2O * ((nw - 1) + nb * (ng - 1))))]
#define OUT(nt, np, nh, nw, ng) \
    out[(nt - 1) + ORC_NTREF * ((np - 1) + ORC_PINT * ((nh - 1) + ORC_REFH2O * ((nw - 1) + nb * (ng - 1))))]
    double xi[4], yi[4];
    for (int nt = 1; nt <= ORC_NTREF; nt++)
        for (int nh = 1; nh <= ORC_REFH2O; nh++)
            for (int nw = 1; nw <= nb; nw++)
                for (int ng = 1; ng <= ORC_NGAUSS; ng++) {
                    int n = 1;
                    for (int m = 1; m <= 5; m++) {
                        double x = pint[m - 1];
                        for (int q = 0; q < 4; q++) {
                            xi[q] = pref[n - 1 + q];
                            yi[q] = RAW(nt, n + q, nh, nw, ng);
                        }
                        OUT(nt, m, nh, nw, ng) = pow(10.0, lagrange(x, xi, yi));
                    }
                    for (n = 2; n <= ORC_NPREF - 2; n++)
                        for (int m = 1; m <= 5; m++) {
                            int i = (n - 1) * 5 + m;
                            double x = pint[i - 1];
                            for (int q = 0; q < 4; q++) {
                                xi[q] = pref[n - 2 + q];
                                yi[q] = RAW(nt, n - 1 + q, nh, nw, ng);
                            }
                            OUT(nt, i, nh, nw, ng) = pow(10.0, lagrange(x, xi, yi));
                        }
                    n = ORC_NPREF - 1;
                    for (int m = 1; m <= 5; m++) {
                        int i = (n - 1) * 5 + m;
                        double x = pint[i - 1];
                        for (int q = 0; q < 4; q++) {
                            xi[q] = pref[n - 3 + q];
                            yi[q] = RAW(nt, n - 2 + q, nh, nw, ng);
                        }
                        OUT(nt, i, nh, nw, ng) = pow(10.0, lagrange(x, xi, yi));
                    }
                    OUT(nt, ORC_PINT, nh, nw, ng) = pow(10.0, RAW(nt, ORC_NPREF, nh, nw, ng));
                }
#undef RAW
#undef OUT
}

void orc_build_tables(orc_tables *t, const double *co2v8_in, const double *fzerov,
                      const double *co2i8_in, const double *fzeroi) {
    memset(t, 0, sizeof(*t));
    /* setspv.f90:56-105 */
    static const double BWNV[8] = {2222.22, 3087.37, 4030.63, 5370.57,
                                   7651.11, 12500.00, 25000.00, 41666.67};
    const double SOLAR[7] = {R4(12.7), R4(24.2), R4(54.6), R4(145.9),
                             R4(354.9), R4(657.5), R4(106.3)};
    const double P0 = 9.423e+6;
    for (int m = 0; m < 7; m++) {
        t->wnov[m] = 0.5 * (BWNV[m + 1] + BWNV[m]);
        t->dwnv[m] = BWNV[m + 1] - BWNV[m];
        t->wavev[m] = 1.0e+4 / t->wnov[m];
    }
    for (int n = 0; n < 7; n++) t->solarf[n] = SOLAR[n];
    for (int n = 0; n < 7; n++) {
        double wl = t->wavev[n];
        double wl2 = wl * wl, wl4 = wl2 * wl2;
        t->tauray[n] = (R4(8.7) / GRAV) * (R4(1.527) * (1.0 + R4(0.013) / wl2) / wl4) * SCALEP / P0;
    }
    /* setspi.f90:45-105 */
    static const double BWNI[6] = {10.000, 166.667, 416.667, 833.333, 1250.000, 2222.222};
    static const double GX[12] = {-0.981560634246719, -0.904117256370475, -0.769902674194305,
                                  -0.587317954286617, -0.367831498998180, -0.125233408511469,
                                  0.125233408511469,  0.367831498998180,  0.587317954286617,
                                  0.769902674194305,  0.904117256370475,  0.981560634246719};
    static const double GW[12] = {0.047175336386512, 0.106939325995318, 0.160078328543346,
                                  0.203167426723066, 0.233492536538355, 0.249147045813403,
                                  0.249147045813403, 0.233492536538355, 0.203167426723066,
                                  0.160078328543346, 0.106939325995318, 0.047175336386512};
    const double c1 = 3.741832e-16, c2 = 1.438786e-2;
    for (int m = 0; m < 5; m++) {
        t->wnoi[m] = 0.5 * (BWNI[m + 1] + BWNI[m]);
        t->dwni[m] = BWNI[m + 1] - BWNI[m];
        t->wavei[m] = 1.0e+4 / t->wnoi[m];
    }
    for (int nw = 0; nw < 5; nw++) {
        double a = 1.0e-2 / BWNI[nw + 1];
        double b = 1.0e-2 / BWNI[nw];
        double bpa = (b + a) / 2.0;
        double bma = (b - a) / 2.0;
        for (int nt = 500; nt <= 9000; nt++) {
            double T = (double)nt / 1.0e+1;
            double ans = 0.0;
            for (int m = 0; m < 12; m++) {
                double y = bma * GX[m] + bpa;
                double y2 = y * y, y5 = y2 * (y * y2);
                ans = ans + GW[m] * c1 / (y5 * (exp(c2 / (y * T)) - 1.0));
            }
            t->planckir[(nt - 500) * 5 + nw] = ans * bma / (PI * t->dwni[nw]);
        }
    }
    /* setrad.f90:73-154 */
    static const double qev1[7] = {1.834, 2.296, 2.672, 2.829, 2.698, 2.452, 2.261};
    static const double qsv1[7] = {1.695, 2.031, 2.583, 2.744, 2.626, 2.225, 1.525};
    static const double gv1[7] = {0.551, 0.640, 0.661, 0.678, 0.690, 0.743, 0.868};
    static const double qei1[5] = {0.008, 0.262, 0.491, 1.017, 0.444};
    static const double qsi1[5] = {0.001, 0.037, 0.122, 0.351, 0.336};
    static const double gi1[5] = {0.004, 0.030, 0.095, 0.214, 0.316};
    const double pg[11] = {R4(1.0e-6), R4(1.0e-5), R4(1.0e-4), R4(1.0e-3), R4(1.0e-2), R4(1.0e-1),
                           R4(1.0),    R4(1.0e+1), R4(1.0e+2), R4(1.0e+3), R4(1.0e+4)};
    for (int n = 0; n < 11; n++) t->pgasref[n] = pg[n];
    for (int n = 0; n < 7; n++) t->tgasref[n] = 50.0 * (n + 1);
    for (int n = 0; n < 7; n++) {
        t->qextv[n] = qev1[n];
        t->qscatv[n] = qsv1[n];
        if (t->qscatv[n] >= t->qextv[n]) t->qscatv[n] = R4(0.99999) * t->qextv[n];
        t->gv[n] = gv1[n];
    }
    for (int n = 0; n < 5; n++) {
        t->qexti[n] = qei1[n];
        t->qscati[n] = qsi1[n];
        if (t->qscati[n] >= t->qexti[n]) t->qscati[n] = R4(0.99999) * t->qexti[n];
        t->gi[n] = gi1[n];
    }
    /* laginterp.f90:191-236 */
    double pref[ORC_NPREF];
    for (int n = 0; n < ORC_NPREF; n++) pref[n] = log10(t->pgasref[n]);
    for (int n = 0; n < ORC_PINT; n++) t->pfgasref[n] = -6.0 + 0.2 * n;
    {
        /* the pin() literals are decimal D0 constants: -6.0D0, -5.8D0, ... 4.0D0 */
        static const char *pin_txt[ORC_PINT] = {
            "-6.0", "-5.8", "-5.6", "-5.4", "-5.2", "-5.0", "-4.8", "-4.6", "-4.4", "-4.2", "-4.0",
            "-3.8", "-3.6", "-3.4", "-3.2", "-3.0", "-2.8", "-2.6", "-2.4", "-2.2", "-2.0", "-1.8",
            "-1.6", "-1.4", "-1.2", "-1.0", "-0.8", "-0.6", "-0.4", "-0.2", "0.0",  "0.2",  "0.4",
            "0.6",  "0.8",  "1.0",  "1.2",  "1.4",  "1.6",  "1.8",  "2.0",  "2.2",  "2.4",  "2.6",
            "2.8",  "3.0",  "3.2",  "3.4",  "3.6",  "3.8",  "4.0"};
        for (int n = 0; n < ORC_PINT; n++) t->pfgasref[n] = strtod(pin_txt[n], NULL);
    }
    const size_t nv = (size_t)ORC_NTREF * ORC_NPREF * ORC_REFH2O * ORC_NSPECTV * ORC_NGAUSS;
    const size_t ni = (size_t)ORC_NTREF * ORC_NPREF * ORC_REFH2O * ORC_NSPECTI * ORC_NGAUSS;
    double *v8 = (double *)malloc(nv * sizeof(double));
    double *i8 = (double *)malloc(ni * sizeof(double));
    /* laginterp.f90:74-98: log10, floor at -200 */
    for (size_t q = 0; q < nv; q++) v8[q] = co2v8_in[q] > 1.0e-200 ? log10(co2v8_in[q]) : -200.0;
    for (size_t q = 0; q < ni; q++) i8[q] = co2i8_in[q] > 1.0e-200 ? log10(co2i8_in[q]) : -200.0;
    lag_family(i8, t->co2i, ORC_NSPECTI, pref, t->pfgasref);
    lag_family(v8, t->co2v, ORC_NSPECTV, pref, t->pfgasref);
    free(v8);
    free(i8);
    for (int n = 0; n < 7; n++) t->fzerov[n] = fzerov[n];
    for (int n = 0; n < 5; n++) t->fzeroi[n] = fzeroi[n];
    for (int n = 0; n < ORC_NGAUSS; n++) t->gweight[n] = GWEIGHT_TAB[n];
    for (int n = 0; n < ORC_REFH2O; n++) t->wrefh2o[n] = WREFH2O_TAB[n];
}

int orc_tables_load(orc_tables *t, const char *vis_path, const char *ir_path) {
    const size_t nv = (size_t)ORC_NTREF * ORC_NPREF * ORC_REFH2O * ORC_NSPECTV * ORC_NGAUSS;
    const size_t ni = (size_t)ORC_NTREF * ORC_NPREF * ORC_REFH2O * ORC_NSPECTI * ORC_NGAUSS;
    double *v8 = (double *)malloc(nv * sizeof(double));
    double *i8 = (double *)malloc(ni * sizeof(double));
    double fv[7], fi[5];
    int rc = orc_read_ktables(vis_path, ir_path, v8, fv, i8, fi);
    if (!rc) orc_build_tables(t, v8, fv, i8, fi);
    free(v8);
    free(i8);
    return rc;
}

/* ------------------------------------------------------------------ */
/* tpindex.f90:72-134                                                   */
/* ------------------------------------------------------------------ */
void orc_tpindex(const orc_tables *t, double pw, double tw, double qh2o, double lcoef[4],
                 int *mt_out, int *mp_out, int *nh2o_out, double *wratio_out) {
    const double *tref = t->tgasref, *pref = t->pfgasref, *wref = t->wrefh2o;
    int mt, mp, nh2o = 0;
    double wratio = 0.0;
    if (tw <= tref[0]) {
        mt = 1;
    } else {
        mt = ORC_NTREF - 1;
        for (int n = 1; n <= ORC_NTREF - 1; n++)
            if (tw > tref[n - 1] && tw <= tref[n]) {
                mt = n;
                break;
            }
    }
    double u = (tw - tref[mt - 1]) / (tref[mt] - tref[mt - 1]);
    /* bins from the host libm LOG10 (as the reference build); the weight
     * from the shared deterministic log10 (the IR solver amplifies its last
     * bit by ~1e9, see include/mgcm_rt_math.h) */
    double pwl = log10(pw);
    mp = ORC_PINT - 1;
    for (int n = 2; n <= ORC_PINT - 1; n++)
        if (pwl <= pref[n - 1]) {
            mp = n - 1;
            break;
        }
#ifndef ORC_LIBM_EXP
    pwl = mgcm_rt_log10(pw);
#endif
    double tt = (pwl - pref[mp - 1]) / (pref[mp] - pref[mp - 1]);
    lcoef[0] = (1.0 - tt) * (1.0 - u);
    lcoef[1] = tt * (1.0 - u);
    lcoef[2] = tt * u;
    lcoef[3] = (1.0 - tt) * u;
    if (qh2o <= wref[0]) {
        nh2o = 1;
        wratio = 0.0;
    } else if (qh2o >= wref[ORC_REFH2O - 1]) {
        nh2o = ORC_REFH2O;
        wratio = 0.0;
    } else {
        for (int n = 2; n <= ORC_REFH2O; n++)
            if (qh2o >= wref[n - 2] && qh2o < wref[n - 1]) {
                nh2o = n - 1;
                wratio = (qh2o - wref[n - 2]) / (wref[n - 1] - wref[n - 2]);
                break;
            }
        /* a NaN qh2o falls through all tests; the Fortran leaves NH2O/WRATIO
         * undefined.  Inputs are validated before this point. */
    }
    *mt_out = mt;
    *mp_out = mp;
    *nh2o_out = nh2o;
    *wratio_out = wratio;
}

/* ------------------------------------------------------------------ */
/* Per-column work space                                                 */
/* ------------------------------------------------------------------ */
#define MAXLEV (2 * ORC_MAXL + 3)
#define MAXLAY (ORC_MAXL + 1)

typedef struct {
    /* optics */
    double dtauk[(MAXLEV + 1) * ORC_NSPECTV * ORC_NGAUSS];
    double dtau[MAXLAY * ORC_NSPECTV * ORC_NGAUSS];
    double wbar[MAXLAY * ORC_NSPECTV * ORC_NGAUSS];
    double cosb[MAXLAY * ORC_NSPECTV * ORC_NGAUSS];
    double taucum[MAXLEV * ORC_NSPECTV * ORC_NGAUSS];
    double taugsurf[ORC_NSPECTV * (ORC_NGAUSS - 1)];
    double tray[(MAXLEV + 1) * ORC_NSPECTV], taeros[(MAXLEV + 1) * ORC_NSPECTV];
    double tcloud[(MAXLEV + 1) * ORC_NSPECTV];
    double taureflk[(MAXLEV + 1) * ORC_NSPECTV], taucldk[(MAXLEV + 1) * ORC_NSPECTV];
    double tauref_l[MAXLEV + 1], taurefcld_l[MAXLEV + 1];
    double dpr[MAXLEV + 1], u[MAXLEV + 1], wratio[MAXLEV + 1], lk[(MAXLEV + 1) * 4];
    int mt[MAXLEV + 1], mp[MAXLEV + 1], nh2o[MAXLEV + 1];
    /* two-stream per call */
    double w0[MAXLAY + 1], cosbar[MAXLAY + 1], dtaul[MAXLAY + 1], tau[MAXLAY + 2];
    double tcum[MAXLEV + 1];
    double g1[MAXLAY + 1], g2[MAXLAY + 1], g3[MAXLAY + 1], lamda[MAXLAY + 1], gama[MAXLAY + 1];
    double cp[MAXLAY + 1], cm[MAXLAY + 1], cpm1[MAXLAY + 1], cmm1[MAXLAY + 1];
    double e1[MAXLAY + 1], e2[MAXLAY + 1], e3[MAXLAY + 1], e4[MAXLAY + 1];
    double b0[MAXLAY + 1], b1[MAXLAY + 1], alpha[MAXLAY + 1];
    double xk1[MAXLAY + 1], xk2[MAXLAY + 1];
    double af[2 * MAXLAY + 2], bf[2 * MAXLAY + 2], cf[2 * MAXLAY + 2], df[2 * MAXLAY + 2];
    double xk[2 * MAXLAY + 2], as[2 * MAXLAY + 2], ds[2 * MAXLAY + 2];
    double fmidp[MAXLAY + 1], fmidm[MAXLAY + 1];
    /* accumulated per column */
    double fmnet[MAXLAY + 1], fup[MAXLAY + 1], fdn[MAXLAY + 1];
} work_t;

/* Fortran-order accessors with 1-based indices; n1 = leading dimension. */
#define A3(arr, n1, nb, i, nw, ng) (arr)[((i)-1) + (n1) * (((nw)-1) + (nb) * ((ng)-1))]
#define A2(arr, n1, i, nw) (arr)[((i)-1) + (n1) * ((nw)-1)]

/* Column input view (1-based accessors for per-column arrays). */
typedef struct {
    int L, lev, nlay;
    const double *plev, *tlev, *pmid, *tmid, *qh2o;
    const double *tauref, *qextrefdst, *taurefcld, *qextrefcld;
    const double *qxvdst, *qsvdst, *gvdst, *qxidst, *qsidst, *gidst;
    const double *qxvcld, *qsvcld, *gvcld, *qxicld, *qsicld, *gicld;
} colview;

static double zero_lev[MAXLEV + 2];
static double one_lev[MAXLEV + 2];
static double zero_band[(MAXLEV + 2) * ORC_NSPECTV];

#define LV(p, k) (p)[(k)-1]
#define BND(p, lev1, k, nw) (p)[((k)-1) + (lev1) * ((nw)-1)]

/* ------------------------------------------------------------------ */
/* optcv.f90:1-284 (column c, visible)                                  */
/* ------------------------------------------------------------------ */
static void optcv(const orc_tables *t, const colview *c, work_t *w) {
    const int LEV = c->lev, NLAY = c->nlay, NB = ORC_NSPECTV, NG = ORC_NGAUSS, LEV1 = LEV + 1;
    for (int ng = 1; ng <= NG - 1; ng++)
        for (int nw = 1; nw <= NB; nw++) w->taugsurf[(nw - 1) + NB * (ng - 1)] = 0.0;
    for (int k = 2; k <= LEV; k++) {
        w->dpr[k] = LV(c->plev, k) - LV(c->plev, k - 1);
        w->u[k] = CMK * w->dpr[k];
        double lc[4];
        orc_tpindex(t, LV(c->pmid, k), LV(c->tmid, k), LV(c->qh2o, k), lc, &w->mt[k], &w->mp[k],
                    &w->nh2o[k], &w->wratio[k]);
        for (int q = 0; q < 4; q++) w->lk[k * 4 + q] = lc[q];
        double qextref = BND(c->qxvdst, LEV1, k, NREFV);
        w->tauref_l[k] = LV(c->tauref, k) / qextref;
        w->taurefcld_l[k] = LV(c->taurefcld, k) / LV(c->qextrefcld, k);
        for (int nw = 1; nw <= NB; nw++) {
            w->tray[k * NB + nw - 1] = t->tauray[nw - 1] * w->dpr[k];
            w->taeros[k * NB + nw - 1] = w->tauref_l[k] * BND(c->qxvdst, LEV1, k, nw);
            w->tcloud[k * NB + nw - 1] = w->taurefcld_l[k] * BND(c->qxvcld, LEV1, k, nw);
        }
    }
    for (int k = 2; k <= LEV; k++) {
        const int mt = w->mt[k], mp = w->mp[k], nh = w->nh2o[k];
        const double wr = w->wratio[k];
        const double *lk = &w->lk[k * 4];
        for (int nw = 1; nw <= NB; nw++) {
            double trayaer = w->tray[k * NB + nw - 1] + w->taeros[k * NB + nw - 1] +
                             w->tcloud[k * NB + nw - 1];
            for (int ng = 1; ng <= NG - 1; ng++) {
                /* CO2V(mt,mp,nh,nw,ng) with Fortran's linear addressing, so
                 * nh+1 = 11 reads the next band's first water slot exactly as
                 * the reference does (it is then multiplied by WRATIO = 0). */
                ORC_GATHERS(8); /* CO2V corners read below */
#define CV(a, b, h) t->co2v[(a - 1) + ORC_NTREF * ((b - 1) + ORC_PINT * ((h - 1) + ORC_REFH2O * ((nw - 1) + NB * (ng - 1))))]
                double k1 = CV(mt, mp, nh) + wr * (CV(mt, mp, nh + 1) - CV(mt, mp, nh));
                double k2 = CV(mt, mp + 1, nh) + wr * (CV(mt, mp + 1, nh + 1) - CV(mt, mp + 1, nh));
                double k3 = CV(mt + 1, mp + 1, nh) + wr * (CV(mt + 1, mp + 1, nh + 1) - CV(mt + 1, mp + 1, nh));
                double k4 = CV(mt + 1, mp, nh) + wr * (CV(mt + 1, mp, nh + 1) - CV(mt + 1, mp, nh));
#undef CV
                double ans = lk[0] * k1 + lk[1] * k2 + lk[2] * k3 + lk[3] * k4;
                double taugas = w->u[k] * ans;
                w->taugsurf[(nw - 1) + NB * (ng - 1)] += taugas;
                A3(w->dtauk, LEV1, NB, k, nw, ng) = taugas + trayaer;
            }
            A3(w->dtauk, LEV1, NB, k, nw, NG) =
                w->taeros[k * NB + nw - 1] + w->tray[k * NB + nw - 1] + w->tcloud[k * NB + nw - 1];
        }
    }
    for (int nw = 1; nw <= NB; nw++)
        for (int k = 2; k <= LEV; k++) {
            w->taureflk[k * NB + nw - 1] = w->tauref_l[k] * BND(c->qsvdst, LEV1, k, nw);
            w->taucldk[k * NB + nw - 1] = w->taurefcld_l[k] * BND(c->qsvcld, LEV1, k, nw);
        }
#define TR(k) w->tray[(k)*NB + nw - 1]
#define TL(k) w->taureflk[(k)*NB + nw - 1]
#define TC(k) w->taucldk[(k)*NB + nw - 1]
    for (int nw = 1; nw <= NB; nw++) {
        int ng = NG;
        for (int l = 1; l <= c->L; l++) {
            int k = 2 * l + 1;
            double dt = A3(w->dtauk, LEV1, NB, k, nw, ng) + A3(w->dtauk, LEV1, NB, k + 1, nw, ng);
            A3(w->dtau, NLAY, NB, l, nw, ng) = dt;
            A3(w->cosb, NLAY, NB, l, nw, ng) =
                (BND(c->gvdst, LEV1, k, nw) * TL(k) + BND(c->gvdst, LEV1, k + 1, nw) * TL(k + 1) +
                 BND(c->gvcld, LEV1, k, nw) * TC(k) + BND(c->gvcld, LEV1, k + 1, nw) * TC(k + 1)) /
                (TR(k) + TR(k + 1) + TL(k) + TL(k + 1) + TC(k) + TC(k + 1));
            A3(w->wbar, NLAY, NB, l, nw, ng) =
                (TL(k) + TL(k + 1) + TC(k) + TC(k + 1) + (TR(k) + TR(k + 1)) * R4(0.9999)) / dt;
        }
        {
            int l = NLAY, k = 2 * l + 1;
            double dt = A3(w->dtauk, LEV1, NB, k, nw, ng);
            A3(w->dtau, NLAY, NB, l, nw, ng) = dt;
            A3(w->cosb, NLAY, NB, l, nw, ng) =
                (BND(c->gvdst, LEV1, k, nw) * TL(k) + BND(c->gvcld, LEV1, k, nw) * TC(k)) /
                (TR(k) + TL(k) + TC(k));
            A3(w->wbar, NLAY, NB, l, nw, ng) = (TL(k) + TC(k) + TR(k) * R4(0.9999)) / dt;
        }
        for (ng = 1; ng <= NG - 1; ng++) {
            for (int l = 1; l <= c->L; l++) {
                int k = 2 * l + 1;
                double dt = A3(w->dtauk, LEV1, NB, k, nw, ng) + A3(w->dtauk, LEV1, NB, k + 1, nw, ng);
                A3(w->dtau, NLAY, NB, l, nw, ng) = dt;
                A3(w->cosb, NLAY, NB, l, nw, ng) = A3(w->cosb, NLAY, NB, l, nw, NG);
                A3(w->wbar, NLAY, NB, l, nw, ng) =
                    (TL(k) + TL(k + 1) + TC(k) + TC(k + 1) + (TR(k) + TR(k + 1)) * R4(0.9999)) / dt;
            }
            int l = NLAY, k = 2 * l + 1;
            double dt = A3(w->dtauk, LEV1, NB, k, nw, ng);
            A3(w->dtau, NLAY, NB, l, nw, ng) = dt;
            A3(w->cosb, NLAY, NB, l, nw, ng) = A3(w->cosb, NLAY, NB, l, nw, NG);
            A3(w->wbar, NLAY, NB, l, nw, ng) = (TL(k) + TC(k) + TR(k) * R4(0.9999)) / dt;
        }
    }
#undef TR
#undef TL
#undef TC
    /* optcv.f90:251-274: TAUV is recomputed inside getdetau/gfluxv from
     * TAUV(1) = 0, so only TAUCUMV is kept. */
    for (int nw = 1; nw <= NB; nw++)
        for (int ng = 1; ng <= NG; ng++) {
            A3(w->taucum, LEV, NB, 1, nw, ng) = 0.0;
            for (int k = 2; k <= LEV; k++)
                A3(w->taucum, LEV, NB, k, nw, ng) =
                    A3(w->taucum, LEV, NB, k - 1, nw, ng) + A3(w->dtauk, LEV1, NB, k, nw, ng);
        }
}

/* ------------------------------------------------------------------ */
/* optci.f90:1-279 (column c, infrared)                                 */
/* ------------------------------------------------------------------ */
static void optci(const orc_tables *t, const colview *c, work_t *w) {
    const int LEV = c->lev, NLAY = c->nlay, NB = ORC_NSPECTI, NG = ORC_NGAUSS, LEV1 = LEV + 1;
    for (int nw = 1; nw <= NB; nw++)
        for (int ng = 1; ng <= NG; ng++) A3(w->dtauk, LEV1, NB, LEV1, nw, ng) = 0.0;
    for (int ng = 1; ng <= NG - 1; ng++)
        for (int nw = 1; nw <= NB; nw++) w->taugsurf[(nw - 1) + NB * (ng - 1)] = 0.0;
    for (int k = 2; k <= LEV; k++) {
        w->dpr[k] = LV(c->plev, k) - LV(c->plev, k - 1);
        w->u[k] = CMK * w->dpr[k];
        double lc[4];
        orc_tpindex(t, LV(c->pmid, k), LV(c->tmid, k), LV(c->qh2o, k), lc, &w->mt[k], &w->mp[k],
                    &w->nh2o[k], &w->wratio[k]);
        for (int q = 0; q < 4; q++) w->lk[k * 4 + q] = lc[q];
        w->tauref_l[k] = LV(c->tauref, k) / LV(c->qextrefdst, k);
        w->taurefcld_l[k] = LV(c->taurefcld, k) / LV(c->qextrefcld, k);
        for (int nw = 1; nw <= NB; nw++) {
            w->taeros[k * NB + nw - 1] = w->tauref_l[k] * BND(c->qxidst, LEV1, k, nw);
            w->tcloud[k * NB + nw - 1] = w->taurefcld_l[k] * BND(c->qxicld, LEV1, k, nw);
        }
    }
    /* TAUREF(L_LEVELS+1) is not divided by QREFV (the division loop stops at
     * L_LEVELS) but is used below at K = L_LEVELS+1 (optci.f90:113-125,183-186). */
    w->tauref_l[LEV1] = LV(c->tauref, LEV1);
    w->taurefcld_l[LEV1] = LV(c->taurefcld, LEV1);
    for (int k = 2; k <= LEV; k++) {
        const int mt = w->mt[k], mp = w->mp[k], nh = w->nh2o[k];
        const double wr = w->wratio[k];
        const double *lk = &w->lk[k * 4];
        for (int nw = 1; nw <= NB; nw++) {
            for (int ng = 1; ng <= NG - 1; ng++) {
                ORC_GATHERS(8); /* CO2I corners read below */
#define CI(a, b, h) t->co2i[(a - 1) + ORC_NTREF * ((b - 1) + ORC_PINT * ((h - 1) + ORC_REFH2O * ((nw - 1) + NB * (ng - 1))))]
                double k1 = CI(mt, mp, nh) + wr * (CI(mt, mp, nh + 1) - CI(mt, mp, nh));
                double k2 = CI(mt, mp + 1, nh) + wr * (CI(mt, mp + 1, nh + 1) - CI(mt, mp + 1, nh));
                double k3 = CI(mt + 1, mp + 1, nh) + wr * (CI(mt + 1, mp + 1, nh + 1) - CI(mt + 1, mp + 1, nh));
                double k4 = CI(mt + 1, mp, nh) + wr * (CI(mt + 1, mp, nh + 1) - CI(mt + 1, mp, nh));
#undef CI
                double ans = lk[0] * k1 + lk[1] * k2 + lk[2] * k3 + lk[3] * k4;
                double taugas = w->u[k] * ans;
                w->taugsurf[(nw - 1) + NB * (ng - 1)] += taugas;
                A3(w->dtauk, LEV1, NB, k, nw, ng) =
                    taugas + w->taeros[k * NB + nw - 1] + w->tcloud[k * NB + nw - 1];
            }
            A3(w->dtauk, LEV1, NB, k, nw, NG) = w->taeros[k * NB + nw - 1] + w->tcloud[k * NB + nw - 1];
        }
    }
    for (int nw = 1; nw <= NB; nw++)
        for (int k = 2; k <= LEV1; k++) {
            w->taureflk[k * NB + nw - 1] = w->tauref_l[k] * BND(c->qsidst, LEV1, k, nw);
            w->taucldk[k * NB + nw - 1] = w->taurefcld_l[k] * BND(c->qsicld, LEV1, k, nw);
        }
#define TL(k) w->taureflk[(k)*NB + nw - 1]
#define TC(k) w->taucldk[(k)*NB + nw - 1]
    const double tiny = R4(1.0e-9);
    for (int nw = 1; nw <= NB; nw++) {
        for (int pass = 0; pass < 2; pass++) {
            int ng_lo = pass == 0 ? NG : 1, ng_hi = pass == 0 ? NG : NG - 1;
            for (int ng = ng_lo; ng <= ng_hi; ng++)
                for (int l = 1; l <= NLAY; l++) {
                    int k = 2 * l + 1;
                    double dt = A3(w->dtauk, LEV1, NB, k, nw, ng) + A3(w->dtauk, LEV1, NB, k + 1, nw, ng) + 1.0e-50;
                    double wb;
                    if (dt > tiny) {
                        wb = (TL(k) + TL(k + 1) + TC(k) + TC(k + 1)) / dt;
                    } else {
                        wb = 0.0;
                        dt = tiny;
                    }
                    A3(w->dtau, NLAY, NB, l, nw, ng) = dt;
                    A3(w->wbar, NLAY, NB, l, nw, ng) = wb;
                    if (pass == 0) {
                        double tauac = TL(k) + TL(k + 1) + TC(k) + TC(k + 1);
                        double cb = 0.0;
                        if (tauac > 0.0)
                            cb = (BND(c->gidst, LEV1, k, nw) * TL(k) + BND(c->gidst, LEV1, k + 1, nw) * TL(k + 1) +
                                  BND(c->gicld, LEV1, k, nw) * TC(k) + BND(c->gicld, LEV1, k + 1, nw) * TC(k + 1)) /
                                 (TL(k) + TL(k + 1) + TC(k) + TC(k + 1));
                        A3(w->cosb, NLAY, NB, l, nw, ng) = cb;
                    } else {
                        A3(w->cosb, NLAY, NB, l, nw, ng) = A3(w->cosb, NLAY, NB, l, nw, NG);
                    }
                }
        }
    }
#undef TL
#undef TC
    for (int nw = 1; nw <= NB; nw++)
        for (int ng = 1; ng <= NG; ng++) {
            A3(w->taucum, LEV, NB, 1, nw, ng) = 0.0;
            for (int k = 2; k <= LEV; k++)
                A3(w->taucum, LEV, NB, k, nw, ng) =
                    A3(w->taucum, LEV, NB, k - 1, nw, ng) + A3(w->dtauk, LEV1, NB, k, nw, ng);
        }
}

/* ------------------------------------------------------------------ */
/* dtridgl.f90:25-38 and dsolver.f90:48-103                             */
/* ------------------------------------------------------------------ */
static void dtridgl(int L, const double *af, const double *bf, const double *cf, const double *df,
                    double *xk, double *as, double *ds) {
    /* arrays are 1-based here */
    as[L] = af[L] / bf[L];
    ds[L] = df[L] / bf[L];
    for (int i = 2; i <= L; i++) {
        double x = 1.0 / (bf[L + 1 - i] - cf[L + 1 - i] * as[L + 2 - i]);
        as[L + 1 - i] = af[L + 1 - i] * x;
        ds[L + 1 - i] = (df[L + 1 - i] - cf[L + 1 - i] * ds[L + 2 - i]) * x;
    }
    xk[1] = ds[1];
    for (int i = 2; i <= L; i++) {
        double xkb = xk[i - 1];
        xk[i] = ds[i] - as[i] * xkb;
    }
}

static void dsolver(int nl, work_t *w, double btop, double bsurf, double rsf) {
    const double *gama = w->gama, *cp = w->cp, *cm = w->cm, *cpm1 = w->cpm1, *cmm1 = w->cmm1;
    const double *e1 = w->e1, *e2 = w->e2, *e3 = w->e3, *e4 = w->e4;
    double *af = w->af, *bf = w->bf, *cf = w->cf, *df = w->df;
    int L = 2 * nl;
    af[1] = 0.0;
    bf[1] = gama[1] + 1.0;
    cf[1] = gama[1] - 1.0;
    df[1] = btop - cmm1[1];
    int n = 0;
    for (int i = 2; i <= L - 2; i += 2) {
        n++;
        af[i] = (e1[n] + e3[n]) * (gama[n + 1] - 1.0);
        bf[i] = (e2[n] + e4[n]) * (gama[n + 1] - 1.0);
        cf[i] = 2.0 * (1.0 - gama[n + 1] * gama[n + 1]);
        df[i] = (gama[n + 1] - 1.0) * (cpm1[n + 1] - cp[n]) + (1.0 - gama[n + 1]) * (cm[n] - cmm1[n + 1]);
    }
    n = 0;
    for (int i = 3; i <= L - 1; i += 2) {
        n++;
        af[i] = 2.0 * (1.0 - gama[n] * gama[n]);
        bf[i] = (e1[n] - e3[n]) * (1.0 + gama[n + 1]);
        cf[i] = (e1[n] + e3[n]) * (gama[n + 1] - 1.0);
        df[i] = e3[n] * (cpm1[n + 1] - cp[n]) + e1[n] * (cm[n] - cmm1[n + 1]);
    }
    af[L] = e1[nl] - rsf * e3[nl];
    bf[L] = e2[nl] - rsf * e4[nl];
    cf[L] = 0.0;
    df[L] = bsurf - cp[nl] + rsf * cm[nl];
    dtridgl(L, af, bf, cf, df, w->xk, w->as, w->ds);
    for (n = 1; n <= nl; n++) {
        w->xk1[n] = w->xk[2 * n - 1] + w->xk[2 * n];
        w->xk2[n] = w->xk[2 * n - 1] - w->xk[2 * n];
        if (w->xk2[n] == 0.0) continue;
        if (fabs(w->xk2[n] / (w->xk[2 * n - 1] + R4(1.e-20))) < R4(1.E-30)) w->xk2[n] = 0.0;
    }
}

/* ------------------------------------------------------------------ */
/* getdetau.f90:304-335 / gfluxv.f90:240-272: delta-Eddington scaling. */
/* dtdel, wdel, cdel: layer arrays (1-based, length nlay); taucumin:     */
/* level array (1-based, length lev).  Fills w0, cosbar, dtaul, tau,     */
/* tcum; returns detau.                                                  */
/* ------------------------------------------------------------------ */
static double deltaedd(int nlay, int lev, const double *dtdel, double tdel1, const double *wdel,
                       const double *cdel, const double *taucumin, work_t *w) {
    double factor = 1.0 - wdel[1] * (cdel[1] * cdel[1]);
    w->tau[1] = tdel1 * factor;
    w->tcum[1] = 0.0;
    w->tcum[2] = taucumin[2] * factor;
    w->tcum[3] = w->tcum[2] + (taucumin[3] - taucumin[2]) * factor;
    for (int l = 1; l <= nlay - 1; l++) {
        factor = 1.0 - wdel[l] * (cdel[l] * cdel[l]);
        w->w0[l] = wdel[l] * (1.0 - cdel[l] * cdel[l]) / factor;
        w->cosbar[l] = cdel[l] / (1.0 + cdel[l]);
        w->dtaul[l] = dtdel[l] * factor;
        w->tau[l + 1] = w->tau[l] + w->dtaul[l];
        int k = 2 * (l + 1);
        w->tcum[k] = w->tau[l + 1];
        w->tcum[k + 1] = w->tcum[k] + (taucumin[k + 1] - taucumin[k]) * factor;
    }
    int l = nlay;
    factor = 1.0 - wdel[l] * (cdel[l] * cdel[l]);
    w->w0[l] = wdel[l] * (1.0 - cdel[l] * cdel[l]) / factor;
    w->cosbar[l] = cdel[l] / (1.0 + cdel[l]);
    w->dtaul[l] = dtdel[l] * factor;
    w->tau[l + 1] = w->tau[l] + w->dtaul[l];
    w->tcum[2 * l + 1] = w->tau[l + 1];
    (void)lev;
    return w->tcum[2 * l + 1];
}

/* gfluxv.f90:274-450 (after the delta-Eddington block). */
static void gfluxv(int nlay, int lev, double ubar0, double f0pi, double rsf, double btop,
                   double bsurf, work_t *w, double *diffv, double *fluxup, double *fluxdn) {
    const double s3 = (double)sqrtf(3.0f); /* SQRT(3.0) folded in REAL*4 */
    const double s3h = (double)(sqrtf(3.0f) * 0.5f);
    double *w0 = w->w0, *cosbar = w->cosbar, *tau = w->tau, *tcum = w->tcum;
    for (int l = 1; l <= nlay; l++) {
        w->g1[l] = s3h * (2.0 - w0[l] * (1.0 + cosbar[l]));
        w->g2[l] = (s3 * w0[l] * 0.5) * (1.0 - cosbar[l]);
        w->g3[l] = 0.5 * (1.0 - s3 * cosbar[l] * ubar0);
        w->lamda[l] = sqrt(w->g1[l] * w->g1[l] - w->g2[l] * w->g2[l]);
        w->gama[l] = (w->g1[l] - w->lamda[l]) / w->g2[l];
    }
    for (int l = 1; l <= nlay; l++) {
        double g4 = 1.0 - w->g3[l];
        double denom = w->lamda[l] * w->lamda[l] - 1.0 / (ubar0 * ubar0);
        if (denom == 0.0) denom = R4(1.E-10);
        double am = f0pi * w0[l] * (g4 * (w->g1[l] + 1.0 / ubar0) + w->g2[l] * w->g3[l]) / denom;
        double ap = f0pi * w0[l] * (w->g3[l] * (w->g1[l] - 1.0 / ubar0) + w->g2[l] * g4) / denom;
        double x0 = tau[l] / ubar0, x1 = tau[l + 1] / ubar0;
        double et0 = cexp_(-(x0 < MAXEXP ? x0 : MAXEXP));
        double et1 = cexp_(-(x1 < MAXEXP ? x1 : MAXEXP));
        w->cpm1[l] = ap * et0;
        w->cmm1[l] = am * et0;
        w->cp[l] = ap * et1;
        w->cm[l] = am * et1;
    }
    for (int l = 1; l <= nlay; l++) {
        double x = w->lamda[l] * w->dtaul[l];
        double exptrm = TAUMAX < x ? TAUMAX : x;
        double ep = cexp_(exptrm);
        double em = 1.0 / ep;
        w->e1[l] = ep + w->gama[l] * em;
        w->e2[l] = ep - w->gama[l] * em;
        w->e3[l] = w->gama[l] * ep + em;
        w->e4[l] = w->gama[l] * ep - em;
    }
    dsolver(nlay, w, btop, bsurf, rsf);
    for (int l = 1; l <= nlay - 1; l++) {
        double x = w->lamda[l] * (tcum[2 * l + 1] - tcum[2 * l]);
        double exptrm = TAUMAX < x ? TAUMAX : x;
        double ep = cexp_(exptrm);
        double em = 1.0 / ep;
        double g4 = 1.0 - w->g3[l];
        double denom = w->lamda[l] * w->lamda[l] - 1.0 / (ubar0 * ubar0);
        if (denom == 0.0) denom = R4(1.E-10);
        double am = f0pi * w0[l] * (g4 * (w->g1[l] + 1.0 / ubar0) + w->g2[l] * w->g3[l]) / denom;
        double ap = f0pi * w0[l] * (w->g3[l] * (w->g1[l] - 1.0 / ubar0) + w->g2[l] * g4) / denom;
        double taumid = tcum[2 * l + 1];
        double xm = taumid / ubar0;
        double et = cexp_(-(xm < MAXEXP ? xm : MAXEXP));
        double cpmid = ap * et;
        double cmmid = am * et;
        w->fmidp[l] = w->xk1[l] * ep + w->gama[l] * w->xk2[l] * em + cpmid;
        w->fmidm[l] = w->xk1[l] * ep * w->gama[l] + w->xk2[l] * em + cmmid;
        w->fmidm[l] = w->fmidm[l] + ubar0 * f0pi * et;
    }
    {
        double ep = 1.0, em = 1.0;
        double g4 = 1.0 - w->g3[1];
        double denom = w->lamda[1] * w->lamda[1] - 1.0 / (ubar0 * ubar0);
        if (denom == 0.0) denom = R4(1.E-10);
        double am = f0pi * w0[1] * (g4 * (w->g1[1] + 1.0 / ubar0) + w->g2[1] * w->g3[1]) / denom;
        double ap = f0pi * w0[1] * (w->g3[1] * (w->g1[1] - 1.0 / ubar0) + w->g2[1] * g4) / denom;
        double cpmid = ap, cmmid = am;
        *fluxup = w->xk1[1] * ep + w->gama[1] * w->xk2[1] * em + cpmid;
        *fluxdn = w->xk1[1] * ep * w->gama[1] + w->xk2[1] * em + cmmid;
        double x = tcum[1] / ubar0;
        *fluxdn = *fluxdn + ubar0 * f0pi * cexp_(-(x < MAXEXP ? x : MAXEXP));
    }
    {
        int l = nlay;
        double x = w->lamda[l] * (tcum[lev] - tcum[lev - 1]);
        double exptrm = TAUMAX < x ? TAUMAX : x;
        double ep = cexp_(exptrm);
        double em = 1.0 / ep;
        double g4 = 1.0 - w->g3[l];
        double denom = w->lamda[l] * w->lamda[l] - 1.0 / (ubar0 * ubar0);
        if (denom == 0.0) denom = R4(1.E-10);
        double am = f0pi * w0[l] * (g4 * (w->g1[l] + 1.0 / ubar0) + w->g2[l] * w->g3[l]) / denom;
        double ap = f0pi * w0[l] * (w->g3[l] * (w->g1[l] - 1.0 / ubar0) + w->g2[l] * g4) / denom;
        double taumid = tcum[lev] < TAUMAX ? tcum[lev] : TAUMAX;
        double xm = taumid / ubar0;
        double et = cexp_(-(xm < MAXEXP ? xm : MAXEXP));
        double cpmid = ap * et;
        double cmmid = am * et;
        w->fmidp[l] = w->xk1[l] * ep + w->gama[l] * w->xk2[l] * em + cpmid;
        w->fmidm[l] = w->xk1[l] * ep * w->gama[l] + w->xk2[l] * em + cmmid;
        *diffv = w->fmidm[l];
        w->fmidm[l] = w->fmidm[l] + ubar0 * f0pi * et;
    }
}

/* Planck table index NT = T*10.0D0-499 assigned to an INTEGER (truncation
 * toward zero): code/sfluxi.f90:54-55, code/gfluxi.f90:73-74,86-87. */
int orc_planck_index(double t) { return (int)(t * 10.0 - 499); }

/* gfluxi.f90:213-344 */
static void gfluxi(int nlay, const orc_tables *t, const double *tlev, int nw, const double *dtau,
                   const double *taucum, const double *w0, const double *cosbar, double rsf,
                   double btop, double bsurf, work_t *w, double *ftopup) {
    for (int l = 1; l <= nlay - 1; l++) {
        w->alpha[l] = sqrt((1.0 - w0[l]) / (1.0 - w0[l] * cosbar[l]));
        w->lamda[l] = w->alpha[l] * (1.0 - w0[l] * cosbar[l]) / UBARI;
        int nt2 = orc_planck_index(tlev[2 * l + 2 - 1]);
        int nt = orc_planck_index(tlev[2 * l - 1]);
        w->b1[l] = (t->planckir[(nt2 - 1) * 5 + nw - 1] - t->planckir[(nt - 1) * 5 + nw - 1]) / dtau[l];
        w->b0[l] = t->planckir[(nt - 1) * 5 + nw - 1];
    }
    {
        int l = nlay;
        w->alpha[l] = sqrt((1.0 - w0[l]) / (1.0 - w0[l] * cosbar[l]));
        w->lamda[l] = w->alpha[l] * (1.0 - w0[l] * cosbar[l]) / UBARI;
        int nt = orc_planck_index(tlev[2 * l + 1 - 1]);
        int nt2 = orc_planck_index(tlev[2 * l - 1]);
        w->b1[l] = (t->planckir[(nt - 1) * 5 + nw - 1] - t->planckir[(nt2 - 1) * 5 + nw - 1]) / dtau[l];
        w->b0[l] = t->planckir[(nt2 - 1) * 5 + nw - 1];
    }
    for (int l = 1; l <= nlay; l++) {
        w->gama[l] = (1.0 - w->alpha[l]) / (1.0 + w->alpha[l]);
        double term = UBARI / (1.0 - w0[l] * cosbar[l]);
        w->cp[l] = w->b0[l] + w->b1[l] * dtau[l] + w->b1[l] * term;
        w->cm[l] = w->b0[l] + w->b1[l] * dtau[l] - w->b1[l] * term;
        w->cpm1[l] = w->b0[l] + w->b1[l] * term;
        w->cmm1[l] = w->b0[l] - w->b1[l] * term;
    }
    for (int l = 1; l <= nlay; l++) {
        double x = w->lamda[l] * dtau[l];
        double ep = cexp_(x < TAUMAX ? x : TAUMAX);
        double em = 1.0 / ep;
        w->e1[l] = ep + w->gama[l] * em;
        w->e2[l] = ep - w->gama[l] * em;
        w->e3[l] = w->gama[l] * ep + em;
        w->e4[l] = w->gama[l] * ep - em;
    }
    dsolver(nlay, w, btop, bsurf, rsf);
    for (int l = 1; l <= nlay - 1; l++) {
        double dtauk = taucum[2 * l + 1] - taucum[2 * l];
        double x = w->lamda[l] * dtauk;
        double ep = cexp_(x < TAUMAX ? x : TAUMAX);
        double em = 1.0 / ep;
        double term = UBARI / (1.0 - w0[l] * cosbar[l]);
        double cpmid = w->b0[l] + w->b1[l] * dtauk + w->b1[l] * term;
        double cmmid = w->b0[l] + w->b1[l] * dtauk - w->b1[l] * term;
        w->fmidp[l] = w->xk1[l] * ep + w->gama[l] * w->xk2[l] * em + cpmid;
        w->fmidm[l] = w->xk1[l] * ep * w->gama[l] + w->xk2[l] * em + cmmid;
        w->fmidp[l] = w->fmidp[l] * PI;
        w->fmidm[l] = w->fmidm[l] * PI;
    }
    {
        int l = nlay;
        double x = w->lamda[l] * dtau[l];
        double ep = cexp_(x < TAUMAX ? x : TAUMAX);
        double em = 1.0 / ep;
        double term = UBARI / (1.0 - w0[l] * cosbar[l]);
        double cpmid = w->b0[l] + w->b1[l] * dtau[l] + w->b1[l] * term;
        double cmmid = w->b0[l] + w->b1[l] * dtau[l] - w->b1[l] * term;
        w->fmidp[l] = w->xk1[l] * ep + w->gama[l] * w->xk2[l] * em + cpmid;
        w->fmidm[l] = w->xk1[l] * ep * w->gama[l] + w->xk2[l] * em + cmmid;
        w->fmidp[l] = w->fmidp[l] * PI;
        w->fmidm[l] = w->fmidm[l] * PI;
    }
    {
        double ep = 1.0, em = 1.0;
        double term = UBARI / (1.0 - w0[1] * cosbar[1]);
        double cpmid = w->b0[1] + w->b1[1] * term;
        double cmmid = w->b0[1] - w->b1[1] * term;
        double fluxup = w->xk1[1] * ep + w->gama[1] * w->xk2[1] * em + cpmid;
        double fluxdn = w->xk1[1] * ep * w->gama[1] + w->xk2[1] * em + cmmid;
        *ftopup = (fluxup - fluxdn) * PI;
    }
}

/* ------------------------------------------------------------------ */
/* Radiation block of comp3.f for one column                             */
/* ------------------------------------------------------------------ */
static void column(const orc_tables *t, const orc_batch *b, int col, work_t *w) {
    const int L = b->L, LEV = 2 * L + 3, NLAY = L + 1, LEV1 = LEV + 1;
    colview c;
    c.L = L;
    c.lev = LEV;
    c.nlay = NLAY;
    c.plev = b->plev + (size_t)col * LEV;
    c.tlev = b->tlev + (size_t)col * LEV;
    c.pmid = b->pmid + (size_t)col * LEV;
    c.tmid = b->tmid + (size_t)col * LEV;
    c.qh2o = b->qh2o + (size_t)col * LEV;
    c.tauref = b->tauref + (size_t)col * LEV1;
    c.qextrefdst = b->qextrefdst + (size_t)col * LEV1;
    c.qxvdst = b->qxvdst + (size_t)col * 7 * LEV1;
    c.qsvdst = b->qsvdst + (size_t)col * 7 * LEV1;
    c.gvdst = b->gvdst + (size_t)col * 7 * LEV1;
    c.qxidst = b->qxidst + (size_t)col * 5 * LEV1;
    c.qsidst = b->qsidst + (size_t)col * 5 * LEV1;
    c.gidst = b->gidst + (size_t)col * 5 * LEV1;
    if (b->taurefcld) {
        c.taurefcld = b->taurefcld + (size_t)col * LEV1;
        c.qextrefcld = b->qextrefcld + (size_t)col * LEV1;
        c.qxvcld = b->qxvcld + (size_t)col * 7 * LEV1;
        c.qsvcld = b->qsvcld + (size_t)col * 7 * LEV1;
        c.gvcld = b->gvcld + (size_t)col * 7 * LEV1;
        c.qxicld = b->qxicld + (size_t)col * 5 * LEV1;
        c.qsicld = b->qsicld + (size_t)col * 5 * LEV1;
        c.gicld = b->gicld + (size_t)col * 5 * LEV1;
    } else {
        /* CLOUDON = .FALSE. (comp3.f:626-630, ini_optcld.f): TAUREFCLD = 0,
         * QEXTREFCLD = 1 and the cloud Q/g arrays are zero. */
        c.taurefcld = zero_lev;
        c.qextrefcld = one_lev;
        c.qxvcld = c.qsvcld = c.gvcld = zero_band;
        c.qxicld = c.qsicld = c.gicld = zero_band;
    }
    const double acosz = b->acosz[col], als = b->als[col], albi = b->albi[col];
    double *detau = b->detau + (size_t)col * 119;
    double *cumtauv = b->cumtauv + (size_t)col * 119;
    double suntot[MAXLAY + 1], irtotal[MAXLAY + 1];
    double *fmnetv = b->fmnetv + (size_t)col * NLAY, *fluxupv = b->fluxupv + (size_t)col * NLAY;
    double *fluxdnv = b->fluxdnv + (size_t)col * NLAY;
    double *fmneti = b->fmneti + (size_t)col * NLAY, *fluxupi = b->fluxupi + (size_t)col * NLAY;
    double *fluxdni = b->fluxdni + (size_t)col * NLAY;
    double nfluxtopv = 0.0, diffvt = 0.0, nfluxtopi = 0.0;

    if (acosz >= R4(1.0e-5)) {
        /* comp3.f:658-681 */
        optcv(t, &c, w);
        for (int nw = 1; nw <= 7; nw++)
            for (int ng = 1; ng <= 17; ng++)
                cumtauv[(nw - 1) + 7 * (ng - 1)] = A3(w->taucum, LEV, 7, LEV, nw, ng);
        /* sfluxv.f90:43-164 */
        for (int l = 1; l <= NLAY; l++) fmnetv[l - 1] = fluxupv[l - 1] = fluxdnv[l - 1] = 0.0;
        const double ubar0 = acosz, rsfv = als;
        double dtdel[MAXLAY + 1], wdel[MAXLAY + 1], cdel[MAXLAY + 1], tci[MAXLEV + 1];
        for (int nw = 1; nw <= 7; nw++) {
            double f0pi = b->sol[nw - 1];
            double fzero = t->fzerov[nw - 1];
            for (int ng = (fzero >= R4(0.99) ? 17 : 1); ng <= 17; ng++) {
                for (int l = 1; l <= NLAY; l++) {
                    dtdel[l] = A3(w->dtau, NLAY, 7, l, nw, ng);
                    wdel[l] = A3(w->wbar, NLAY, 7, l, nw, ng);
                    cdel[l] = A3(w->cosb, NLAY, 7, l, nw, ng);
                }
                for (int k = 1; k <= LEV; k++) tci[k] = A3(w->taucum, LEV, 7, k, nw, ng);
                /* getdetau (sfluxv.f90:68-70,130-132): TAUV(1) = 0 */
                double de = deltaedd(NLAY, LEV, dtdel, 0.0, wdel, cdel, tci, w);
                detau[(nw - 1) + 7 * (ng - 1)] = de;
                double wgt;
                if (ng < 17) {
                    if (w->taugsurf[(nw - 1) + 7 * (ng - 1)] < TLIMITS) {
                        fzero = fzero + (1.0 - t->fzerov[nw - 1]) * t->gweight[ng - 1];
                        continue;
                    }
                }
                double btop = 0.0;
                double x = de / ubar0;
                double eterm = x < MAXEXP ? x : MAXEXP;
                double bsurf = rsfv * ubar0 * b->sol[nw - 1] * cexp_(-eterm);
                double diffv, fluxup, fluxdn;
                gfluxv(NLAY, LEV, ubar0, f0pi, rsfv, btop, bsurf, w, &diffv, &fluxup, &fluxdn);
                if (ng < 17) {
                    nfluxtopv = nfluxtopv + (fluxup - fluxdn) * t->gweight[ng - 1] * (1.0 - t->fzerov[nw - 1]);
                    for (int l = 1; l <= NLAY; l++) {
                        fmnetv[l - 1] = fmnetv[l - 1] + (w->fmidp[l] - w->fmidm[l]) * t->gweight[ng - 1] * (1.0 - t->fzerov[nw - 1]);
                        fluxupv[l - 1] = fluxupv[l - 1] + w->fmidp[l] * t->gweight[ng - 1] * (1.0 - t->fzerov[nw - 1]);
                        fluxdnv[l - 1] = fluxdnv[l - 1] + w->fmidm[l] * t->gweight[ng - 1] * (1.0 - t->fzerov[nw - 1]);
                    }
                    diffvt = diffvt + diffv * t->gweight[ng - 1] * (1.0 - t->fzerov[nw - 1]);
                } else {
                    wgt = fzero;
                    nfluxtopv = nfluxtopv + (fluxup - fluxdn) * wgt;
                    for (int l = 1; l <= NLAY; l++) {
                        fmnetv[l - 1] = fmnetv[l - 1] + (w->fmidp[l] - w->fmidm[l]) * wgt;
                        fluxupv[l - 1] = fluxupv[l - 1] + w->fmidp[l] * wgt;
                        fluxdnv[l - 1] = fluxdnv[l - 1] + w->fmidm[l] * wgt;
                    }
                    diffvt = diffvt + diffv * wgt;
                }
            }
        }
        suntot[1] = fmnetv[0] - nfluxtopv;
        for (int l = 2; l <= NLAY; l++) suntot[l] = fmnetv[l - 1] - fmnetv[l - 2];
    } else {
        /* comp3.f:683-696 (the reference leaves FMNETV, NFLUXTOPV and the
         * interior FLUXUPV stale; they are zero here) */
        for (int l = 1; l <= NLAY; l++) {
            suntot[l] = 0.0;
            fmnetv[l - 1] = fluxupv[l - 1] = fluxdnv[l - 1] = 0.0;
        }
        diffvt = 0.0;
        nfluxtopv = 0.0;
    }
    b->nfluxtopv[col] = nfluxtopv;
    b->diffvt[col] = diffvt;
    b->dnvflux[col] = fluxdnv[NLAY - 1];
    b->dndiffv[col] = diffvt;

    /* comp3.f:712-738: IR */
    optci(t, &c, w);
    {
        const double *tlev = c.tlev, *plev = c.plev;
        for (int l = 1; l <= NLAY; l++) fmneti[l - 1] = fluxupi[l - 1] = fluxdni[l - 1] = 0.0;
        double ttop = tlev[2 - 1], tsurf = tlev[LEV - 1];
        int nts = orc_planck_index(tsurf);
        int ntt = orc_planck_index(ttop);
        double dtau[MAXLAY + 1], wb[MAXLAY + 1], cb[MAXLAY + 1], tci[MAXLEV + 1];
        for (int nw = 1; nw <= 5; nw++) {
            double bsurf = (1.0 - albi) * t->planckir[(nts - 1) * 5 + nw - 1];
            double pltop = t->planckir[(ntt - 1) * 5 + nw - 1];
            double fzero = t->fzeroi[nw - 1];
            for (int ng = (fzero >= R4(0.99) ? 17 : 1); ng <= 17; ng++) {
                if (ng < 17 && w->taugsurf[(nw - 1) + 5 * (ng - 1)] < TLIMITI) {
                    fzero = fzero + (1.0 - t->fzeroi[nw - 1]) * t->gweight[ng - 1];
                    continue;
                }
                for (int l = 1; l <= NLAY; l++) {
                    dtau[l] = A3(w->dtau, NLAY, 5, l, nw, ng);
                    wb[l] = A3(w->wbar, NLAY, 5, l, nw, ng);
                    cb[l] = A3(w->cosb, NLAY, 5, l, nw, ng);
                }
                for (int k = 1; k <= LEV; k++) tci[k] = A3(w->taucum, LEV, 5, k, nw, ng);
                double tautop = dtau[1] * plev[2 - 1] / (plev[4 - 1] - plev[2 - 1]);
                double btop = (1.0 - cexp_(-tautop / UBARI)) * pltop;
                double ftopup;
                gfluxi(NLAY, t, tlev, nw, dtau, tci, wb, cb, albi, btop, bsurf, w, &ftopup);
                double dw = t->dwni[nw - 1];
                if (ng < 17) {
                    double g = t->gweight[ng - 1], f = 1.0 - t->fzeroi[nw - 1];
                    nfluxtopi = nfluxtopi + ftopup * dw * g * f;
                    for (int l = 1; l <= NLAY; l++) {
                        fmneti[l - 1] = fmneti[l - 1] + (w->fmidp[l] - w->fmidm[l]) * dw * g * f;
                        fluxupi[l - 1] = fluxupi[l - 1] + w->fmidp[l] * dw * g * f;
                        fluxdni[l - 1] = fluxdni[l - 1] + w->fmidm[l] * dw * g * f;
                    }
                } else {
                    nfluxtopi = nfluxtopi + ftopup * dw * fzero;
                    for (int l = 1; l <= NLAY; l++) {
                        fmneti[l - 1] = fmneti[l - 1] + (w->fmidp[l] - w->fmidm[l]) * dw * fzero;
                        fluxupi[l - 1] = fluxupi[l - 1] + w->fmidp[l] * dw * fzero;
                        fluxdni[l - 1] = fluxdni[l - 1] + w->fmidm[l] * dw * fzero;
                    }
                }
            }
        }
    }
    irtotal[1] = fmneti[0] - nfluxtopi;
    for (int l = 2; l <= NLAY; l++) irtotal[l] = fmneti[l - 1] - fmneti[l - 2];
    b->nfluxtopi[col] = nfluxtopi;
    b->dnirflux[col] = fluxdni[NLAY - 1];
    b->fluxsurf[col] = (1.0 - als) * fluxdnv[NLAY - 1];

    /* comp3.f:765-771 with YM (comp3.f:480-484) and OM (potemp1.f:95-106).
     * PL(K) = PLEV(K) for K >= 2 (fillpt.f90:30-35, potemp1.f:95-101). */
    double *suntot_o = b->suntot + (size_t)col * NLAY, *irtotal_o = b->irtotal + (size_t)col * NLAY;
    double *qrad = b->qrad + (size_t)col * NLAY;
    const double ptrop = b->ptrop, p = b->pcol[col];
    const double *plev = c.plev;
    for (int l = 1; l <= NLAY; l++) {
        int k = 2 * l; /* QRAD(K), K = 2,4,...,2L+2 */
        double ym = (k == 2) ? ptrop * SCALEP / GRAV : (plev[k + 1 - 1] - plev[k - 1 - 1]) * SCALEP / GRAV;
        double om = pow(plev[k - 1] / plev[LEV - 1], KAPA);
        double pnlte = b->sigma[k - 1] * (p - ptrop) + ptrop;
        double sunlte = suntot[l] * 2.2e4 * pnlte / (1.0 + 2.2e4 * pnlte);
        qrad[l - 1] = (sunlte + irtotal[l]) / (CPHEAT * ym * om);
        suntot_o[l - 1] = suntot[l];
        irtotal_o[l - 1] = irtotal[l];
    }
}

static void init_consts(void) {
    static int done = 0;
    if (done) return;
    for (int i = 0; i < MAXLEV + 2; i++) one_lev[i] = 1.0;
    done = 1;
}

typedef struct {
    const orc_tables *t;
    const orc_batch *b;
    int c0, c1, err;
} runarg_t;

static void *run_range(void *p) {
    runarg_t *a = (runarg_t *)p;
    work_t *w = (work_t *)malloc(sizeof(work_t));
    if (!w) {
        a->err = -2;
        return NULL;
    }
    for (int col = a->c0; col < a->c1; col++) column(a->t, a->b, col, w);
    free(w);
    return NULL;
}

int orc_run_batch(const orc_tables *t, const orc_batch *b, int nthreads) {
    if (b->L < 1 || b->L > ORC_MAXL) return -1;
    init_consts();
    int nt = nthreads;
    if (nt <= 0) nt = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nt < 1) nt = 1;
    if (nt > b->ncol) nt = b->ncol > 0 ? b->ncol : 1;
    runarg_t *args = (runarg_t *)calloc((size_t)nt, sizeof(runarg_t));
    pthread_t *th = (pthread_t *)calloc((size_t)nt, sizeof(pthread_t));
    int per = (b->ncol + nt - 1) / nt;
    for (int i = 0; i < nt; i++) {
        args[i].t = t;
        args[i].b = b;
        args[i].c0 = i * per < b->ncol ? i * per : b->ncol;
        args[i].c1 = (i + 1) * per < b->ncol ? (i + 1) * per : b->ncol;
    }
    for (int i = 1; i < nt; i++) pthread_create(&th[i], NULL, run_range, &args[i]);
    run_range(&args[0]);
    int err = args[0].err;
    for (int i = 1; i < nt; i++) {
        pthread_join(th[i], NULL);
        if (args[i].err) err = args[i].err;
    }
    free(args);
    free(th);
    return err;
}

void orc_optics_column(const orc_tables *t, const orc_batch *b, int col, double *dtauv,
                       double *wbarv, double *cosbv, double *taucumv, double *taugsurfv,
                       double *dtaui, double *wbari, double *cosbi, double *taucumi,
                       double *taugsurfi) {
    init_consts();
    const int L = b->L, LEV = 2 * L + 3, NLAY = L + 1, LEV1 = LEV + 1;
    work_t *w = (work_t *)malloc(sizeof(work_t));
    colview c;
    c.L = L;
    c.lev = LEV;
    c.nlay = NLAY;
    c.plev = b->plev + (size_t)col * LEV;
    c.tlev = b->tlev + (size_t)col * LEV;
    c.pmid = b->pmid + (size_t)col * LEV;
    c.tmid = b->tmid + (size_t)col * LEV;
    c.qh2o = b->qh2o + (size_t)col * LEV;
    c.tauref = b->tauref + (size_t)col * LEV1;
    c.qextrefdst = b->qextrefdst + (size_t)col * LEV1;
    c.qxvdst = b->qxvdst + (size_t)col * 7 * LEV1;
    c.qsvdst = b->qsvdst + (size_t)col * 7 * LEV1;
    c.gvdst = b->gvdst + (size_t)col * 7 * LEV1;
    c.qxidst = b->qxidst + (size_t)col * 5 * LEV1;
    c.qsidst = b->qsidst + (size_t)col * 5 * LEV1;
    c.gidst = b->gidst + (size_t)col * 5 * LEV1;
    if (b->taurefcld) {
        c.taurefcld = b->taurefcld + (size_t)col * LEV1;
        c.qextrefcld = b->qextrefcld + (size_t)col * LEV1;
        c.qxvcld = b->qxvcld + (size_t)col * 7 * LEV1;
        c.qsvcld = b->qsvcld + (size_t)col * 7 * LEV1;
        c.gvcld = b->gvcld + (size_t)col * 7 * LEV1;
        c.qxicld = b->qxicld + (size_t)col * 5 * LEV1;
        c.qsicld = b->qsicld + (size_t)col * 5 * LEV1;
        c.gicld = b->gicld + (size_t)col * 5 * LEV1;
    } else {
        c.taurefcld = zero_lev;
        c.qextrefcld = one_lev;
        c.qxvcld = c.qsvcld = c.gvcld = zero_band;
        c.qxicld = c.qsicld = c.gicld = zero_band;
    }
    optcv(t, &c, w);
    memcpy(dtauv, w->dtau, sizeof(double) * NLAY * 7 * 17);
    memcpy(wbarv, w->wbar, sizeof(double) * NLAY * 7 * 17);
    memcpy(cosbv, w->cosb, sizeof(double) * NLAY * 7 * 17);
    memcpy(taucumv, w->taucum, sizeof(double) * LEV * 7 * 17);
    memcpy(taugsurfv, w->taugsurf, sizeof(double) * 7 * 16);
    optci(t, &c, w);
    memcpy(dtaui, w->dtau, sizeof(double) * NLAY * 5 * 17);
    memcpy(wbari, w->wbar, sizeof(double) * NLAY * 5 * 17);
    memcpy(cosbi, w->cosb, sizeof(double) * NLAY * 5 * 17);
    memcpy(taucumi, w->taucum, sizeof(double) * LEV * 5 * 17);
    memcpy(taugsurfi, w->taugsurf, sizeof(double) * 5 * 16);
    free(w);
}

/* dsolflux.f:28-45 with the day test of comp3.f:335-349. */
void orc_dsolflux(const orc_tables *t, int ncol, const double *sol, const double *acosz,
                  const double *detau, double *directsol) {
    for (int col = 0; col < ncol; col++) {
        double ubar0 = acosz[col];
        double ds = 0.0;
        if (ubar0 >= R4(1.0e-5)) {
            const double *de = detau + (size_t)col * 119;
            for (int nw = 1; nw <= 7; nw++) {
                double factor = ubar0 * sol[nw - 1];
                for (int ng = 1; ng <= 16; ng++) {
                    double d = de[(nw - 1) + 7 * (ng - 1)];
                    if (d <= 5.0)
                        ds = ds + factor * cexp_(-d / ubar0) * t->gweight[ng - 1] * (1.0 - t->fzerov[nw - 1]);
                }
                double d = de[(nw - 1) + 7 * 16];
                if (d <= 5.0) ds = ds + factor * cexp_(-d / ubar0) * t->fzerov[nw - 1];
            }
        }
        directsol[col] = ds;
    }
}

/* The column exponential and logarithm, exported for tests. */
double orc_exp(double x) { return cexp_(x); }
double orc_log10(double x) { return mgcm_rt_log10(x); }
double orc_erf(double x) { return mgcm_rt_erf(x); }
double orc_ln(double x) { return mgcm_rt_ln(x); }
double orc_pow(double x, double y) { return mgcm_rt_pow(x, y); }

/* ======================================================================
 * Aerosol optics.  Table set-up: code/initcld.f:141-190 (bins, REAL*4
 * literals, ATHIRD = REAL*4 (1./3.)), code/setrad.f90:73-105,132-155.
 * Per column: code/opt_dst.f:55-161, code/opt_cld.f:55-188,
 * code/ini_optdst.f:29-51, the choice in code/comp3.f:592-630.  Powers,
 * logs, exps and DERF use the deterministic routines of mgcm_rt_math.h. */
static int read_real4(const char *path, double *v, size_t n) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    size_t k = 0;
    char tok[64];
    while (k < n && fscanf(f, "%63s", tok) == 1) v[k++] = (double)strtof(tok, NULL);
    fclose(f);
    return k == n ? 0 : -2;
}

int orc_aero_load(orc_aero *a, const char *dir) {
    const double athird = (double)(1.0f / 3.0f);
    double rad[ORC_NBIN];
    rad[0] = R4(1.e-7);
    rad[ORC_NBIN - 1] = R4(50.e-6);
    a->radb[0] = R4(0.0001e-6);
    a->radb[ORC_NBIN] = R4(1.e-2);
    double vrat = log(rad[ORC_NBIN - 1] / rad[0]) / (double)(float)(ORC_NBIN - 1) * 3.0;
    vrat = exp(vrat);
    for (int i = 0; i < ORC_NBIN - 1; ++i) {
        rad[i + 1] = rad[i] * pow(vrat, athird);
        a->radb[i + 1] = pow((2.0 * vrat) / (vrat + 1.0), athird) * rad[i];
    }
    const size_t ncv = (size_t)ORC_NRATIO * ORC_NBIN * 3 * ORC_NSPECTV, nci = (size_t)ORC_NRATIO * ORC_NBIN * 3 * ORC_NSPECTI;
    const size_t ndv = (size_t)ORC_NBIN * 3 * ORC_NSPECTV, ndi = (size_t)ORC_NBIN * 3 * ORC_NSPECTI;
    double *cv = (double *)malloc(ncv * sizeof(double)), *ci = (double *)malloc(nci * sizeof(double));
    double *dv = (double *)malloc(ndv * sizeof(double)), *di = (double *)malloc(ndi * sizeof(double));
    char path[4096];
    int rc = 0;
    snprintf(path, sizeof path, "%s/waterCoated_vis_JD_12bands.dat", dir);
    rc = rc ? rc : read_real4(path, cv, ncv);
    snprintf(path, sizeof path, "%s/waterCoated_ir_JD_12bands.dat", dir);
    rc = rc ? rc : read_real4(path, ci, nci);
    snprintf(path, sizeof path, "%s/Dust_vis_wolff2010_JD_12bands.dat", dir);
    rc = rc ? rc : read_real4(path, dv, ndv);
    snprintf(path, sizeof path, "%s/Dust_ir_wolff2010_JD_12bands.dat", dir);
    rc = rc ? rc : read_real4(path, di, ndi);
    if (!rc) {
        size_t p = 0, q = 0;
        /* read(60) (qextv_cld(j,i,l), l=1,7) then qscatv, gv, for j, i */
        for (int j = 0; j < ORC_NRATIO; ++j)
            for (int i = 0; i < ORC_NBIN; ++i)
                for (int m = 0; m < 3; ++m) {
                    for (int l = 0; l < ORC_NSPECTV; ++l) a->cld_v[m][j][i][l] = cv[p++];
                    for (int l = 0; l < ORC_NSPECTI; ++l) a->cld_i[m][j][i][l] = ci[q++];
                }
        p = q = 0;
        for (int i = 0; i < ORC_NBIN; ++i)
            for (int m = 0; m < 3; ++m) {
                for (int l = 0; l < ORC_NSPECTV; ++l) a->dst_v[m][i][l] = dv[p++];
                for (int l = 0; l < ORC_NSPECTI; ++l) a->dst_i[m][i][l] = di[q++];
            }
    }
    free(cv);
    free(ci);
    free(dv);
    free(di);
    if (rc) return rc;
    static const float cr[ORC_NRATIO] = {0.1f, 0.2f, 0.25f, 0.3f, 0.35f, 0.4f, 0.45f, 0.5f,
                                         0.55f, 0.6f, 0.65f, 0.7f, 0.8f, 0.9f, 0.99f};
    memcpy(a->cor_ratio, cr, sizeof cr);
    static const double qev1[7] = {1.834, 2.296, 2.672, 2.829, 2.698, 2.452, 2.261};
    static const double qsv1[7] = {1.695, 2.031, 2.583, 2.744, 2.626, 2.225, 1.525};
    static const double gv1[7] = {0.551, 0.640, 0.661, 0.678, 0.690, 0.743, 0.868};
    static const double qei1[5] = {0.008, 0.262, 0.491, 1.017, 0.444};
    static const double qsi1[5] = {0.001, 0.037, 0.122, 0.351, 0.336};
    static const double gi1[5] = {0.004, 0.030, 0.095, 0.214, 0.316};
    for (int n = 0; n < 7; ++n) {
        a->qextv[n] = qev1[n];
        a->qscatv[n] = qsv1[n] >= qev1[n] ? R4(0.99999) * qev1[n] : qsv1[n];
        a->gv[n] = gv1[n];
    }
    for (int n = 0; n < 5; ++n) {
        a->qexti[n] = qei1[n];
        a->qscati[n] = qsi1[n] >= qei1[n] ? R4(0.99999) * qei1[n] : qsi1[n];
        a->gi[n] = gi1[n];
    }
    return 0;
}

/* One column of OPT_DST (cld = 0) or OPT_CLD (cld = 1). */
static void opt_aerosol(const orc_aero *a, int cld, int L, const double *pl, const double *ma,
                        const double *mcor, const double *nb, double *tauref, double *qextref,
                        double *qxv, double *qsv, double *gv, double *qxi, double *qsi, double *gi) {
    const int lev1 = 2 * L + 4;
    const double PIc = 3.1415926535897932, GRAVc = 3.72;
    const double athird = (double)(1.0f / 3.0f);
    const double dpden_dt = R4(2.5E+3), dpden_ice = R4(917.);
    for (int k = 0; k < lev1; ++k) {
        qextref[k] = 1.0;
        tauref[k] = 0.0;
    }
    for (int i = 0; i < ORC_NSPECTV; ++i)
        for (int k = 0; k < lev1; ++k) {
            qxv[i * lev1 + k] = qextref[k];
            qsv[i * lev1 + k] = qextref[k] * R4(0.99);
            gv[i * lev1 + k] = 0.0;
        }
    for (int i = 0; i < ORC_NSPECTI; ++i)
        for (int k = 0; k < lev1; ++k) {
            qxi[i * lev1 + k] = qextref[k];
            qsi[i * lev1 + k] = qextref[k] * R4(0.99);
            gi[i * lev1 + k] = 0.0;
        }
    const double dev = cld ? R4(0.3087) : R4(0.63676);
    const double dev2 = 1.0 / ((double)sqrtf(2.0f) * dev);
    for (int l = 1; l <= L; ++l) {
        double Mo, No, dens;
        int irap = ORC_NRATIO;
        if (!cld) {
            if (!(ma[l - 1] > R4(1.e-8) && nb[l - 1] > 1.0)) continue;
            Mo = ma[l - 1];
            No = nb[l - 1] + 1.0;
            dens = dpden_dt;
        } else {
            if (!(ma[l - 1] + mcor[l - 1] > R4(1.e-7) && nb[l - 1] > 1.0)) continue;
            float mtc = (float)(mcor[l - 1] / dpden_dt / (ma[l - 1] / dpden_ice + mcor[l - 1] / dpden_dt));
            mtc = (float)mgcm_rt_pow((double)mtc, athird);
            for (int i = 1; i <= ORC_NRATIO; ++i) {
                if (mtc < a->cor_ratio[i - 1] && i != 1) {
                    irap = i - 1;
                    break;
                } else if (mtc == a->cor_ratio[i - 1]) {
                    irap = i;
                    break;
                } else if (mtc < a->cor_ratio[i - 1] && i == 1) {
                    irap = 1;
                    break;
                }
            }
            Mo = ma[l - 1] + mcor[l - 1];
            No = nb[l - 1];
            dens = ma[l - 1] / Mo * dpden_ice + mcor[l - 1] / Mo * dpden_dt;
        }
        const double cst = 0.75 / (PIc * dens);
        double Rs = mgcm_rt_pow(Mo / No * cst, athird) * mgcm_rt_exp(-0.5 * (dev * dev));
        const double Ao = No * PIc * (Rs * Rs);
        Rs = Rs * mgcm_rt_exp(1.5 * (dev * dev));
        const double rmax = cld ? R4(100.e-6) : R4(50.e-6);
        Rs = fmin(fmax(Rs, R4(1.e-7)), rmax);
        Rs = 1.0 / Rs;
        double surf[ORC_NBIN];
        for (int i = 0; i < ORC_NBIN; ++i)
            surf[i] = 0.5 * (mgcm_rt_erf(mgcm_rt_ln(a->radb[i + 1] * Rs) * dev2) -
                             mgcm_rt_erf(mgcm_rt_ln(a->radb[i] * Rs) * dev2));
        for (int nn = 1; nn <= 2; ++nn) {
            const int k = 2 * l + 1 + nn; /* 1-based */
            for (int iw = 0; iw < ORC_NSPECTV; ++iw) {
                double x = 0.0, sc = 0.0, g = gv[iw * lev1 + k - 1];
                for (int i = 0; i < ORC_NBIN; ++i) {
                    const double qe = cld ? a->cld_v[0][irap - 1][i][iw] : a->dst_v[0][i][iw];
                    const double qs = cld ? a->cld_v[1][irap - 1][i][iw] : a->dst_v[1][i][iw];
                    const double qg = cld ? a->cld_v[2][irap - 1][i][iw] : a->dst_v[2][i][iw];
                    x = x + surf[i] * qe;
                    sc = sc + surf[i] * qs;
                    g = g + surf[i] * qg;
                }
                qxv[iw * lev1 + k - 1] = x;
                qsv[iw * lev1 + k - 1] = fmin(sc, R4(0.99999) * x);
                gv[iw * lev1 + k - 1] = g;
            }
            for (int iw = 0; iw < ORC_NSPECTI; ++iw) {
                double x = 0.0, sc = 0.0, g = gi[iw * lev1 + k - 1];
                for (int i = 0; i < ORC_NBIN; ++i) {
                    const double qe = cld ? a->cld_i[0][irap - 1][i][iw] : a->dst_i[0][i][iw];
                    const double qs = cld ? a->cld_i[1][irap - 1][i][iw] : a->dst_i[1][i][iw];
                    const double qg = cld ? a->cld_i[2][irap - 1][i][iw] : a->dst_i[2][i][iw];
                    x = x + surf[i] * qe;
                    sc = sc + surf[i] * qs;
                    g = g + surf[i] * qg;
                }
                qxi[iw * lev1 + k - 1] = x;
                qsi[iw * lev1 + k - 1] = fmin(sc, R4(0.99999) * x);
                gi[iw * lev1 + k - 1] = g;
            }
            qextref[k - 1] = qxv[5 * lev1 + k - 1]; /* L_NREFV = 6 */
            const double mass = 100.0 * (pl[k - 1] - pl[k - 2]) / GRAVc;
            tauref[k - 1] = Ao * qextref[k - 1] * mass;
        }
    }
}

static void aerosols_range(const orc_aero *a, const orc_tracers *t, int c0, int c1);

typedef struct {
    const orc_aero *a;
    const orc_tracers *t;
    int c0, c1;
} aero_job;

static void *aero_thread(void *p) {
    const aero_job *j = (const aero_job *)p;
    aerosols_range(j->a, j->t, j->c0, j->c1);
    return NULL;
}

void orc_aerosols_mt(const orc_aero *a, const orc_tracers *t, int nthreads) {
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads > 256) nthreads = 256;
    if (nthreads <= 1 || t->ncol < 2 * nthreads) {
        aerosols_range(a, t, 0, t->ncol);
        return;
    }
    pthread_t th[256];
    aero_job jobs[256];
    for (int i = 0; i < nthreads; ++i) {
        jobs[i].a = a;
        jobs[i].t = t;
        jobs[i].c0 = (int)((long long)t->ncol * i / nthreads);
        jobs[i].c1 = (int)((long long)t->ncol * (i + 1) / nthreads);
        pthread_create(&th[i], NULL, aero_thread, &jobs[i]);
    }
    for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
}

void orc_aerosols(const orc_aero *a, const orc_tracers *t) { aerosols_range(a, t, 0, t->ncol); }

static void aerosols_range(const orc_aero *a, const orc_tracers *t, int c0, int c1) {
    const int L = t->L, lev = 2 * L + 3, lev1 = lev + 1;
    for (int c = c0; c < c1; ++c) {
        const double *pl = t->plev + (size_t)c * lev;
        double *tr = t->tauref + (size_t)c * lev1, *qr = t->qextrefdst + (size_t)c * lev1;
        double *xv = t->qxvdst + (size_t)c * 7 * lev1, *sv = t->qsvdst + (size_t)c * 7 * lev1;
        double *gv = t->gvdst + (size_t)c * 7 * lev1, *xi = t->qxidst + (size_t)c * 5 * lev1;
        double *si = t->qsidst + (size_t)c * 5 * lev1, *gi = t->gidst + (size_t)c * 5 * lev1;
        if (t->active_dust) {
            opt_aerosol(a, 0, L, pl, t->dust_mass + (size_t)c * L, NULL, t->dust_number + (size_t)c * L,
                        tr, qr, xv, sv, gv, xi, si, gi);
            for (int k = 0; k < 3; ++k) tr[k] = 0.0; /* code/comp3.f:602-605 */
        } else { /* code/ini_optdst.f:29-51 with TAUREF from filltaucum */
            for (int k = 0; k < lev1; ++k) {
                qr[k] = a->qextv[5];
                tr[k] = t->tauref_in[(size_t)c * lev1 + k];
            }
            for (int i = 0; i < 7; ++i)
                for (int k = 0; k < lev1; ++k) {
                    xv[i * lev1 + k] = a->qextv[i];
                    sv[i * lev1 + k] = a->qscatv[i];
                    gv[i * lev1 + k] = a->gv[i];
                }
            for (int i = 0; i < 5; ++i)
                for (int k = 0; k < lev1; ++k) {
                    xi[i * lev1 + k] = a->qexti[i];
                    si[i * lev1 + k] = a->qscati[i];
                    gi[i * lev1 + k] = a->gi[i];
                }
        }
        tr[lev1 - 1] = 0.0; /* code/comp3.f:618 */
        if (t->cloudon)
            opt_aerosol(a, 1, L, pl, t->ice_mass + (size_t)c * L, t->ice_core + (size_t)c * L,
                        t->ice_number + (size_t)c * L, t->taurefcld + (size_t)c * lev1,
                        t->qextrefcld + (size_t)c * lev1, t->qxvcld + (size_t)c * 7 * lev1,
                        t->qsvcld + (size_t)c * 7 * lev1, t->gvcld + (size_t)c * 7 * lev1,
                        t->qxicld + (size_t)c * 5 * lev1, t->qsicld + (size_t)c * 5 * lev1,
                        t->gicld + (size_t)c * 5 * lev1);
    }
}

/* ------------------------------------------------------------ column prep */

/* code/dustprofile.f:32-37: REFPR = (5.0*PSF/PTROP)**(1.0/(FLOAT(NPDST)-1.0)),
 * the exponent evaluated in REAL*4; PRDST(1) = PTROP, PRDST(n) = REFPR*PRDST(n-1). */
void orc_dust_grid(double psf, double ptrop, double *prdst) {
    const float e = 1.0f / ((float)ORC_NPDST - 1.0f);
    const double refpr = mgcm_rt_pow(5.0 * psf / ptrop, (double)e);
    prdst[0] = ptrop;
    for (int n = 2; n <= ORC_NPDST; ++n) prdst[n - 1] = refpr * prdst[n - 2];
}

/* code/dustprofile.f:59-114 for one column: the normalising sum of the
 * Conrath profile up to RPTAU, the mixing ratio QRDST per PRDST interval
 * and its running integral TAUDST.  The literals 1. and 1.0 are exact. */
void orc_dust_profile(const double *prdst, double rptau, double conr, double tautot, double *taudst) {
#define PR(n) prdst[(n) - 1]
    double sum = 0.0;
    int n;
    for (n = 2; n <= ORC_NPDST; ++n) {
        if (PR(n) < rptau) {
            const double pave = 0.5 * (PR(n) + PR(n - 1));
            sum = sum + cexp_(conr * (1.0 - (rptau / pave))) * (PR(n) - PR(n - 1));
        }
        if (PR(n) >= rptau) break;
    }
    /* n = NPDST+1 when the loop ran to its end (code/dustprofile.f:70-73) */
    {
        const double pave = 0.5 * (rptau + PR(n - 1));
        sum = sum + cexp_(conr * (1.0 - (rptau / pave))) * (rptau - PR(n - 1));
    }
    const double qrdst0 = tautot / sum;
    double qrdst[ORC_NPDST];
    for (n = 1; n <= ORC_NPDST - 1; ++n) {
        qrdst[n - 1] = 0.0; /* every case below fails only for a NaN RPTAU */
        if (rptau > PR(n + 1)) {
            const double pave = 0.5 * (PR(n + 1) + PR(n));
            qrdst[n - 1] = qrdst0 * cexp_(conr * (1.0 - (rptau / pave)));
        }
        if (rptau <= PR(n + 1) && rptau >= PR(n)) {
            const double pave = 0.5 * (PR(n) + rptau);
            const double pdif1 = rptau - PR(n), pdif2 = PR(n + 1) - rptau;
            qrdst[n - 1] = qrdst0 * (cexp_(conr * (1.0 - (rptau / pave))) * pdif1 + pdif2) / (PR(n + 1) - PR(n));
        }
        if (rptau < PR(n)) qrdst[n - 1] = qrdst0;
    }
    taudst[0] = 0.0;
    for (n = 2; n <= ORC_NPDST; ++n) taudst[n - 1] = taudst[n - 2] + qrdst[n - 2] * (PR(n) - PR(n - 1));
#undef PR
}

/* code/jsrchgt.f90: index of the first SX(j) > TARGET by bisection. */
int orc_jsrchgt(int n, const double *sx, double target) {
    if (n < 1) return 0;
    if (target > sx[n - 1]) return n + 1;
    if (target < sx[0]) return 1;
    int jl = 1, jh = n;
    while (jh - jl > 1) {
        const int jm = (jl + jh) / 2;
        if (target > sx[jm - 1]) jl = jm;
        else jh = jm;
    }
    if (target == sx[jh - 1]) jh = jh + 1;
    return jh;
}

void orc_prep(const orc_prep_batch *b) {
    const int L = b->L, lev = 2 * L + 3, lev1 = lev + 1;
    double prdst[ORC_NPDST], taudst[ORC_NPDST], taucum[2 * ORC_MAXL + 4];
    if (b->prescribed_dust) orc_dust_grid(b->psf, b->ptrop, prdst);
    const double ptrop = b->ptrop;
    const double *sig = b->sigma;
    for (int c = 0; c < b->ncol; ++c) {
        const double p = b->pcol[c];
        const double *tl = b->t + (size_t)c * L;
        double *plev = b->plev + (size_t)c * lev, *tlev = b->tlev + (size_t)c * lev;
        double *pmid = b->pmid + (size_t)c * lev, *tmid = b->tmid + (size_t)c * lev;
        double *qh = b->qh2o + (size_t)c * lev;
        /* PL (code/potemp1.f:95-106) into PLEV (code/fillpt.f90:30-35) */
        plev[0] = ptrop / 2.0;
        plev[1] = ptrop / 2.0;
        for (int k = 3; k <= lev - 1; ++k) plev[k - 1] = ptrop + sig[k - 1] * p;
        plev[lev - 1] = ptrop + p;
        /* TLEV (code/fillpt.f90:37-51): TSTRAT on 1-3, TL(2l+2) on the even
         * levels, log-pressure interpolation on the odd ones, GT at the bottom */
        for (int k = 1; k <= 3; ++k) tlev[k - 1] = b->tstrat[c];
        for (int k = 4; k <= lev - 1; k += 2) tlev[k - 1] = tl[k / 2 - 2];
        for (int k = 5; k <= lev - 2; k += 2)
            tlev[k - 1] = tlev[k] + (tlev[k - 2] - tlev[k]) * mgcm_rt_ln(plev[k - 1] / plev[k]) /
                                        mgcm_rt_ln(plev[k - 2] / plev[k]);
        tlev[lev - 1] = b->gt[c];
        /* TMID/PMID (code/fillpt.f90:53-70) */
        tmid[0] = tlev[1];
        tmid[1] = tlev[1];
        pmid[0] = plev[0];
        pmid[1] = plev[1];
        for (int l = 1; l <= L; ++l) {
            tmid[2 * l] = tlev[2 * l];
            tmid[2 * l + 1] = tlev[2 * l];
            pmid[2 * l] = plev[2 * l];
            pmid[2 * l + 1] = plev[2 * l];
        }
        tmid[lev - 1] = tlev[lev - 1];
        pmid[lev - 1] = plev[lev - 1];
        /* QH2O (code/comp3.f:576-589) */
        qh[0] = qh[1] = qh[2] = 0.0;
        for (int l = 1; l <= L; ++l) {
            const int k = 2 * l + 2;
            qh[k - 1] = b->active_water ? b->mwratio * b->vapour[(size_t)c * L + l - 1] : R4(1.0E-7);
            qh[k] = qh[k - 1];
        }
        if (!b->prescribed_dust) continue;
        /* TAUREF (code/filltaucum.f:39-55, code/comp3.f:618) */
        double *tr = b->tauref + (size_t)c * lev1;
        orc_dust_profile(prdst, b->rptau, b->conr[c], b->tautot[c], taudst);
        for (int k = 1; k <= 3; ++k) {
            taucum[k - 1] = 0.0;
            tr[k - 1] = 0.0;
        }
        for (int k = 4; k <= lev; ++k) {
            const double pstar = p * sig[k - 1] + ptrop;
            const double pstar1 = pstar > prdst[0] ? pstar : prdst[0];
            int nstar = orc_jsrchgt(ORC_NPDST - 1, prdst, pstar1) - 1;
            if (nstar > ORC_NPDST - 1) nstar = ORC_NPDST - 1;
            if (nstar < 1) nstar = 1; /* PSTAR1 >= PRDST(1) gives nstar >= 1 (kept for NaN inputs) */
            taucum[k - 1] = taudst[nstar - 1] + (pstar1 - prdst[nstar - 1]) * (taudst[nstar] - taudst[nstar - 1]) /
                                                    (prdst[nstar] - prdst[nstar - 1]);
            tr[k - 1] = taucum[k - 1] - taucum[k - 2];
        }
        tr[lev1 - 1] = 0.0;
    }
}

/* Per level of every column: the TPINDEX bins and weights (levels 2..LEV,
 * as OPTCV/OPTCI call it, code/optcv.f90:103-108, code/optci.f90:113-118;
 * zeros at level 1) and the Planck index of TLEV (levels 1..LEV).  Outputs
 * [ncol][LEV]; lcoef [ncol][LEV][4]. */
void orc_bins_batch(const orc_tables *t, const orc_batch *b, int *mt, int *mp, int *nh2o, int *npl,
                    double *wratio, double *lcoef) {
    const int LEV = 2 * b->L + 3;
    for (int c = 0; c < b->ncol; c++)
        for (int k = 1; k <= LEV; k++) {
            const size_t i = (size_t)c * LEV + k - 1;
            npl[i] = orc_planck_index(b->tlev[i]);
            if (k == 1) {
                mt[i] = mp[i] = nh2o[i] = 0;
                wratio[i] = 0.0;
                for (int q = 0; q < 4; q++) lcoef[i * 4 + q] = 0.0;
                continue;
            }
            orc_tpindex(t, b->pmid[i], b->tmid[i], b->qh2o[i], &lcoef[i * 4], &mt[i], &mp[i], &nh2o[i],
                        &wratio[i]);
        }
}
