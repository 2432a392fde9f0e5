// Host set-up of the radiation tables, restating the reference RADSETUP chain:
//   code/setspv.f90:67-105  visible bands, SOLARF (REAL*4 literals), TAURAY
//   code/setspi.f90:70-105  IR bands and the Planck table (12-point Gauss-Legendre)
//   code/setrad.f90:112-130  PGASREF (REAL*4 literals) and TGASREF
//   code/laginterp.f90:71-236 log10 of the k records, 4-point Lagrange onto 51 log-p
//                            points, 10**ans; code/lagrange.f90:17-31
// Compiled without FMA contraction so the tables match the reference's x86-64 build.
#include "tables.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace mgcm {

namespace {

inline double r4(double x) { return static_cast<double>(static_cast<float>(x)); }

int read_rec(std::FILE *f, double *dst, size_t n) {
    int32_t a = 0, b = 0;
    if (std::fread(&a, 4, 1, f) != 1) return -1;
    if (static_cast<size_t>(a) != n * sizeof(double)) return -2;
    if (std::fread(dst, sizeof(double), n, f) != n) return -3;
    if (std::fread(&b, 4, 1, f) != 1 || a != b) return -4;
    return 0;
}

// 4-point Lagrange polynomial through (xi, yi) evaluated at x, term order of lagrange.f90.
double lag4(double x, const double *xi, const double *yi) {
    const double f1 = x - xi[0], f2 = x - xi[1], f3 = x - xi[2], f4 = x - xi[3];
    return f2 * f3 * f4 * yi[0] / ((xi[0] - xi[1]) * (xi[0] - xi[2]) * (xi[0] - xi[3])) +
           f1 * f3 * f4 * yi[1] / ((xi[1] - xi[0]) * (xi[1] - xi[2]) * (xi[1] - xi[3])) +
           f1 * f2 * f4 * yi[2] / ((xi[2] - xi[0]) * (xi[2] - xi[1]) * (xi[2] - xi[3])) +
           f1 * f2 * f3 * yi[3] / ((xi[3] - xi[0]) * (xi[3] - xi[1]) * (xi[3] - xi[2]));
}

// Interpolates one family (nb bands) from 11 to 51 pressures in log10 space.
void interp_family(const std::vector<double> &logk, std::vector<double> &out, int nb,
                   const double *lp11, const double *lp51) {
    auto in = [&](int nt, int np, int nh, int nw, int ng) {
        return logk[nt + NT * (np + NP11 * (nh + NH * (nw + nb * ng)))];
    };
    out.assign(static_cast<size_t>(NT) * NP * NH * nb * NG, 0.0);
    auto at = [&](int nt, int np, int nh, int nw, int ng) -> double & {
        return out[nt + NT * (np + NP * (nh + NH * (nw + nb * ng)))];
    };
    double xi[4], yi[4];
    for (int ng = 0; ng < NG; ++ng)
        for (int nw = 0; nw < nb; ++nw)
            for (int nh = 0; nh < NH; ++nh)
                for (int nt = 0; nt < NT; ++nt) {
                    // source interval n (0-based 0..9) -> stencil start
                    for (int n = 0; n < NP11 - 1; ++n) {
                        int s = n == 0 ? 0 : (n == NP11 - 2 ? NP11 - 4 : n - 1);
                        for (int q = 0; q < 4; ++q) {
                            xi[q] = lp11[s + q];
                            yi[q] = in(nt, s + q, nh, nw, ng);
                        }
                        for (int m = 0; m < 5; ++m) {
                            const int i = n * 5 + m;
                            at(nt, i, nh, nw, ng) = std::pow(10.0, lag4(lp51[i], xi, yi));
                        }
                    }
                    at(nt, NP - 1, nh, nw, ng) = std::pow(10.0, in(nt, NP11 - 1, nh, nw, ng));
                }
}

}  // namespace

int read_ktables(const std::string &dir, std::vector<double> &co2v8, double fzerov[NV],
                 std::vector<double> &co2i8, double fzeroi[NI]) {
    co2v8.assign(static_cast<size_t>(NT) * NP11 * NH * NV * NG, 0.0);
    co2i8.assign(static_cast<size_t>(NT) * NP11 * NH * NI * NG, 0.0);
    const std::string pv = dir + "/CO2H2O_V_12_95_INTEL", pi = dir + "/CO2H2O_IR_12_95_INTEL";
    std::FILE *f = std::fopen(pv.c_str(), "rb");
    if (!f) return -1;
    int rc = read_rec(f, co2v8.data(), co2v8.size());
    if (!rc) rc = read_rec(f, fzerov, NV);
    std::fclose(f);
    if (rc) return -2;
    f = std::fopen(pi.c_str(), "rb");
    if (!f) return -1;
    rc = read_rec(f, co2i8.data(), co2i8.size());
    if (!rc) rc = read_rec(f, fzeroi, NI);
    std::fclose(f);
    return rc ? -2 : 0;
}

void build_tables(HostTables &t, const std::vector<double> &co2v8, const double fzerov[NV],
                  const std::vector<double> &co2i8, const double fzeroi[NI]) {
    const double PI = 3.1415926535897932, GRAV = 3.72, SCALEP = 100.0;
    // visible bands (setspv.f90:113-151)
    const double bwnv[NV + 1] = {2222.22, 3087.37, 4030.63, 5370.57,
                                 7651.11, 12500.00, 25000.00, 41666.67};
    const double solar[NV] = {12.7, 24.2, 54.6, 145.9, 354.9, 657.5, 106.3};
    for (int m = 0; m < NV; ++m) {
        const double wno = 0.5 * (bwnv[m + 1] + bwnv[m]);
        t.dwnv[m] = bwnv[m + 1] - bwnv[m];
        const double wl = 1.0e+4 / wno;
        const double wl2 = wl * wl, wl4 = wl2 * wl2;
        t.solarf[m] = r4(solar[m]);
        t.tauray[m] = (r4(8.7) / GRAV) * (r4(1.527) * (1.0 + r4(0.013) / wl2) / wl4) * SCALEP / 9.423e+6;
    }
    // IR bands and Planck integrals (setspi.f90:224-259)
    const double bwni[NI + 1] = {10.000, 166.667, 416.667, 833.333, 1250.000, 2222.222};
    const double gx[12] = {-0.981560634246719, -0.904117256370475, -0.769902674194305,
                           -0.587317954286617, -0.367831498998180, -0.125233408511469,
                           0.125233408511469,  0.367831498998180,  0.587317954286617,
                           0.769902674194305,  0.904117256370475,  0.981560634246719};
    const double gw[12] = {0.047175336386512, 0.106939325995318, 0.160078328543346,
                           0.203167426723066, 0.233492536538355, 0.249147045813403,
                           0.249147045813403, 0.233492536538355, 0.203167426723066,
                           0.160078328543346, 0.106939325995318, 0.047175336386512};
    const double c1 = 3.741832e-16, c2 = 1.438786e-2;
    t.planckir.assign(static_cast<size_t>(NI) * NPLANCK, 0.0);
    for (int nw = 0; nw < NI; ++nw) {
        t.dwni[nw] = bwni[nw + 1] - bwni[nw];
        const double a = 1.0e-2 / bwni[nw + 1], b = 1.0e-2 / bwni[nw];
        const double bpa = (b + a) / 2.0, bma = (b - a) / 2.0;
        for (int it = 0; it < NPLANCK; ++it) {
            const double T = static_cast<double>(it + 500) / 1.0e+1;
            double ans = 0.0;
            for (int m = 0; m < 12; ++m) {
                const double y = bma * gx[m] + bpa;
                const double y2 = y * y;
                const double y5 = y2 * (y * y2);  // gfortran's y**5 addition chain
                ans = ans + gw[m] * c1 / (y5 * (std::exp(c2 / (y * T)) - 1.0));
            }
            t.planckir[static_cast<size_t>(it) * NI + nw] = ans * bma / (PI * t.dwni[nw]);
        }
    }
    // reference grids (setrad.f90:112-130, laginterp.f90:191-210)
    const double pg[NP11] = {1.0e-6, 1.0e-5, 1.0e-4, 1.0e-3, 1.0e-2, 1.0e-1,
                             1.0,    1.0e+1, 1.0e+2, 1.0e+3, 1.0e+4};
    double lp11[NP11];
    for (int n = 0; n < NP11; ++n) {
        t.pgasref[n] = r4(pg[n]);
        lp11[n] = std::log10(t.pgasref[n]);
    }
    static const char *pin[NP] = {
        "-6.0", "-5.8", "-5.6", "-5.4", "-5.2", "-5.0", "-4.8", "-4.6", "-4.4", "-4.2", "-4.0",
        "-3.8", "-3.6", "-3.4", "-3.2", "-3.0", "-2.8", "-2.6", "-2.4", "-2.2", "-2.0", "-1.8",
        "-1.6", "-1.4", "-1.2", "-1.0", "-0.8", "-0.6", "-0.4", "-0.2", "0.0",  "0.2",  "0.4",
        "0.6",  "0.8",  "1.0",  "1.2",  "1.4",  "1.6",  "1.8",  "2.0",  "2.2",  "2.4",  "2.6",
        "2.8",  "3.0",  "3.2",  "3.4",  "3.6",  "3.8",  "4.0"};
    for (int n = 0; n < NP; ++n) t.pfgasref[n] = std::strtod(pin[n], nullptr);
    for (int n = 0; n < NT; ++n) t.tgasref[n] = 50.0 * (n + 1);
    // k tables: log10 with the -200 floor, then the Lagrange interpolation
    std::vector<double> lv(co2v8.size()), li(co2i8.size());
    for (size_t q = 0; q < co2v8.size(); ++q) lv[q] = co2v8[q] > 1.0e-200 ? std::log10(co2v8[q]) : -200.0;
    for (size_t q = 0; q < co2i8.size(); ++q) li[q] = co2i8[q] > 1.0e-200 ? std::log10(co2i8[q]) : -200.0;
    interp_family(lv, t.co2v, NV, lp11, t.pfgasref);
    interp_family(li, t.co2i, NI, lp11, t.pfgasref);
    std::memcpy(t.fzerov, fzerov, sizeof(double) * NV);
    std::memcpy(t.fzeroi, fzeroi, sizeof(double) * NI);
    // radcommon_h parameters (modules.f90:335-353)
    const double gwt[NG] = {4.8083554740e-02, 1.0563099137e-01, 1.4901065679e-01, 1.7227479710e-01,
                            1.7227479710e-01, 1.4901065679e-01, 1.0563099137e-01, 4.8083554740e-02,
                            2.5307134073e-03, 5.5595258613e-03, 7.8426661469e-03, 9.0670945845e-03,
                            9.0670945845e-03, 7.8426661469e-03, 5.5595258613e-03, 2.5307134073e-03,
                            0.0};
    std::memcpy(t.gweight, gwt, sizeof(gwt));
    const double wr[NH] = {1.0e-7, 1.0e-6, 1.0e-5, 1.0e-4, 1.0e-3, 1.0e-2, 1.0e-1, 2.0e-1, 3.0e-1, 4.0e-1};
    std::memcpy(t.wrefh2o, wr, sizeof(wr));
    // Pressure limits for the tpindex bin search: plimit[n] = max{p : log10(p) <= pfgasref[n]}.
    for (int n = 0; n < NP; ++n) {
        const double target = t.pfgasref[n];
        double lo = std::pow(10.0, target) * 0.5, hi = std::pow(10.0, target) * 2.0;
        // bisection on the bit pattern (positive doubles order like their integers)
        uint64_t a, b;
        std::memcpy(&a, &lo, 8);
        std::memcpy(&b, &hi, 8);
        while (b - a > 1) {
            const uint64_t m = a + (b - a) / 2;
            double pm;
            std::memcpy(&pm, &m, 8);
            if (std::log10(pm) <= target) a = m; else b = m;
        }
        std::memcpy(&t.plimit[n], &a, 8);
    }
}

int load_tables(const std::string &dir, HostTables &t) {
    std::vector<double> v8, i8;
    double fv[NV], fi[NI];
    const int rc = read_ktables(dir, v8, fv, i8, fi);
    if (rc) return rc;
    build_tables(t, v8, fv, i8, fi);
    return 0;
}

// Whitespace-separated REAL*4 values of a formatted Mie table file, as
// code/initcld.f:161-178 reads them.
static int read_real4(const std::string &path, std::vector<double> &v, size_t n) {
    FILE *f = std::fopen(path.c_str(), "r");
    if (!f) return -1;
    v.clear();
    char tok[64];
    while (v.size() < n && std::fscanf(f, "%63s", tok) == 1) v.push_back((double)std::strtof(tok, nullptr));
    std::fclose(f);
    return v.size() == n ? 0 : -2;
}

int load_aerosol_tables(const std::string &dir, AerosolTables &a) {
    const auto R4 = [](double x) { return (double)(float)x; };
    // size bins of the radiative transfer (code/initcld.f:141-156); the
    // literals are REAL*4, ATHIRD = REAL*4 (1./3.)
    const double athird = (double)(1.0f / 3.0f);
    double rad[NBIN_RT];
    rad[0] = R4(1.e-7);
    rad[NBIN_RT - 1] = R4(50.e-6);
    a.radb[0] = R4(0.0001e-6);
    a.radb[NBIN_RT] = R4(1.e-2);
    double vrat = std::log(rad[NBIN_RT - 1] / rad[0]) / (double)(float)(NBIN_RT - 1) * 3.0;
    vrat = std::exp(vrat);
    for (int i = 0; i < NBIN_RT - 1; ++i) {
        rad[i + 1] = rad[i] * std::pow(vrat, athird);
        a.radb[i + 1] = std::pow((2.0 * vrat) / (vrat + 1.0), athird) * rad[i];
    }
    std::vector<double> cv, ci, dv, di;
    int rc = read_real4(dir + "/waterCoated_vis_JD_12bands.dat", cv, (size_t)NRATIO * NBIN_RT * 3 * NV);
    if (!rc) rc = read_real4(dir + "/waterCoated_ir_JD_12bands.dat", ci, (size_t)NRATIO * NBIN_RT * 3 * NI);
    if (!rc) rc = read_real4(dir + "/Dust_vis_wolff2010_JD_12bands.dat", dv, (size_t)NBIN_RT * 3 * NV);
    if (!rc) rc = read_real4(dir + "/Dust_ir_wolff2010_JD_12bands.dat", di, (size_t)NBIN_RT * 3 * NI);
    if (rc) return rc;
    size_t p = 0, q = 0;
    for (int j = 0; j < NRATIO; ++j)
        for (int i = 0; i < NBIN_RT; ++i)
            for (int m = 0; m < 3; ++m) {
                for (int l = 0; l < NV; ++l) a.cld_v[m][j][i][l] = cv[p++];
                for (int l = 0; l < NI; ++l) a.cld_i[m][j][i][l] = ci[q++];
            }
    p = q = 0;
    for (int i = 0; i < NBIN_RT; ++i)
        for (int m = 0; m < 3; ++m) {
            for (int l = 0; l < NV; ++l) a.dst_v[m][i][l] = dv[p++];
            for (int l = 0; l < NI; ++l) a.dst_i[m][i][l] = di[q++];
        }
    const float cr[NRATIO] = {0.1f, 0.2f, 0.25f, 0.3f, 0.35f, 0.4f, 0.45f, 0.5f,
                              0.55f, 0.6f, 0.65f, 0.7f, 0.8f, 0.9f, 0.99f};
    for (int j = 0; j < NRATIO; ++j) a.cor_ratio[j] = (double)cr[j];
    // prescribed dust band properties (code/setrad.f90:73-105,132-155)
    const double qev1[NV] = {1.834, 2.296, 2.672, 2.829, 2.698, 2.452, 2.261};
    const double qsv1[NV] = {1.695, 2.031, 2.583, 2.744, 2.626, 2.225, 1.525};
    const double gv1[NV] = {0.551, 0.640, 0.661, 0.678, 0.690, 0.743, 0.868};
    const double qei1[NI] = {0.008, 0.262, 0.491, 1.017, 0.444};
    const double qsi1[NI] = {0.001, 0.037, 0.122, 0.351, 0.336};
    const double gi1[NI] = {0.004, 0.030, 0.095, 0.214, 0.316};
    for (int n = 0; n < NV; ++n) {
        a.qextv[n] = qev1[n];
        a.qscatv[n] = qsv1[n] >= qev1[n] ? R4(0.99999) * qev1[n] : qsv1[n];
        a.gv[n] = gv1[n];
    }
    for (int n = 0; n < NI; ++n) {
        a.qexti[n] = qei1[n];
        a.qscati[n] = qsi1[n] >= qei1[n] ? R4(0.99999) * qei1[n] : qsi1[n];
        a.gi[n] = gi1[n];
    }
    return 0;
}

void gauss_fastest(const HostTables &t, std::vector<double> &kv, std::vector<double> &ki) {
    auto pack = [](const std::vector<double> &src, int nb, std::vector<double> &dst) {
        dst.assign(static_cast<size_t>(nb) * NT * NP * NH * NGK, 0.0);
        for (int nw = 0; nw < nb; ++nw)
            for (int nt = 0; nt < NT; ++nt)
                for (int np = 0; np < NP; ++np)
                    for (int nh = 0; nh < NH; ++nh)
                        for (int ng = 0; ng < NGK; ++ng)
                            dst[((((static_cast<size_t>(nw) * NT + nt) * NP + np) * NH + nh) * NGK) + ng] =
                                src[nt + NT * (np + NP * (nh + NH * (nw + nb * ng)))];
    };
    pack(t.co2v, NV, kv);
    pack(t.co2i, NI, ki);
}

}  // namespace mgcm
