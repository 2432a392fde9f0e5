// Per-column staging shared by the radiation kernels: level bins (tpindex),
// per-band aerosol/Rayleigh opacities and the per-layer scattering sums.
#pragma once
#include "rt_common.cuh"
#include "../../include/mgcm_rt_math.h"

namespace mgcm {

#define R4(x) ((double)(float)(x))

__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// Locate the segment (grid) that owns global column g.
__device__ __forceinline__ int find_seg(const SegTable *__restrict__ st, int g) {
    int s = 0;
    while (s + 1 < st->nseg && st->seg[s + 1].col0 <= g) ++s;
    return s;
}

// What every system's k-table gather needs of level k (tpindex and U), in
// one 64-byte record so a thread fetches it with four 16-byte loads: the
// bilinear weights LCOEF(1..4), WRATIO, U = Cmk*DPR, the element offset of
// the (MT, MP, NH2O) corner within a band's table and the step to the
// NH2O+1 row (0 where NH2O = 10, whose WRATIO is 0).
struct alignas(16) KLevel {
    double lk[4];
    double wr, u;
    int kofs, kdh;
    int pad[2];
};
static_assert(sizeof(KLevel) == 64, "KLevel is one 64-byte record");

// Shared-memory layout of one column; sized by the launch's largest NL.
struct ColSmem {
    // per level (1-based k = 1..LEV+1)
    KLevel *klev;
    double *dpr;
    double *tref_v, *tref_i, *tref_c;   // TAUREF/QEXTREF (vis, IR), TAUREFCLD/QEXTREFCLD
    // per level and band
    double *trayaer;                    // [k][7] visible TRAY+TAEROS+TCLOUD
    double *taer_i, *tcld_i;            // [k][5] IR TAEROS, TCLOUD
    // per layer and band
    double *cosb_v, *wnum_v;            // [l][7]
    double *cbs_v;                      // [l][7] COSBV/(1+COSBV), the delta-Eddington COSBAR
    double *cosb_i, *wnum_i;            // [l][5]
    double *b0_i, *pdif_i;              // [l][5] Planck B0 and B1*DTAU numerator
    double *bsurf_i, *pltop_i;          // [5]
    // reduction staging
    double *fmp, *fmm;                  // [sys][l]
    double *sc0, *sc1, *sc2;            // [sys] FLUXUP, FLUXDN, DIFFV (vis) / FTOPUP (IR)
    unsigned char *skip;                // [sys] 0 = solved, 1 = TLIMIT skip, 2 = no work
    int *meta;                          // [2*SCREEN_GROUPS] list base/count of kept systems per group
    double *fmnet_v, *fmnet_i;          // [l] reduced net fluxes for the divergences
    double *misc;                       // [4] NFLUXTOPV, NFLUXTOPI
    int day;
};

// Largest dynamic shared memory a CTA may use (227 KB opt-in on sm_100).
constexpr size_t SMEM_CAP = 227 * 1024;

// Bytes of the per-system flux staging (FMIDP/FMIDM for every system).
__host__ __device__ inline size_t red_bytes(int nl) { return 2 * (size_t)NSYS * nl * sizeof(double); }

// Shared memory of one column.  With red_in_smem false the flux staging
// lives in a global scratch slab per CTA instead (large L).
__host__ __device__ inline size_t col_smem_bytes(int nl, bool red_in_smem = true) {
    const size_t lev1 = 2 * nl + 3;   // 1-based k up to LEV+1 = 2L+4 = 2NL+2
    size_t b = 0;
    b += (lev1 + 1) * sizeof(KLevel);
    b += (lev1 + 1) * (1 + 3) * sizeof(double);
    b += (lev1 + 1) * (D_NV + 2 * D_NI) * sizeof(double);
    b += (nl + 1) * (3 * D_NV + 4 * D_NI) * sizeof(double);
    b += 2 * D_NI * sizeof(double);
    if (red_in_smem) b += red_bytes(nl);
    b += 3 * NSYS * sizeof(double);
    b += 2 * (nl + 1) * sizeof(double) + 4 * sizeof(double);
    b += NSYS + 16 + 2 * SCREEN_GROUPS * sizeof(int) + 16;
    return b;
}

__device__ inline ColSmem carve_smem(unsigned char *base, int nl, double *red_global = nullptr,
                                     bool with_red = true) {
    ColSmem s;
    const int lev1 = 2 * nl + 3;
    s.klev = reinterpret_cast<KLevel *>(base);   // base is 16-byte aligned
    double *d = reinterpret_cast<double *>(base + (size_t)(lev1 + 1) * sizeof(KLevel));
    auto take = [&](size_t n) { double *p = d; d += n; return p; };
    s.dpr = take(lev1 + 1);
    s.tref_v = take(lev1 + 1);
    s.tref_i = take(lev1 + 1);
    s.tref_c = take(lev1 + 1);
    s.trayaer = take((lev1 + 1) * D_NV);
    s.taer_i = take((lev1 + 1) * D_NI);
    s.tcld_i = take((lev1 + 1) * D_NI);
    s.cosb_v = take((nl + 1) * D_NV);
    s.wnum_v = take((nl + 1) * D_NV);
    s.cbs_v = take((nl + 1) * D_NV);
    s.cosb_i = take((nl + 1) * D_NI);
    s.wnum_i = take((nl + 1) * D_NI);
    s.b0_i = take((nl + 1) * D_NI);
    s.pdif_i = take((nl + 1) * D_NI);
    s.bsurf_i = take(D_NI);
    s.pltop_i = take(D_NI);
    if (!with_red) {
        s.fmp = s.fmm = nullptr;
    } else if (red_global) {
        s.fmp = red_global;
        s.fmm = red_global + (size_t)NSYS * nl;
    } else {
        s.fmp = take((size_t)NSYS * nl);
        s.fmm = take((size_t)NSYS * nl);
    }
    s.sc0 = take(NSYS);
    s.sc1 = take(NSYS);
    s.sc2 = take(NSYS);
    s.fmnet_v = take(nl + 1);
    s.fmnet_i = take(nl + 1);
    s.misc = take(4);
    int *ip = reinterpret_cast<int *>(d);
    s.skip = reinterpret_cast<unsigned char *>(ip);
    s.meta = reinterpret_cast<int *>(((reinterpret_cast<uintptr_t>(s.skip + NSYS) + 15) / 16) * 16);
    s.day = 0;
    return s;
}

// Planck table index INT(T*10-499) (code/sfluxi.f90:54-55, code/gfluxi.f90:73-74,86-87),
// formed without contraction; clamped to the table with a status flag.
__device__ __forceinline__ int planck_index(double t, uint32_t *status) {
    const double x = __dsub_rn(__dmul_rn(t, 10.0), 499.0);
    int it = (x > -2.0e9 && x < 2.0e9) ? __double2int_rz(x) : 0;
    if (it < 1 || it > D_NPLANCK) {
        atomicOr(status, ST_PLANCK_RANGE);
        it = it < 1 ? 1 : D_NPLANCK;
    }
    return it;
}

// tpindex (code/tpindex.f90:72-134).  The log10 bin search is done on the
// pressure against host-computed limits so bins agree bit-for-bit with the
// host libm; the weight T uses mgcm_rt_log10, bit-identical to the oracle's.
__device__ __forceinline__ void tpindex_dev(const RtConst &c, double pw, double tw, double qh2o,
                                            int &mt, int &mp, int &nh, double &wratio,
                                            double lk[4]) {
    // temperature: TREF = 50,100,..,350
    if (tw <= 50.0) {
        mt = 1;
    } else {
        mt = D_NT - 1;
#pragma unroll
        for (int n = 1; n <= D_NT - 1; ++n)
            if (tw > 50.0 * n && tw <= 50.0 * (n + 1)) { mt = n; break; }
    }
    const double uu = (tw - 50.0 * mt) / (50.0 * (mt + 1) - 50.0 * mt);
    mp = D_NP - 1;
    for (int n = 2; n <= D_NP - 1; ++n)
        if (pw <= c.plimit[n - 1]) { mp = n - 1; break; }
    const double pwl = mgcm_rt_log10(pw);
    const double tt = (pwl - c.pfgasref[mp - 1]) / (c.pfgasref[mp] - c.pfgasref[mp - 1]);
    lk[0] = (1.0 - tt) * (1.0 - uu);
    lk[1] = tt * (1.0 - uu);
    lk[2] = tt * uu;
    lk[3] = (1.0 - tt) * uu;
    wratio = 0.0;
    nh = 1;
    if (qh2o <= c.wrefh2o[0]) {
        nh = 1;
    } else if (qh2o >= c.wrefh2o[D_NH - 1]) {
        nh = D_NH;
    } else {
        for (int n = 2; n <= D_NH; ++n)
            if (qh2o >= c.wrefh2o[n - 2] && qh2o < c.wrefh2o[n - 1]) {
                nh = n - 1;
                wratio = (qh2o - c.wrefh2o[n - 2]) / (c.wrefh2o[n - 1] - c.wrefh2o[n - 2]);
                break;
            }
    }
}

}  // namespace mgcm
