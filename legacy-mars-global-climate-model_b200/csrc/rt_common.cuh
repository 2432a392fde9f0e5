// Device-side definitions shared by the radiation kernels.
#pragma once
#include <cstddef>
#include <cstdint>

namespace mgcm {

constexpr int D_NV = 7, D_NI = 5, D_NG = 17, D_NGK = 16, D_NT = 7, D_NP = 51, D_NH = 10;
constexpr int D_NPLANCK = 8501;
constexpr int D_MAXL = 99;
constexpr int D_MAXNL = D_MAXL + 1;        // NLAYRAD
constexpr int D_MAXLEV = 2 * D_MAXL + 3;   // L_LEVELS
constexpr int NSYS_V = D_NV * D_NG;        // 119 visible systems per column
constexpr int NSYS_I = D_NI * D_NG;        // 85 IR systems per column
constexpr int NSYS = NSYS_V + NSYS_I;      // 204
constexpr int NREFV_IDX = 5;               // L_NREFV = 6 (0.67 um band), 0-based

// Screening groups of a column: warp-sized runs of systems that never mix the
// families -- visible 0-31, 32-63, 64-95, 96-118; IR 119-150, 151-182, 183-203.
constexpr int SCREEN_GROUPS = 7, SCREEN_GROUPS_V = 4;
__host__ __device__ constexpr int group_first(int w) {
    return w < SCREEN_GROUPS_V ? 32 * w : NSYS_V + 32 * (w - SCREEN_GROUPS_V);
}
__host__ __device__ constexpr int group_end(int w) {
    return w < SCREEN_GROUPS_V ? (32 * (w + 1) < NSYS_V ? 32 * (w + 1) : NSYS_V)
                               : (NSYS_V + 32 * (w - SCREEN_GROUPS_V + 1) < NSYS
                                      ? NSYS_V + 32 * (w - SCREEN_GROUPS_V + 1)
                                      : NSYS);
}

// Layers per lane of the four-lane solvers for a largest NL (0: NL > 52,
// the one-thread-per-system solvers run).
__host__ __device__ constexpr int quad_r_for(int nl) {
    return nl <= 28 ? 7 : (nl <= 40 ? 10 : (nl <= 52 ? 13 : 0));
}

// device status bits (OR-ed into the status word)
// Flux rows of the pipeline's solves, in blocks of 32 consecutive list
// positions: within a block, value k (of 2 max_nl: upward then downward
// midpoint fluxes) of the 32 systems is contiguous, so a warp of solver
// threads stores one 256-byte segment per value, and a system's row stays
// inside its block's 512 max_nl bytes.  Value k of position p is at
// row_base(p, max_nl) + 32 k; scalar q (of 4) at sc_base(p) + 32 q.
constexpr int ROW_BLK = 32;
__host__ __device__ inline size_t row_base(size_t p, int max_nl) {
    return (p / ROW_BLK) * (size_t)(2 * ROW_BLK * max_nl) + p % ROW_BLK;
}
__host__ __device__ inline size_t sc_base(size_t p) { return (p / ROW_BLK) * (size_t)(4 * ROW_BLK) + p % ROW_BLK; }
// List positions rounded up to whole blocks (row and scalar buffer sizes).
__host__ __device__ inline size_t row_slots(size_t n) { return (n + ROW_BLK - 1) / ROW_BLK * ROW_BLK; }

constexpr uint32_t ST_PLANCK_RANGE = 1u;   // a Planck index left 1..8501 (clamped)
constexpr uint32_t ST_NONFINITE = 2u;      // validation: NaN/Inf or p <= 0 in an input
constexpr uint32_t ST_TEMP = 4u;           // validation: T outside [50,900)
constexpr uint32_t ST_BADL = 8u;           // a segment with L outside 1..99

// Constant tables (radcommon_h and friends).
struct RtConst {
    double tauray[D_NV];
    double fzerov[D_NV];
    double fzeroi[D_NI];
    double gweight[D_NG];
    double dwni[D_NI];
    double pfgasref[D_NP];
    double plimit[D_NP];     // bin search limits: log10(p) <= pfgasref[n] <=> p <= plimit[n]
    double wrefh2o[D_NH];
};

// Pointers of one batch (one vertical grid) on the device.
struct SegDev {
    int ncol, L;
    int col0;                 // first global column index of this segment (multi-grid)
    double ptrop;
    const double *sigma, *sol;
    const double *plev, *tlev, *pmid, *tmid, *qh2o;
    const double *tauref, *qextrefdst, *taurefcld, *qextrefcld;
    // Prescribed dust (INI_OPTDST): when set, these 36 band properties --
    // QEXTV[7], QSCATV[7], GV[7], QEXTI[5], QSCATI[5], GI[5] -- stand for the
    // per-level dust arrays (the same values at every level), QEXTREFDST is
    // QEXTV(L_NREFV) and TAUREF(L_LEVELS+1) is 0 (code/ini_optdst.f:29-51,
    // code/comp3.f:618); the qx/qs/g dust pointers are then unused.
    const double *dust_band;
    const double *qxvdst, *qsvdst, *gvdst, *qxidst, *qsidst, *gidst;
    const double *qxvcld, *qsvcld, *gvcld, *qxicld, *qsicld, *gicld;
    const double *acosz, *als, *albi, *pcol;
    double *detau, *cumtauv;
    double *fmnetv, *fluxupv, *fluxdnv, *fmneti, *fluxupi, *fluxdni;
    double *suntot, *irtotal, *qrad;
    double *nfluxtopv, *nfluxtopi, *diffvt, *dnvflux, *dndiffv, *dnirflux, *fluxsurf;
};

constexpr int MAX_SEGS = 64;

struct SegTable {
    int nseg;
    int total_cols;
    SegDev seg[MAX_SEGS];
};

// Device-resident tables.
struct TabDev {
    const double *kv;        // [7][7][51][10][16] FP64, Gauss point fastest
    const double *ki;        // [5][7][51][10][16]
    const float *kvf;        // FP32 copies for the mixed path
    const float *kif;
    const double *planck;    // [8501][5]
};

}  // namespace mgcm
