// Device aerosol optics (rt_aerosol.cu): constants and the batch view.
#pragma once
#include <cstddef>

namespace mgcm {

constexpr int AERO_NV = 7, AERO_NI = 5, AERO_NBIN = 20, AERO_NRATIO = 15;
// Mie tables on the device, one array: dust [3][bin][7] then [3][bin][5];
// water ice [3][ratio][bin][7] then [3][ratio][bin][5]; quantity order
// QEXT, QSCAT, G.
constexpr int AERO_DST_SIZE = 3 * AERO_NBIN * (AERO_NV + AERO_NI);
constexpr int AERO_MIE_SIZE = AERO_DST_SIZE + 3 * AERO_NRATIO * AERO_NBIN * (AERO_NV + AERO_NI);

struct AeroConst {
    double radb[AERO_NBIN + 1];    // radb_rt (code/initcld.f:141-156)
    float cor_ratio[AERO_NRATIO];  // REAL*4 core ratios (cldcommon_h)
    double qextv[AERO_NV], qscatv[AERO_NV], gv[AERO_NV];   // prescribed dust (setrad)
    double qexti[AERO_NI], qscati[AERO_NI], gi[AERO_NI];
};

// One batch: tracers in ([ncol][L]), full per-level arrays out (layout of
// mgcm_rt_batch_in).  Device pointers.
struct AeroSeg {
    int ncol, L, active_dust, cloudon;
    const double *plev, *tauref_in;
    const double *dust_mass, *dust_number, *ice_mass, *ice_core, *ice_number;
    double *tauref, *qextrefdst, *qxvdst, *qsvdst, *gvdst, *qxidst, *qsidst, *gidst;
    double *taurefcld, *qextrefcld, *qxvcld, *qsvcld, *gvcld, *qxicld, *qsicld, *gicld;
};

constexpr int AERO_WARPS = 4;   // columns (warps) per CTA of rt_aerosol
__global__ void rt_aerosol(const AeroSeg a, const AeroConst K, const double *__restrict__ mie);

}  // namespace mgcm
