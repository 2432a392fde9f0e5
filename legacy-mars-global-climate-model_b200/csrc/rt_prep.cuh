// Column prep on the device (rt_prep.cu): the radiation's level inputs from
// the GCM state of each column.
#pragma once
#include <cstddef>

namespace mgcm {

constexpr int PREP_NPDST = 100;   // L_NPDST (code/modules.f90:114)

// One batch, device pointers.  Inputs [ncol] or [ncol][L]; outputs in the
// layout of mgcm_rt_batch_in ([ncol][2L+3], TAUREF [ncol][2L+4]).
struct PrepSeg {
    int ncol, L, active_water, prescribed_dust;
    double ptrop, psf, rptau, mwratio;
    const double *sigma;                     // [2L+3]
    const double *pcol, *tstrat, *gt;        // P(J,I), TSTRAT, GT
    const double *t;                         // TL(2l+2), l = 1..L
    const double *vapour;                    // QTRACE(J,I,L,iMa_vap) (active_water)
    const double *tautot, *conr;             // TAUTOTJI, Conrath parameter (prescribed_dust)
    double *plev, *tlev, *pmid, *tmid, *qh2o;
    double *tauref;                          // (prescribed_dust)
};

constexpr int PREP_THREADS = 128;
__global__ void rt_prep(const PrepSeg a);

}  // namespace mgcm
