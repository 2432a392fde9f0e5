// Mixed-precision solver for the kept visible systems (pipeline K2, MIXED
// mode).
//
// The visible opacity work -- the 8-corner gather of the k table, the
// H2O/T/P interpolation and the per-level gas optical depth
// (code/optcv.f90:128-176) -- runs in FP32 on a table of Cmk*k (k itself
// reaches 1e-49, below the FP32 range); the screen kernel does the same.
// Everything after the per-level optical depth stays FP64: the layer sums,
// the delta-Eddington scaling, the two-stream coefficients and exponentials,
// the DSOLVER rows, the DTRIDGL solve and the midpoint fluxes.
//
// The IR family runs the FP64 solver in MIXED mode too.  Measured against
// the FP64 oracle, rounding only the IR per-level optical depths to FP32
// moves IR heating rates by up to 6.4e-3 K/sol on 400 columns and 1.1e-2 K/sol
// on a 64,800-column grid (the error sits in mid-atmosphere layers: one FP32
// rounding of a layer's optical depth acting on its gross emission and
// absorption), at or above the 1e-2 K/sol tolerance; the visible family
// under the same rounding moves heating by 4e-6 K/sol.  FP32 two-stream
// coefficients put ~0.2 K/sol of rounding noise into the thin top layers.
#include "rt_quad.cuh"

namespace mgcm {

__global__ void __launch_bounds__(128, MGCM_VIS_SOLVE_MINB)   // 72 registers, as the FP64 visible solve
rt_mixed_solve_vis(const SegTable *__restrict__ st, int col_begin, int max_nl,
               unsigned char *__restrict__ blocks, size_t stride, const float *__restrict__ ktabf,
               const double *__restrict__ ktab, const RtConst K, const int *__restrict__ list,
               const unsigned int *count, double *__restrict__ fl, double *__restrict__ sc) {
    const unsigned int n = count[0];
    fp64::SysLocal w;
    unsigned int dummy = 0;
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int e = list[i];
        const int g = e >> 8, sidx = e & 255;
        const SegDev &sg = st->seg[find_seg(st, g)];
        const int c = g - sg.col0;
        ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        double *row = fl + row_base(i, max_nl), *scr = sc + sc_base(i);
        double *rdn = row + (size_t)max_nl * ROW_BLK;   // downward fluxes
        fp64::solve_vis<2, true>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, sidx, s, K, ktab, w,
                                 dummy, row, rdn, scr, scr + ROW_BLK, scr + 2 * ROW_BLK, ktabf,
                                 ROW_BLK);
    }
}

// Four-lane form (L <= 51), as rt_quad_solve<true, R> with FP32 opacities.
template <int R>
__global__ void __launch_bounds__(128)
rt_quad_mixed_vis(const SegTable *__restrict__ st, int col_begin, int max_nl,
                  unsigned char *__restrict__ blocks, size_t stride, const float *__restrict__ ktabf,
                  const double *__restrict__ ktab, const RtConst K, const int *__restrict__ list,
                  const unsigned int *count, double *__restrict__ fl, double *__restrict__ sc) {
    const unsigned int n = count[0];
    const unsigned int lane = threadIdx.x & 31;
    const unsigned int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (unsigned int base = warp * 8; base < n; base += nwarps * 8) {
        const unsigned int i = base + (lane >> 2);
        const bool live = i < n;
        const unsigned int ii = live ? i : n - 1;
        const int e = list[ii];
        const int g = e >> 8, sidx = e & 255;
        const SegDev &sg = st->seg[find_seg(st, g)];
        const int c = g - sg.col0;
        const ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        double *row = fl + row_base(ii, max_nl), *scr = sc + sc_base(ii);
        double *rdn = row + (size_t)max_nl * ROW_BLK;   // downward fluxes
        fp64::quad_vis<R, true>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, s, K, ktab, ktabf, live, row,
                                rdn, scr, ROW_BLK);
    }
}

#define QUADM_ARGS                                                                                     \
    const SegTable *__restrict__, int, int, unsigned char *__restrict__, size_t, const float *__restrict__,  \
        const double *__restrict__, const RtConst, const int *__restrict__, const unsigned int *,      \
        double *__restrict__, double *__restrict__
template __global__ void rt_quad_mixed_vis<7>(QUADM_ARGS);
template __global__ void rt_quad_mixed_vis<10>(QUADM_ARGS);
template __global__ void rt_quad_mixed_vis<13>(QUADM_ARGS);
#undef QUADM_ARGS

}  // namespace mgcm
