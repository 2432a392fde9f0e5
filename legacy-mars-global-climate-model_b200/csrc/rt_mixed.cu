// Mixed-precision solver for the kept systems (pipeline K2, MIXED mode).
//
// The opacity work -- the 8-corner gather of the k table, the H2O/T/P
// interpolation and the per-level gas optical depth (code/optcv.f90:279-303,
// code/optci.f90:143-167) -- runs in FP32 on a table of Cmk*k (k itself
// reaches 1e-49, below the FP32 range); the screen kernel does the same.
// Everything after the per-level optical depth stays FP64: the layer sums,
// the delta-Eddington scaling, the two-stream coefficients and exponentials,
// the DSOLVER rows, the DTRIDGL solve and the midpoint fluxes.  Measured on
// the workload, FP32 two-stream coefficients put ~0.2 K/sol of rounding noise
// into the heating of the thin top layers (layer masses of 0.02 kg/m^2 turn
// 1e-7 relative flux noise into tenths of K/sol), above the 1e-2 K/sol
// tolerance; FP32 opacities stay within it.
#include "rt_fp64_sys.cuh"

namespace mgcm {

template <bool VIS>
__global__ void __launch_bounds__(128)
rt_mixed_solve(const SegTable *__restrict__ st, int col_begin, int max_nl,
               unsigned char *__restrict__ blocks, size_t stride, const float *__restrict__ ktabf,
               const double *__restrict__ ktab, const RtConst K, const int *__restrict__ list,
               const unsigned int *count, double *__restrict__ fl, double *__restrict__ sc) {
    const unsigned int n = VIS ? count[0] : count[1];
    fp64::SysLocal w;
    unsigned int dummy = 0;
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int e = list[i];
        const int g = e >> 8, sidx = e & 255;
        const SegDev &sg = st->seg[find_seg(st, g)];
        const int c = g - sg.col0;
        ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        double *row = fl + (size_t)i * 2 * max_nl, *scr = sc + (size_t)i * 4;
        if (VIS) {
            fp64::solve_vis<2, true>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, sidx, s, K, ktab, w,
                                     dummy, row, row + max_nl, scr, scr + 1, scr + 2, ktabf);
        } else {
            const int j = sidx - NSYS_V;
            fp64::solve_ir<2, true>(sg, c, j / D_NG + 1, j % D_NG + 1, sidx, s, K, ktab, w, dummy,
                                    row, row + max_nl, scr, ktabf);
        }
    }
}

template __global__ void rt_mixed_solve<true>(const SegTable *__restrict__, int, int, unsigned char *__restrict__,
                                              size_t, const float *__restrict__, const double *__restrict__,
                                              const RtConst, const int *__restrict__, const unsigned int *,
                                              double *__restrict__, double *__restrict__);
template __global__ void rt_mixed_solve<false>(const SegTable *__restrict__, int, int, unsigned char *__restrict__,
                                               size_t, const float *__restrict__, const double *__restrict__,
                                               const RtConst, const int *__restrict__, const unsigned int *,
                                               double *__restrict__, double *__restrict__);

}  // namespace mgcm
