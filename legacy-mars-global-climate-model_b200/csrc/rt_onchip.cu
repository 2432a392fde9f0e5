// Solve kernels of the pipeline with the per-system arrays on chip
// (rt_onchip.cuh): one thread per kept (band, Gauss) system, T threads per
// CTA, one CTA per SM holding T slices of 7NL+1 doubles in shared memory.
// Built with --fmad=false like rt_fp64.cu, so the FP64 forms reproduce the
// oracle's rounding; the MIXED visible form takes its gas opacities from the
// FP32 table.
#include "rt_onchip.cuh"

namespace mgcm {

template <bool VIS, bool F32, int T>
__global__ void __launch_bounds__(T, 1)
rt_solve_oc(const SegTable *__restrict__ st, int col_begin, int max_nl, unsigned char *__restrict__ blocks,
            size_t stride, const double *__restrict__ ktab, const float *__restrict__ ktabf, const RtConst K,
            const int *__restrict__ list, const unsigned int *count, double *__restrict__ fl,
            double *__restrict__ sc) {
    extern __shared__ __align__(16) double oc_slots[];
    const onchip::SmemSlots<T> ss{oc_slots, (int)threadIdx.x};
    const unsigned int n = VIS ? count[0] : count[1];
    for (unsigned int i = blockIdx.x * T + threadIdx.x; i < n; i += gridDim.x * T) {
        const int e = list[i];
        const int g = e >> 8, sidx = e & 255;
        const SegDev &sg = st->seg[find_seg(st, g)];
        const int c = g - sg.col0;
        const ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        double *row = fl + row_base(i, max_nl), *scr = sc + sc_base(i);
        double *rdn = row + (size_t)max_nl * ROW_BLK;   // downward fluxes
        if (VIS) {
            onchip::solve_vis_oc<onchip::SmemSlots<T>, F32>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, s, K, ktab,
                                                            ktabf, ss, row, rdn, scr, scr + ROW_BLK,
                                                            scr + 2 * ROW_BLK, ROW_BLK);
        } else {
            const int j = sidx - NSYS_V;
            onchip::solve_ir_oc(sg, c, j / D_NG + 1, j % D_NG + 1, s, ktab, ss, row, rdn, scr,
                                ROW_BLK);
        }
    }
}

// The same with tensor memory in front of shared memory: W warps, one CTA
// per SM, the CTA's 512 TMEM columns split between the warps that share a
// lane quarter (warps w and w+4, w+8, ...), vt doubles per thread.  Loops
// are warp-uniform: every warp takes 32 consecutive list entries; lanes past
// the end repeat the last entry (identical values to the same rows).  All
// systems of the launch have one layer count (the host checks), so the
// per-system loops run the same trips on every lane.
template <bool VIS, bool F32, int W>
__global__ void __launch_bounds__(32 * W, 1)
rt_solve_tm(const SegTable *__restrict__ st, int col_begin, int max_nl, unsigned char *__restrict__ blocks,
            size_t stride, const double *__restrict__ ktab, const float *__restrict__ ktabf, const RtConst K,
            const int *__restrict__ list, const unsigned int *count, double *__restrict__ fl,
            double *__restrict__ sc) {
    constexpr int T = 32 * W;
    constexpr int GROUPS = (W + 3) / 4;
    constexpr uint32_t COLS = (512 / GROUPS) & ~1u;   // TMEM columns per thread
    extern __shared__ __align__(16) double oc_slots[];
    __shared__ uint32_t tm_base;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) tmem_alloc(&tm_base, 512);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t taddr = tm_base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(warp >> 2) * COLS;
    const onchip::HybridSlots<T> ss{oc_slots, (int)threadIdx.x, taddr, (int)(COLS / 2)};
    const unsigned int n = VIS ? count[0] : count[1];
    for (unsigned int base = blockIdx.x * T + 32 * warp; base < n; base += gridDim.x * T) {
        const unsigned int i = min(base + lane, n - 1);
        const int e = list[i];
        const int g = e >> 8, sidx = e & 255;
        const SegDev &sg = st->seg[find_seg(st, g)];
        const int c = g - sg.col0;
        const ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        double *row = fl + row_base(i, max_nl), *scr = sc + sc_base(i);
        double *rdn = row + (size_t)max_nl * ROW_BLK;   // downward fluxes
        if (VIS) {
            onchip::solve_vis_oc<onchip::HybridSlots<T>, F32>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, s, K,
                                                              ktab, ktabf, ss, row, rdn, scr,
                                                              scr + ROW_BLK, scr + 2 * ROW_BLK, ROW_BLK);
        } else {
            const int j = sidx - NSYS_V;
            onchip::solve_ir_oc(sg, c, j / D_NG + 1, j % D_NG + 1, s, ktab, ss, row, rdn, scr,
                                ROW_BLK);
        }
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    if (warp == 0) tmem_dealloc(tm_base, 512);
}

#define OC_ARGS                                                                                          \
    const SegTable *__restrict__, int, int, unsigned char *__restrict__, size_t, const double *__restrict__, \
        const float *__restrict__, const RtConst, const int *__restrict__, const unsigned int *,         \
        double *__restrict__, double *__restrict__
#define OC_INST(T)                                                        \
    template __global__ void rt_solve_oc<true, false, T>(OC_ARGS);       \
    template __global__ void rt_solve_oc<true, true, T>(OC_ARGS);        \
    template __global__ void rt_solve_oc<false, false, T>(OC_ARGS);
OC_INST(32)
OC_INST(64)
OC_INST(96)
OC_INST(128)
OC_INST(160)
OC_INST(192)
OC_INST(224)
OC_INST(256)
#undef OC_INST
#define TM_INST(W)                                                        \
    template __global__ void rt_solve_tm<true, false, W>(OC_ARGS);       \
    template __global__ void rt_solve_tm<true, true, W>(OC_ARGS);        \
    template __global__ void rt_solve_tm<false, false, W>(OC_ARGS);
TM_INST(4)
TM_INST(6)
TM_INST(8)
TM_INST(9)
#undef TM_INST
#undef OC_ARGS

}  // namespace mgcm
