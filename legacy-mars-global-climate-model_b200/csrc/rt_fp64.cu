// Plain FP64 column radiative transfer, reference operation order.
//
// One CTA per column (persistent grid-stride loop over the columns of every
// segment), 224 threads: thread s < 119 owns visible system (nw, ng) =
// (s/17+1, s%17+1), 119 <= s < 204 owns IR system ((s-119)/17+1, ...).
//
// Per system the reference calls OPTCV/OPTCI (one column of DTAUK),
// GETDETAU, then GFLUXV/GFLUXI -> DSOLVER -> DTRIDGL.  Here a system runs:
//   pass A  top-down over levels: 8-corner k gather and H2O/T/P interpolation
//           (code/optcv.f90:279-303, code/optci.f90:143-167), cumulative TAUCUM,
//           per-layer DTAU/WBAR and the delta-Eddington scaling
//           (code/getdetau.f90:308-335 = code/gfluxv.f90:245-272);
//   pass C  bottom-up over layers: two-stream coefficients
//           (code/gfluxv.f90:277-332, code/gfluxi.f90:219-273), the DSOLVER rows
//           (code/dsolver.f90:54-85) generated in the order DTRIDGL eliminates
//           them (code/dtridgl.f90:131-138), eliminated on the fly;
//   pass D  top-down: DTRIDGL back-substitution (code/dtridgl.f90:140-144),
//           unmixing (code/dsolver.f90:91-103) and the midpoint fluxes
//           (code/gfluxv.f90:339-449, code/gfluxi.f90:286-344).
// The flux sums over bands and Gauss points are then formed by one thread
// per output in the reference's order (code/sfluxv.f90:60-164,
// code/sfluxi.f90:57-145) and turned into SUNTOT/IRTOTAL/QRAD
// (code/comp3.f:677-681,735-738,765-771).
//
// Built with --fmad=false: like the reference's x86-64 build, no multiply-add
// is contracted, so every operation rounds as the Fortran does.  Every
// exponential goes through mgcm_rt_exp (include/mgcm_rt_math.h), the routine
// the CPU oracle uses too, so host and device agree bit-for-bit.
#include "rt_fp64_sys.cuh"
#include "rt_tma.cuh"
#include "../../include/mgcm_rt_math.h"

namespace mgcm {

using namespace fp64;

__global__ void __launch_bounds__(224, 2)
rt_fp64_kernel(const SegTable *__restrict__ st, const double *__restrict__ kv,
               const double *__restrict__ ki, const double *__restrict__ planck,
               const RtConst K, int max_nl, uint32_t *status, unsigned long long *nsys,
               double *red_scratch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ColSmem s = carve_smem(smem_raw, max_nl,
                           red_scratch ? red_scratch + (size_t)blockIdx.x * 2 * NSYS * max_nl : nullptr);
    SysLocal w;
    unsigned int nsolved = 0;
    const int total = st->total_cols;
    for (int g = blockIdx.x; g < total; g += gridDim.x) {
        const int si = find_seg(st, g);
        const SegDev &sg = st->seg[si];
        const int c = g - sg.col0;
        const int L = sg.L, NL = L + 1, LEV = 2 * L + 3;
        const bool day = sg.acosz[c] >= R4(1.0e-5);
        stage_column(sg, c, K, planck, s, status);
        __syncthreads();
        const int t = threadIdx.x;
        if (t < NSYS_V) {
            if (day)
                solve_vis<0>(sg, c, t / D_NG + 1, t % D_NG + 1, t, s, K, kv, w, nsolved,
                             s.fmp + (size_t)t * NL, s.fmm + (size_t)t * NL, &s.sc0[t], &s.sc1[t],
                             &s.sc2[t]);
        } else if (t < NSYS) {
            const int j = t - NSYS_V;
            solve_ir<0>(sg, c, j / D_NG + 1, j % D_NG + 1, t, s, K, ki, w, nsolved,
                        s.fmp + (size_t)t * NL, s.fmm + (size_t)t * NL, &s.sc0[t]);
        }
        __syncthreads();
        reduce_and_heat(
            sg, c, [&](bool vis, int q, int l) { return reduce_family(s, K, vis, q, l, NL); },
            s.fmnet_v, s.fmnet_i, s.misc, day);
        __syncthreads();
    }
    if (nsys) {
        // warp-aggregated count of solved systems
        unsigned int v = nsolved;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(nsys, (unsigned long long)v);
    }
}

// ---------------------------------------------------------------------------
// Three-kernel pipeline over a chunk of columns [col_begin, col_end).  Each
// column owns a block of global memory laid out like the fused kernel's shared
// memory (ColSmem, stride bytes): the stage data, the TLIMIT flags and the
// per-system midpoint fluxes.  Solved systems are listed per family so the
// solver keeps every thread busy (night columns and TLIMIT skips drop out).

// K1: stage the column and screen every system (optics sums, TLIMIT test,
// DETAU, CUMTAUV); append kept systems to the family lists.
template <bool F32>
__global__ void __launch_bounds__(224, 2)
rt_fp64_screen(const SegTable *__restrict__ st, int col_begin, int col_end, int max_nl,
               unsigned char *__restrict__ blocks, size_t stride, const double *__restrict__ kv,
               const double *__restrict__ ki, const double *__restrict__ planck, const RtConst K,
               int *__restrict__ list_v, int *__restrict__ list_i, unsigned int *counts,
               uint32_t *status, unsigned long long *nsys, const float *__restrict__ kvf,
               const float *__restrict__ kif) {
    __shared__ int warp_v[8], warp_i[8], base_v, base_i;
    SysLocal w;
    unsigned int nsolved = 0;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    for (int g = col_begin + blockIdx.x; g < col_end; g += gridDim.x) {
        const int si = find_seg(st, g);
        const SegDev &sg = st->seg[si];
        const int c = g - sg.col0;
        ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        const bool day = sg.acosz[c] >= R4(1.0e-5);
        stage_column(sg, c, K, planck, s, status);
        __syncthreads();
        bool act_v = false, act_i = false;
        if (t < NSYS_V) {
            if (day) {
                solve_vis<1, F32>(sg, c, t / D_NG + 1, t % D_NG + 1, t, s, K, kv, w, nsolved, nullptr,
                                  nullptr, nullptr, nullptr, nullptr, kvf);
                act_v = s.skip[t] == 0;
            }
        } else if (t < NSYS) {
            const int j = t - NSYS_V;
            solve_ir<1, F32>(sg, c, j / D_NG + 1, j % D_NG + 1, t, s, K, ki, w, nsolved, nullptr, nullptr,
                             nullptr, kif);
            act_i = s.skip[t] == 0;
        }
        const unsigned bv = __ballot_sync(0xffffffffu, act_v), bi = __ballot_sync(0xffffffffu, act_i);
        if (lane == 0) {
            warp_v[wid] = __popc(bv);
            warp_i[wid] = __popc(bi);
        }
        __syncthreads();
        if (t == 0) {
            int nv = 0, ni = 0;
            for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
                const int a = warp_v[q], b = warp_i[q];
                warp_v[q] = nv;
                warp_i[q] = ni;
                nv += a;
                ni += b;
            }
            base_v = nv ? (int)atomicAdd(&counts[0], (unsigned)nv) : 0;
            base_i = ni ? (int)atomicAdd(&counts[1], (unsigned)ni) : 0;
            s.meta[0] = base_v;
            s.meta[1] = nv;
            s.meta[2] = base_i;
            s.meta[3] = ni;
        }
        __syncthreads();
        const unsigned below = (1u << lane) - 1u;
        if (act_v) list_v[base_v + warp_v[wid] + __popc(bv & below)] = (g << 8) | t;
        if (act_i) list_i[base_i + warp_i[wid] + __popc(bi & below)] = (g << 8) | t;
        __syncthreads();
    }
    if (nsys) {
        unsigned int v = nsolved;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(nsys, (unsigned long long)v);
    }
}

template __global__ void rt_fp64_screen<false>(const SegTable *__restrict__, int, int, int,
                                               unsigned char *__restrict__, size_t, const double *__restrict__,
                                               const double *__restrict__, const double *__restrict__,
                                               const RtConst, int *__restrict__, int *__restrict__,
                                               unsigned int *, uint32_t *, unsigned long long *,
                                               const float *__restrict__, const float *__restrict__);
template __global__ void rt_fp64_screen<true>(const SegTable *__restrict__, int, int, int,
                                              unsigned char *__restrict__, size_t, const double *__restrict__,
                                              const double *__restrict__, const double *__restrict__,
                                              const RtConst, int *__restrict__, int *__restrict__,
                                              unsigned int *, uint32_t *, unsigned long long *,
                                              const float *__restrict__, const float *__restrict__);

// K2: solve the listed systems of one family, one thread per system.
template <bool VIS>
__global__ void __launch_bounds__(128)
rt_fp64_solve(const SegTable *__restrict__ st, int col_begin, int max_nl,
              unsigned char *__restrict__ blocks, size_t stride, const double *__restrict__ ktab,
              const RtConst K, const int *__restrict__ list, const unsigned int *count,
              double *__restrict__ fl, double *__restrict__ sc) {
    SysLocal w;
    unsigned int dummy = 0;
    const unsigned int n = VIS ? count[0] : count[1];
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int e = list[i];
        const int g = e >> 8, sidx = e & 255;
        const int si = find_seg(st, g);
        const SegDev &sg = st->seg[si];
        const int c = g - sg.col0;
        ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        double *row = fl + (size_t)i * 2 * max_nl, *scr = sc + (size_t)i * 4;
        if (VIS) {
            solve_vis<2>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, sidx, s, K, ktab, w, dummy, row,
                         row + max_nl, scr, scr + 1, scr + 2);
        } else {
            const int j = sidx - NSYS_V;
            solve_ir<2>(sg, c, j / D_NG + 1, j % D_NG + 1, sidx, s, K, ktab, w, dummy, row,
                        row + max_nl, scr);
        }
    }
}

template __global__ void rt_fp64_solve<true>(const SegTable *__restrict__, int, int, unsigned char *__restrict__,
                                             size_t, const double *__restrict__, const RtConst,
                                             const int *__restrict__, const unsigned int *,
                                             double *__restrict__, double *__restrict__);
template __global__ void rt_fp64_solve<false>(const SegTable *__restrict__, int, int, unsigned char *__restrict__,
                                              size_t, const double *__restrict__, const RtConst,
                                              const int *__restrict__, const unsigned int *,
                                              double *__restrict__, double *__restrict__);

// K3: ordered sums and heating per column.  The column's kept systems sit
// in contiguous rows of the compact flux buffers; one thread pulls them into
// shared memory with TMA bulk copies completed on an mbarrier, then one
// thread per output sums them in the reference order.
__global__ void __launch_bounds__(160)
rt_fp64_reduce(const SegTable *__restrict__ st, int col_begin, int col_end, int max_nl,
               unsigned char *__restrict__ blocks, size_t stride, const RtConst K,
               const double *__restrict__ fl_v, const double *__restrict__ sc_v,
               const double *__restrict__ fl_i, const double *__restrict__ sc_i,
               uint32_t *status, int pool_rows) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned char skip[NSYS];
    __shared__ double fmnet_v[D_MAXNL + 1], fmnet_i[D_MAXNL + 1], misc[4];
    __shared__ double mv[3][NSYS_V], mi[3][NSYS_I];
    __shared__ int rows_v, rows_i;
    const size_t row = (size_t)2 * max_nl;
    // a pool of cap_rows rows (visible rows first, then IR) and their scalars
    const int cap_rows = pool_rows;
    double *pool = reinterpret_cast<double *>(smem_raw);
    double *scpool = pool + (size_t)cap_rows * row;
    const int t = threadIdx.x;
    if (t == 0) mbar_init(&bar, 1);
    __syncthreads();
    uint32_t phase = 0;
    for (int g = col_begin + blockIdx.x; g < col_end; g += gridDim.x) {
        const int si = find_seg(st, g);
        const SegDev &sg = st->seg[si];
        const int c = g - sg.col0;
        const ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        const bool day = sg.acosz[c] >= R4(1.0e-5);
        const int bv = s.meta[0], nv = day ? s.meta[1] : 0, bi = s.meta[2], ni = s.meta[3];
        double *flv = pool, *fli = pool + (size_t)nv * row;
        double *scv = scpool, *sci = scpool + (size_t)nv * 4;
        if (nv + ni > cap_rows) {   // more kept systems than the pool holds: sum from global memory
            for (int i = t; i < NSYS; i += blockDim.x) skip[i] = (i < NSYS_V && !day) ? 2 : s.skip[i];
            __syncthreads();
            if (t == 0 && day) rows_v = family_multipliers(skip, K, true, mv[0], mv[1], mv[2]);
            if (t == 32) rows_i = family_multipliers(skip, K, false, mi[0], mi[1], mi[2]);
            __syncthreads();
            reduce_and_heat(
                sg, c,
                [&](bool vis, int q, int l) {
                    return vis ? reduce_rows(fl_v + (size_t)bv * row, sc_v + (size_t)bv * 4, max_nl,
                                             rows_v, mv[0], mv[1], mv[2], true, q, l)
                               : reduce_rows(fl_i + (size_t)bi * row, sc_i + (size_t)bi * 4, max_nl,
                                             rows_i, mi[0], mi[1], mi[2], false, q, l);
                },
                fmnet_v, fmnet_i, misc, day);
            __syncthreads();
            continue;
        }
        if (t == 0) {
            fence_proxy_async_smem();
            const uint32_t bytes = (uint32_t)((nv + ni) * (row * 8 + 32));
            mbar_arrive_expect_tx(&bar, bytes);
            if (nv) {
                bulk_g2s(flv, fl_v + (size_t)bv * row, (uint32_t)(nv * row * 8), &bar);
                bulk_g2s(scv, sc_v + (size_t)bv * 4, (uint32_t)(nv * 32), &bar);
            }
            if (ni) {
                bulk_g2s(fli, fl_i + (size_t)bi * row, (uint32_t)(ni * row * 8), &bar);
                bulk_g2s(sci, sc_i + (size_t)bi * 4, (uint32_t)(ni * 32), &bar);
            }
        }
        for (int i = t; i < NSYS; i += blockDim.x) skip[i] = (i < NSYS_V && !day) ? 2 : s.skip[i];
        __syncthreads();
        if (t == 0 && day) rows_v = family_multipliers(skip, K, true, mv[0], mv[1], mv[2]);
        if (t == 32) rows_i = family_multipliers(skip, K, false, mi[0], mi[1], mi[2]);
        const bool ok = mbar_wait(&bar, phase, status);
        phase ^= 1u;
        __syncthreads();
        if (!ok) {   // copies still in flight: wait for them again, then give up
            mbar_wait(&bar, phase ^ 1u, status);
            return;
        }
        reduce_and_heat(
            sg, c,
            [&](bool vis, int q, int l) {
                return vis ? reduce_rows(flv, scv, max_nl, rows_v, mv[0], mv[1], mv[2], true, q, l)
                           : reduce_rows(fli, sci, max_nl, rows_i, mi[0], mi[1], mi[2], false, q, l);
            },
            fmnet_v, fmnet_i, misc, day);
        __syncthreads();
    }
}

// Shared memory of rt_fp64_reduce: a pool of `rows` kept-system rows.
size_t reduce_smem_bytes(int max_nl, int rows) { return (size_t)rows * (16 * max_nl + 32); }

// Partial radiation: DIRECTSOL from DETAU (code/dsolflux.f:28-45) and
// DNVFLUX = DNDIFFV + DIRECTSOL (code/comp3.f:335-351).
__global__ void rt_dsolflux_kernel(int ncol, const double *__restrict__ sol,
                                   const double *__restrict__ acosz,
                                   const double *__restrict__ detau,
                                   const double *__restrict__ dndiffv,
                                   double *__restrict__ dnvflux, const RtConst K) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncol) return;
    const double u0 = acosz[c];
    double ds = 0.0;
    if (u0 >= R4(1.0e-5)) {
        const double *de = detau + (size_t)c * 119;
        for (int nw = 1; nw <= D_NV; ++nw) {
            const double factor = u0 * sol[nw - 1];
            for (int ng = 1; ng <= D_NG - 1; ++ng) {
                const double d = de[(nw - 1) + 7 * (ng - 1)];
                if (d <= 5.0) ds = ds + factor * mgcm_rt_exp(-d / u0) * K.gweight[ng - 1] * (1.0 - K.fzerov[nw - 1]);
            }
            const double d = de[(nw - 1) + 7 * 16];
            if (d <= 5.0) ds = ds + factor * mgcm_rt_exp(-d / u0) * K.fzerov[nw - 1];
        }
    }
    dnvflux[c] = dndiffv[c] + ds;
}

}  // namespace mgcm
