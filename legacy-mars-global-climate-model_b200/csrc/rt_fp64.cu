// Plain FP64 column radiative transfer, reference operation order.
//
// One CTA per column (persistent grid-stride loop over the columns of every
// segment), 224 threads: thread s < 119 owns visible system (nw, ng) =
// (s/17+1, s%17+1), 119 <= s < 204 owns IR system ((s-119)/17+1, ...).
//
// Per system the reference calls OPTCV/OPTCI (one column of DTAUK),
// GETDETAU, then GFLUXV/GFLUXI -> DSOLVER -> DTRIDGL.  Here a system runs:
//   pass A  top-down over levels: 8-corner k gather and H2O/T/P interpolation
//           (code/optcv.f90:128-176, code/optci.f90:143-167), cumulative TAUCUM,
//           per-layer DTAU/WBAR and the delta-Eddington scaling
//           (code/getdetau.f90:29-56 = code/gfluxv.f90:76-103);
//   pass C  bottom-up over layers: two-stream coefficients
//           (code/gfluxv.f90:108-163, code/gfluxi.f90:69-123), the DSOLVER rows
//           (code/dsolver.f90:54-85) generated in the order DTRIDGL eliminates
//           them (code/dtridgl.f90:25-32), eliminated on the fly;
//   pass D  top-down: DTRIDGL back-substitution (code/dtridgl.f90:34-38),
//           unmixing (code/dsolver.f90:91-103) and the midpoint fluxes
//           (code/gfluxv.f90:170-280, code/gfluxi.f90:136-194).
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
#include "rt_quad.cuh"
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

// K0: stage the columns (bins, per-band opacity terms, Planck terms) into
// their global blocks, STAGE_COLS columns per CTA at a time: the level items
// of all of them, a barrier, then their band items.
constexpr int STAGE_COLS = 4;

__global__ void __launch_bounds__(256, 4)   // 64 registers: 4 CTAs/SM (95 unbounded: 2 CTAs; 14.6 -> 14.15 ms per c1 call)
rt_stage(const SegTable *__restrict__ st, int col_begin, int col_end, int max_nl,
         unsigned char *__restrict__ blocks, size_t stride, const double *__restrict__ planck,
         const RtConst K, uint32_t *status) {
    const int per_lev = 2 * max_nl + 1;                             // k = 2 .. 2NL+2
    const int per_band = (max_nl + 1) * (D_NV + D_NI) + D_NI;       // stage_band_items(max L)
    for (int g0 = col_begin + blockIdx.x * STAGE_COLS; g0 < col_end; g0 += gridDim.x * STAGE_COLS) {
        const int ng = min(STAGE_COLS, col_end - g0);
        for (int it = threadIdx.x; it < ng * per_lev; it += blockDim.x) {
            const int g = g0 + it / per_lev, k = 2 + it % per_lev;
            const SegDev &sg = st->seg[find_seg(st, g)];
            if (k > 2 * sg.L + 4) continue;
            ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
            stage_level(sg, g - sg.col0, K, s, k);
        }
        __syncthreads();
        for (int it = threadIdx.x; it < ng * per_band; it += blockDim.x) {
            const int g = g0 + it / per_band, j = it % per_band;
            const SegDev &sg = st->seg[find_seg(st, g)];
            if (j >= stage_band_items(sg.L)) continue;
            ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
            stage_band(sg, g - sg.col0, K, planck, s, j, status);
        }
        __syncthreads();
    }
}

// K1: screen every system (optics sums, TLIMIT test, DETAU, CUMTAUV) and
// append the kept ones to the family lists.  F32 (mixed precision): visible
// gas opacities from the FP32 table; the IR family always screens in FP64.  One warp per (column, group);
// warps never wait on one another.  A group's kept systems take one
// contiguous run of list positions in ascending order; its base and count go
// to the column's meta words.
template <bool F32>
__global__ void __launch_bounds__(128, 8)   // 64 registers: 8 CTAs/SM (measured 6% faster than 80)
rt_fp64_screen(const SegTable *__restrict__ st, int col_begin, int col_end, int max_nl,
               unsigned char *__restrict__ blocks, size_t stride, const double *__restrict__ kv,
               const double *__restrict__ ki, const RtConst K, int *__restrict__ list_v,
               int *__restrict__ list_i, unsigned int *counts, unsigned long long *nsys,
               const float *__restrict__ kvf) {
    SysLocal w;
    unsigned int nsolved = 0;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const long long items = (long long)(col_end - col_begin) * SCREEN_GROUPS;
    for (long long it = (long long)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); it < items; it += nwarps) {
        const int g = col_begin + (int)(it / SCREEN_GROUPS), grp = (int)(it % SCREEN_GROUPS);
        const SegDev &sg = st->seg[find_seg(st, g)];
        const int c = g - sg.col0;
        ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        const bool vis = grp < SCREEN_GROUPS_V;
        const int t = group_first(grp) + lane;
        bool act = false;
        if (vis) {
            if (t < group_end(grp) && sg.acosz[c] >= R4(1.0e-5)) {
                solve_vis<1, F32>(sg, c, t / D_NG + 1, t % D_NG + 1, t, s, K, kv, w, nsolved, nullptr,
                                  nullptr, nullptr, nullptr, nullptr, kvf);
                act = s.skip[t] == 0;
            }
        } else if (t < group_end(grp)) {
            const int j = t - NSYS_V;
            solve_ir<1>(sg, c, j / D_NG + 1, j % D_NG + 1, t, s, K, ki, w, nsolved, nullptr, nullptr,
                        nullptr);
            act = s.skip[t] == 0;
        }
        const unsigned m = __ballot_sync(0xffffffffu, act);
        const int n = __popc(m);
        int base = 0;
        if (lane == 0) {
            base = n ? (int)atomicAdd(&counts[vis ? 0 : 1], (unsigned)n) : 0;
            s.meta[2 * grp] = base;
            s.meta[2 * grp + 1] = n;
        }
        base = __shfl_sync(0xffffffffu, base, 0);
        if (act) (vis ? list_v : list_i)[base + __popc(m & ((1u << lane) - 1u))] = (g << 8) | t;
    }
    if (nsys) {
        unsigned int v = nsolved;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(nsys, (unsigned long long)v);
    }
}

#define SCREEN_ARGS                                                                                    \
    const SegTable *__restrict__, int, int, int, unsigned char *__restrict__, size_t,                \
        const double *__restrict__, const double *__restrict__, const RtConst, int *__restrict__,    \
        int *__restrict__, unsigned int *, unsigned long long *, const float *__restrict__
template __global__ void rt_fp64_screen<false>(SCREEN_ARGS);
template __global__ void rt_fp64_screen<true>(SCREEN_ARGS);
#undef SCREEN_ARGS

// K2: solve the listed systems of one family, one thread per system.
template <bool VIS>
__global__ void __launch_bounds__(128, VIS ? MGCM_VIS_SOLVE_MINB : MGCM_IR_SOLVE_MINB)
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
        double *row = fl + row_base(i, max_nl), *scr = sc + sc_base(i);
        double *rdn = row + (size_t)max_nl * ROW_BLK;   // downward fluxes
        if (VIS) {
            solve_vis<2>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, sidx, s, K, ktab, w, dummy, row,
                         rdn, scr, scr + ROW_BLK, scr + 2 * ROW_BLK, nullptr, ROW_BLK);
        } else {
            const int j = sidx - NSYS_V;
            solve_ir<2>(sg, c, j / D_NG + 1, j % D_NG + 1, sidx, s, K, ktab, w, dummy, row,
                        rdn, scr, ROW_BLK);
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

// K2 (four-lane form, L <= 51): a quad of lanes per kept system, 8 systems
// per warp, per-layer values in registers (rt_quad.cuh).  A quad past the
// end of the list repeats the last system and stores nothing.
template <bool VIS, int R>
__global__ void __launch_bounds__(128)
rt_quad_solve(const SegTable *__restrict__ st, int col_begin, int max_nl,
              unsigned char *__restrict__ blocks, size_t stride, const double *__restrict__ ktab,
              const RtConst K, const int *__restrict__ list, const unsigned int *count,
              double *__restrict__ fl, double *__restrict__ sc) {
    const unsigned int n = VIS ? count[0] : count[1];
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
        if (VIS) {
            quad_vis<R, false>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, s, K, ktab, nullptr, live, row,
                               rdn, scr, ROW_BLK);
        } else {
            const int j = sidx - NSYS_V;
            quad_ir<R>(sg, c, j / D_NG + 1, j % D_NG + 1, s, K, ktab, live, row, rdn, scr,
                       ROW_BLK);
        }
    }
}

#define QUAD_ARGS                                                                                      \
    const SegTable *__restrict__, int, int, unsigned char *__restrict__, size_t, const double *__restrict__, \
        const RtConst, const int *__restrict__, const unsigned int *, double *__restrict__,             \
        double *__restrict__
template __global__ void rt_quad_solve<true, 7>(QUAD_ARGS);
template __global__ void rt_quad_solve<true, 10>(QUAD_ARGS);
template __global__ void rt_quad_solve<true, 13>(QUAD_ARGS);
template __global__ void rt_quad_solve<false, 7>(QUAD_ARGS);
template __global__ void rt_quad_solve<false, 10>(QUAD_ARGS);
template __global__ void rt_quad_solve<false, 13>(QUAD_ARGS);
#undef QUAD_ARGS

// K3: ordered sums and heating, one warp per column.  The solves store their
// flux rows in blocks of 32 list positions (row_base, sc_base): value k of
// the system at position p is fl[row_base(p) + 32 k] (k < max_nl: upward
// midpoint flux of layer k+1; max_nl + k: downward), scalar q
// sc[sc_base(p) + 32 q].  A column's kept systems sit in one run of
// positions per screening group, in ascending (band, Gauss) order.  Lane j
// owns levels j+1, j+33, ... and sums its outputs over the systems in the
// reference order, each scaled by the multipliers of family_multipliers; the
// loads of RB systems are issued before they are summed.
constexpr int RED_WARPS = 4;
constexpr int RED_LPL = (D_MAXNL + 1 + 31) / 32;   // levels per lane

// Shared memory of one warp: the multipliers of both families, FMNET per
// level of both families, the top-of-atmosphere values, and one family's
// kept list positions in order.
__host__ __device__ inline size_t red_warp_bytes() {
    size_t b = (size_t)3 * NSYS * 8;                  // multipliers
    b += (size_t)2 * (D_MAXNL + 2) * 8 + 4 * 8;       // FMNET per level, top values
    b += (size_t)NSYS * 4;                            // list positions
    return (b + 127) / 128 * 128;
}

// Multipliers of both families for one column, one lane per band (visible
// bands on lanes 0-6, IR bands on lanes 8-12); each lane walks its band as
// family_multipliers does, at the band's offset among the kept rows.
__device__ inline void warp_multipliers(const unsigned char *skip, bool day, const RtConst &K,
                                        double *m1, double *m2, double *m3) {
    const int lane = threadIdx.x & 31;
    const bool isv = lane < D_NV && day, isi = lane >= 8 && lane < 8 + D_NI;
    const int nw = isv ? lane + 1 : (isi ? lane - 7 : 0);
    const int base = isv ? 0 : NSYS_V;
    const double fz = isv ? K.fzerov[nw - 1] : (isi ? K.fzeroi[nw - 1] : 0.0);
    const unsigned char *sk = skip + base + (nw > 0 ? nw - 1 : 0) * D_NG;
    int cnt = 0;
    if (isv || isi) {
        if (!(fz >= R4(0.99)))
            for (int ng = 1; ng <= D_NG - 1; ++ng) cnt += sk[ng - 1] == 0;
        cnt += 1;
    }
    // exclusive prefix over the lanes of the same family
    const int first = isv ? 0 : 8;
    int pos = 0;
    for (int k = 1; k < 8; ++k) {
        const int v = __shfl_up_sync(0xffffffffu, cnt, k);
        if (lane - k >= first) pos += v;
    }
    if (!(isv || isi)) return;
    double *p1 = m1 + base, *p2 = m2 + base, *p3 = m3 + base;
    double fzero = fz;
    const double dw = isv ? 1.0 : K.dwni[nw - 1];
    if (!(fz >= R4(0.99))) {
        for (int ng = 1; ng <= D_NG - 1; ++ng) {
            if (sk[ng - 1] != 0) {
                fzero = fzero + (1.0 - fz) * K.gweight[ng - 1];
                continue;
            }
            if (isv) {
                p1[pos] = K.gweight[ng - 1];
                p2[pos] = 1.0 - fz;
                p3[pos] = 1.0;
            } else {
                p1[pos] = dw;
                p2[pos] = K.gweight[ng - 1];
                p3[pos] = 1.0 - fz;
            }
            ++pos;
        }
    }
    if (isv) {
        p1[pos] = fzero;
        p2[pos] = 1.0;
    } else {
        p1[pos] = dw;
        p2[pos] = fzero;
    }
    p3[pos] = 1.0;
}

template <bool ONE_LEVEL, int RB>   // ONE_LEVEL: max NL <= 32, one level per lane
__global__ void __launch_bounds__(32 * RED_WARPS)
rt_fp64_reduce(const SegTable *__restrict__ st, int col_begin, int col_end, int max_nl,
               unsigned char *__restrict__ blocks, size_t stride, const RtConst K,
               const double *__restrict__ fl_v, const double *__restrict__ sc_v,
               const double *__restrict__ fl_i, const double *__restrict__ sc_i) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int LPL = ONE_LEVEL ? 1 : RED_LPL;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned char *ws = smem_raw + (size_t)wid * red_warp_bytes();
    double *m1 = reinterpret_cast<double *>(ws);
    double *m2 = m1 + NSYS, *m3 = m2 + NSYS;
    double *fmv = m3 + NSYS, *fmi = fmv + (D_MAXNL + 2), *misc = fmi + (D_MAXNL + 2);
    int *rpos = reinterpret_cast<int *>(misc + 4);

    for (int g = col_begin + blockIdx.x * RED_WARPS + wid; g < col_end; g += gridDim.x * RED_WARPS) {
        const int si = find_seg(st, g);
        const SegDev &sg = st->seg[si];
        const int c = g - sg.col0;
        const int NL = sg.L + 1;
        const ColSmem s = carve_smem(blocks + (size_t)(g - col_begin) * stride, max_nl, nullptr, false);
        const bool day = sg.acosz[c] >= R4(1.0e-5);
        warp_multipliers(s.skip, day, K, m1, m2, m3);
        for (int fam = 0; fam < 2; ++fam) {
            const bool vis = fam == 0;
            // list positions of the family's kept systems (none at night for
            // the visible family: its outputs are zeros)
            int nrow = 0;
            if (!vis || day) {
                const int w0 = vis ? 0 : SCREEN_GROUPS_V, w1 = vis ? SCREEN_GROUPS_V : SCREEN_GROUPS;
                for (int gw = w0; gw < w1; ++gw) {
                    const int gb = s.meta[2 * gw], gn = s.meta[2 * gw + 1];
                    for (int q = lane; q < gn; q += 32) rpos[nrow + q] = gb + q;
                    nrow += gn;
                }
            }
            __syncwarp();
            const double *fl = vis ? fl_v : fl_i, *sc = vis ? sc_v : sc_i;
            const double *f1 = vis ? m1 : m1 + NSYS_V, *f2 = vis ? m2 : m2 + NSYS_V, *f3 = vis ? m3 : m3 + NSYS_V;
            double top = 0.0, dif = 0.0;
#pragma unroll 1
            for (int r = 0; r < LPL; ++r) {
                if (32 * r >= NL) break;
                const int l = lane + 1 + 32 * r;
                const bool lv = l <= NL;
                const size_t ou = (size_t)(lv ? l - 1 : 0) * ROW_BLK, od = ou + (size_t)max_nl * ROW_BLK;
                double a0 = 0.0, a1 = 0.0, a2 = 0.0;
                for (int f0 = 0; f0 < nrow; f0 += RB) {
                    double up[RB], dn[RB], t0[RB], t1[RB];
#pragma unroll
                    for (int q = 0; q < RB; ++q) {
                        up[q] = dn[q] = t0[q] = t1[q] = 0.0;
                        if (f0 + q < nrow) {
                            const int p = rpos[f0 + q];
                            const double *pr = fl + row_base(p, max_nl);
                            if (lv) {
                                up[q] = __ldg(pr + ou);
                                dn[q] = __ldg(pr + od);
                            }
                            if (r == 0) {
                                const double *ps = sc + sc_base(p);
                                t0[q] = vis ? __ldg(ps) - __ldg(ps + ROW_BLK) : __ldg(ps);
                                if (vis) t1[q] = __ldg(ps + 2 * ROW_BLK);
                            }
                        }
                    }
#pragma unroll
                    for (int q = 0; q < RB; ++q) {
                        if (f0 + q < nrow) {
                            const double a = f1[f0 + q], b = f2[f0 + q], e = f3[f0 + q];
                            // ((v*a)*b)*e in the reference order; a factor that is
                            // exactly 1.0 leaves the product unchanged and is
                            // skipped (warp-uniform)
                            const bool b1 = b == 1.0, e1 = e == 1.0;
                            auto wt = [&](double v) {
                                double x = v * a;
                                if (!b1) x = x * b;
                                if (!e1) x = x * e;
                                return x;
                            };
                            a0 = a0 + wt(up[q] - dn[q]);
                            a1 = a1 + wt(up[q]);
                            a2 = a2 + wt(dn[q]);
                            if (r == 0) {
                                top = top + wt(t0[q]);
                                if (vis) dif = dif + wt(t1[q]);
                            }
                        }
                    }
                }
                if (lv) {
                    const size_t o = (size_t)c * NL + l - 1;
                    if (vis) {
                        sg.fmnetv[o] = a0;
                        sg.fluxupv[o] = a1;
                        sg.fluxdnv[o] = a2;
                        fmv[l] = a0;
                        if (l == NL) {
                            sg.dnvflux[c] = a2;
                            sg.fluxsurf[c] = (1.0 - sg.als[c]) * a2;
                        }
                    } else {
                        sg.fmneti[o] = a0;
                        sg.fluxupi[o] = a1;
                        sg.fluxdni[o] = a2;
                        fmi[l] = a0;
                        if (l == NL) sg.dnirflux[c] = a2;
                    }
                }
            }
            if (lane == 0) {
                if (vis) {
                    sg.nfluxtopv[c] = top;
                    sg.diffvt[c] = dif;
                    sg.dndiffv[c] = dif;
                    misc[0] = top;
                } else {
                    sg.nfluxtopi[c] = top;
                    misc[1] = top;
                }
            }
            __syncwarp();   // rpos is rewritten by the next family
        }
        // divergences and heating rates (code/comp3.f:677-681,735-738,765-771)
        const double *plev = sg.plev + (size_t)c * (2 * sg.L + 3);
        const int LEV = 2 * sg.L + 3;
        for (int l = 1 + lane; l <= NL; l += 32) {
            const double sun = day ? (l == 1 ? fmv[1] - misc[0] : fmv[l] - fmv[l - 1]) : 0.0;
            const double irt = l == 1 ? fmi[1] - misc[1] : fmi[l] - fmi[l - 1];
            const int k = 2 * l;
            const double ptrop = sg.ptrop, p = sg.pcol[c];
            const double ym = k == 2 ? ptrop * 100.0 / 3.72 : (plev[k + 1 - 1] - plev[k - 1 - 1]) * 100.0 / 3.72;
            const double om = pow(plev[k - 1] / plev[LEV - 1], 0.25684);
            const double pnlte = sg.sigma[k - 1] * (p - ptrop) + ptrop;
            const double sunlte = sun * 2.2e4 * pnlte / (1.0 + 2.2e4 * pnlte);
            const size_t o = (size_t)c * NL + l - 1;
            sg.suntot[o] = sun;
            sg.irtotal[o] = irt;
            sg.qrad[o] = (sunlte + irt) / (735.94 * ym * om);
        }
        __syncwarp();   // fmv, fmi, misc and the multipliers are rewritten by the next column
    }
}

#define REDUCE_ARGS                                                                                    \
    const SegTable *__restrict__, int, int, int, unsigned char *__restrict__, size_t, const RtConst,  \
        const double *__restrict__, const double *__restrict__, const double *__restrict__,          \
        const double *__restrict__
#define REDUCE_INST(RB)                                              \
    template __global__ void rt_fp64_reduce<true, RB>(REDUCE_ARGS);  \
    template __global__ void rt_fp64_reduce<false, RB>(REDUCE_ARGS);
REDUCE_INST(1)
REDUCE_INST(2)
REDUCE_INST(4)
REDUCE_INST(8)
#undef REDUCE_INST
#undef REDUCE_ARGS

// Shared memory of rt_fp64_reduce (the same for every batch size).
size_t reduce_smem_bytes(int max_nl, int rb) {
    (void)max_nl;
    (void)rb;
    return (size_t)RED_WARPS * red_warp_bytes();
}
// Systems whose loads the reduce issues before it sums them, by default
// (measured on the 64,800-column call: 4 -> 8 saves 0.07 ms; 16 needs 182
// registers and is slower).
int reduce_rows_per_chunk(int max_nl) {
    (void)max_nl;
    return 8;
}
// The reduce kernel of a launch: one level per lane up to NL = 32, and RB
// in {1, 2, 4, 8} (other values round down).
const void *reduce_kernel(int max_nl, int rb) {
    const bool one = max_nl <= 32;
    if (rb >= 8) return one ? (const void *)rt_fp64_reduce<true, 8> : (const void *)rt_fp64_reduce<false, 8>;
    if (rb >= 4) return one ? (const void *)rt_fp64_reduce<true, 4> : (const void *)rt_fp64_reduce<false, 4>;
    if (rb >= 2) return one ? (const void *)rt_fp64_reduce<true, 2> : (const void *)rt_fp64_reduce<false, 2>;
    return one ? (const void *)rt_fp64_reduce<true, 1> : (const void *)rt_fp64_reduce<false, 1>;
}

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


// Integer bins as the pipeline uses them, for the bit-exact check of
// tpindex (code/tpindex.f90:72-134) and of the Planck index INT(T*10-499)
// (code/sfluxi.f90:54-55, code/gfluxi.f90:73-74,86-87).  Reads the column
// blocks rt_stage wrote -- each level's k-table corner offset and NH2O step
// -- and turns them back into MT, MP, NH2O; copies WRATIO and LCOEF(1..4);
// and evaluates planck_index, the function rt_stage uses, on every TLEV.
// One thread per (column, level K = 1..LEV); outputs [ncol][LEV] (LCOEF
// [ncol][LEV][4]); level 1 has no tpindex call and gets zeros.
__global__ void rt_bins_decode(const SegTable *__restrict__ st, int ncol, int max_nl,
                               const unsigned char *__restrict__ blocks, size_t stride,
                               uint32_t *status, int *__restrict__ mt, int *__restrict__ mp,
                               int *__restrict__ nh, int *__restrict__ npl, double *__restrict__ wr,
                               double *__restrict__ lk) {
    const SegDev &sg = st->seg[0];
    const int LEV = 2 * sg.L + 3;
    const long long n = (long long)ncol * LEV;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i / LEV), k = (int)(i % LEV) + 1;
        npl[i] = planck_index(sg.tlev[(size_t)c * LEV + k - 1], status);
        if (k == 1) {
            mt[i] = mp[i] = nh[i] = 0;
            wr[i] = 0.0;
            for (int q = 0; q < 4; ++q) lk[i * 4 + q] = 0.0;
            continue;
        }
        const ColSmem s = carve_smem(const_cast<unsigned char *>(blocks) + (size_t)c * stride, max_nl,
                                     nullptr, false);
        const KLevel &r = s.klev[k];
        const int e = r.kofs / D_NGK;   // ((MT-1)*NP + MP-1)*NH + NH2O-1
        nh[i] = e % D_NH + 1;
        mp[i] = (e / D_NH) % D_NP + 1;
        mt[i] = e / (D_NH * D_NP) + 1;
        wr[i] = r.wr;
        for (int q = 0; q < 4; ++q) lk[i * 4 + q] = r.lk[q];
    }
}

}  // namespace mgcm
