// Persistent fused radiation kernel: one launch per call for any number of
// columns on any mix of vertical grids (the segments of a SegTable).
//
// Every CTA claims tiles of TC consecutive columns from a global counter (one
// atomicAdd per tile) and runs the whole path on them:
//   stage   bins (tpindex), per-band opacity terms, Planck terms into the
//           tile's column blocks, a warp per column (code/tpindex.f90:72-134,
//           code/optcv.f90:103-124,182-247, code/optci.f90:113-131,182-220,
//           code/sfluxi.f90:51-62, code/gfluxi.f90:69-87);
//   screen  a warp per (column, screening group): optics sums, TLIMIT test,
//           DETAU and CUMTAUV (code/sfluxv.f90:60-75, code/sfluxi.f90:72-75,
//           code/getdetau.f90:29-56); kept systems appended to the tile's
//           list in shared memory, each group's run in ascending order;
//   solve   a thread per kept system, visible and IR in one index space
//           (code/gfluxv.f90:108-280, code/gfluxi.f90:69-194,
//           code/dsolver.f90:54-103, code/dtridgl.f90:25-38), flux rows to
//           the tile's scratch;
//   reduce  a warp per column: ordered sums over (band, Gauss), SUNTOT,
//           IRTOTAL, QRAD (code/sfluxv.f90:102-162, code/sfluxi.f90:95-143,
//           code/comp3.f:677-681,735-738,765-771).
// Two tiles are in flight per CTA, in two buffers, and the phases of
// consecutive tiles overlap:
//   phase X  solve tile k; a warp whose threads have no system left stages
//            tile k+1;
//   phase Y  reduce tile k and screen tile k+1;
// with one CTA barrier after each phase.  Threads and warps take their items
// (systems, columns, groups) from counters in shared memory, so a phase ends
// when its work does, not when a static share does.  CTAs never wait on one
// another, so no wait in the kernel can hang.
//
// The arithmetic is the one of the multi-kernel pipeline (rt_fp64.cu), so
// the FP64 form is bit-identical to it; built with --fmad=false.
#include "rt_fp64_sys.cuh"

namespace mgcm {

using namespace fp64;

// Per-warp reduce scratch: the folded FZERO of 7 + 5 bands, FMNET of both
// families per level, the top-of-atmosphere values, and one family's kept
// rows in order (three weights and a scratch row index each).
constexpr int FZ_WARP_DOUBLES = 12 + 2 * (D_MAXNL + 2) + 4 + 3 * NSYS_V + (NSYS_V + 1) / 2;
constexpr int FZ_RB = 4;   // rows whose loads are issued before they are summed
constexpr int FZ_LPL = (D_MAXNL + 31) / 32;   // levels per lane

// Shared memory of a CTA of `warps` warps and TC columns per tile: the kept
// lists of both buffers and the warps' reduce scratch.
__host__ __device__ inline size_t fused_smem_bytes(int warps, int tc) {
    size_t b = 0;
    b += (size_t)2 * tc * NSYS * sizeof(int);
    b += (size_t)warps * FZ_WARP_DOUBLES * 8;
    b += 64;
    return (b + 127) / 128 * 128;
}

// Global scratch of one buffer: TC column blocks and the flux rows of every
// system a tile can keep (whole blocks of ROW_BLK rows); a CTA holds two.
__host__ __device__ inline size_t fused_buf_bytes(int tc, int max_nl, size_t stride) {
    const size_t row = (size_t)2 * max_nl * 8;
    return ((size_t)tc * stride + row_slots((size_t)tc * NSYS) * (row + 32) + 255) / 256 * 256;
}

// One tile in one buffer.
struct FzBuf {
    unsigned char *blocks;   // TC column blocks
    double *fl, *sc;         // flux rows and scalars of the solve order (row_base, sc_base)
    int *list;               // kept systems: visible from 0 up, IR from TC*NSYS-1 down
    int g0, ng;              // first global column, columns (0: no tile)
};

// Stage column j of a tile: its level items, then its band items, one warp.
__device__ __forceinline__ void fz_stage_column(const SegTable *__restrict__ st, const RtConst &K,
                                                const double *__restrict__ planck, const FzBuf &b, int j,
                                                int max_nl, size_t stride, uint32_t *status, int lane) {
    const int g = b.g0 + j;
    const SegDev &sg = st->seg[find_seg(st, g)];
    const int c = g - sg.col0;
    ColSmem s = carve_smem(b.blocks + (size_t)j * stride, max_nl, nullptr, false);
    const int lev1 = 2 * sg.L + 4;
    for (int k = 2 + lane; k <= lev1; k += 32) stage_level(sg, c, K, s, k);
    __syncwarp();
    const int nb = stage_band_items(sg.L);
    for (int it = lane; it < nb; it += 32) stage_band(sg, c, K, planck, s, it, status);
}

// Screen one (column, group) item of a tile, one warp; kept systems go to
// the tile's list through the per-family counters cnt[0] (visible), cnt[1].
template <bool F32, int TC>
__device__ __forceinline__ void fz_screen_item(const SegTable *__restrict__ st, const RtConst &K,
                                               const double *__restrict__ kv, const double *__restrict__ ki,
                                               const float *__restrict__ kvf, const FzBuf &b, int item, int max_nl,
                                               size_t stride, SysLocal &w, unsigned int &nsolved, int *cnt,
                                               int lane) {
    const int j = item / SCREEN_GROUPS, grp = item % SCREEN_GROUPS, g = b.g0 + j;
    const SegDev &sg = st->seg[find_seg(st, g)];
    const int c = g - sg.col0;
    ColSmem s = carve_smem(b.blocks + (size_t)j * stride, max_nl, nullptr, false);
    const bool vis = grp < SCREEN_GROUPS_V;
    const int t = group_first(grp) + lane;
    bool act = false;
    if (vis) {
        if (t < group_end(grp) && sg.acosz[c] >= R4(1.0e-5)) {
            solve_vis<1, F32>(sg, c, t / D_NG + 1, t % D_NG + 1, t, s, K, kv, w, nsolved, nullptr, nullptr, nullptr,
                              nullptr, nullptr, kvf);
            act = s.skip[t] == 0;
        }
    } else if (t < group_end(grp)) {
        const int jj = t - NSYS_V;
        solve_ir<1>(sg, c, jj / D_NG + 1, jj % D_NG + 1, t, s, K, ki, w, nsolved, nullptr, nullptr, nullptr);
        act = s.skip[t] == 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, act);
    const int n = __popc(m);
    int base = 0;
    if (lane == 0) {
        base = n ? atomicAdd(&cnt[vis ? 0 : 1], n) : 0;
        s.meta[2 * grp] = base;
        s.meta[2 * grp + 1] = n;
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    const int pos = base + __popc(m & ((1u << lane) - 1u));
    if (act) b.list[vis ? pos : TC * NSYS - 1 - pos] = (j << 8) | t;
}

// Solve kept system i of a tile (visible entries [0, nv), IR after), one
// thread; its flux row is row i, so the 32 threads of a warp, which take 32
// consecutive systems, store one 256-byte segment per value.
template <bool F32, int TC>
__device__ __forceinline__ void fz_solve_one(const SegTable *__restrict__ st, const RtConst &K,
                                             const double *__restrict__ kv, const double *__restrict__ ki,
                                             const float *__restrict__ kvf, const FzBuf &b, int i, int nv,
                                             int max_nl, size_t stride, SysLocal &w) {
    const bool vis = i < nv;
    const int li = vis ? i : i - nv;
    const int e = b.list[vis ? li : TC * NSYS - 1 - li];
    const int j = e >> 8, sidx = e & 255, g = b.g0 + j;
    const SegDev &sg = st->seg[find_seg(st, g)];
    const int c = g - sg.col0;
    ColSmem s = carve_smem(b.blocks + (size_t)j * stride, max_nl, nullptr, false);
    double *fr = b.fl + row_base(i, max_nl), *scr = b.sc + sc_base(i);
    double *fdn = fr + (size_t)max_nl * ROW_BLK;
    unsigned int dummy = 0;
    if (vis) {
        solve_vis<2, F32>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, sidx, s, K, kv, w, dummy, fr, fdn, scr,
                          scr + ROW_BLK, scr + 2 * ROW_BLK, kvf, ROW_BLK);
    } else {
        const int jj = sidx - NSYS_V;
        solve_ir<2>(sg, c, jj / D_NG + 1, jj % D_NG + 1, sidx, s, K, ki, w, dummy, fr, fdn, scr, ROW_BLK);
    }
}

// Reduce column j of a tile, one warp (ws: the warp's scratch).  Each kept
// row is weighted as the reference weights it: visible
// (v*GWEIGHT)*(1-FZEROV), Gauss point 17 v*FZERO; IR
// ((v*DWNI)*GWEIGHT)*(1-FZEROI), Gauss point 17 (v*DWNI)*FZERO, where FZERO
// has the weights of the TLIMIT-skipped points folded in, in ascending order
// (code/sfluxv.f90:72-75,102-162, code/sfluxi.f90:72-75,95-143).  Per family
// the lanes first lay out the kept rows' positions and weights in order;
// then each level's sums run over the rows in that order, FZ_RB rows' loads
// issued before they are added.  Then SUNTOT, IRTOTAL and QRAD
// (code/comp3.f:677-681,735-738,765-771).
template <int TC>
__device__ __forceinline__ void fz_reduce_column(const SegTable *__restrict__ st, const RtConst &K, const FzBuf &bf,
                                                 int j, int nv, int max_nl, size_t stride, double *ws, int lane) {
    double *fzf = ws;
    double *fmv = fzf + 12, *fmi = fmv + (D_MAXNL + 2), *misc = fmi + (D_MAXNL + 2);
    double *wa = misc + 4, *wb = wa + NSYS_V, *we = wb + NSYS_V;
    int *rpos = reinterpret_cast<int *>(we + NSYS_V);
    const int g = bf.g0 + j;
    const SegDev &sg = st->seg[find_seg(st, g)];
    const int c = g - sg.col0;
    const int NL = sg.L + 1, LEV = 2 * sg.L + 3;
    const ColSmem s = carve_smem(bf.blocks + (size_t)j * stride, max_nl, nullptr, false);
    const bool day = sg.acosz[c] >= R4(1.0e-5);
    if ((lane < D_NV && day) || (lane >= 8 && lane < 8 + D_NI)) {
        const bool v = lane < D_NV;
        const int nw = v ? lane + 1 : lane - 7;
        const double fz = v ? K.fzerov[nw - 1] : K.fzeroi[nw - 1];
        const unsigned char *sk = s.skip + (v ? 0 : NSYS_V) + (nw - 1) * D_NG;
        double f = fz;
        if (!(fz >= R4(0.99)))
            for (int q = 1; q <= D_NG - 1; ++q)
                if (sk[q - 1] != 0) f = f + (1.0 - fz) * K.gweight[q - 1];
        fzf[v ? nw - 1 : D_NV + nw - 1] = f;
    }
    __syncwarp();
    for (int fam = 0; fam < 2; ++fam) {
        const bool vis = fam == 0;
        // kept rows of the family in order: scratch row index and weights
        int nrow = 0;
        if (!vis || day) {
            const int w0 = vis ? 0 : SCREEN_GROUPS_V, w1 = vis ? SCREEN_GROUPS_V : SCREEN_GROUPS;
            for (int gw = w0; gw < w1; ++gw) {
                const int gb = s.meta[2 * gw], gn = s.meta[2 * gw + 1];
                if (lane < gn) {
                    const int li = gb + lane;
                    const int sidx = bf.list[vis ? li : TC * NSYS - 1 - li] & 255;
                    const int q = vis ? sidx : sidx - NSYS_V;
                    const int nw = q / D_NG + 1, ngs = q % D_NG + 1;
                    double a, b, e;
                    if (vis) {
                        if (ngs < D_NG) { a = K.gweight[ngs - 1]; b = 1.0 - K.fzerov[nw - 1]; }
                        else { a = fzf[nw - 1]; b = 1.0; }
                        e = 1.0;
                    } else {
                        a = K.dwni[nw - 1];
                        if (ngs < D_NG) { b = K.gweight[ngs - 1]; e = 1.0 - K.fzeroi[nw - 1]; }
                        else { b = fzf[D_NV + nw - 1]; e = 1.0; }
                    }
                    wa[nrow + lane] = a;
                    wb[nrow + lane] = b;
                    we[nrow + lane] = e;
                    rpos[nrow + lane] = vis ? li : nv + li;   // row = solve order
                }
                nrow += gn;
            }
        }
        __syncwarp();
        double top = 0.0, dif = 0.0;
        for (int r = 0; r < FZ_LPL && 32 * r < NL; ++r) {
            const int l = lane + 1 + 32 * r;
            const bool lv = l <= NL;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0;
            for (int f0 = 0; f0 < nrow; f0 += FZ_RB) {
                double up[FZ_RB], dn[FZ_RB], t0[FZ_RB], t1[FZ_RB];
#pragma unroll
                for (int q = 0; q < FZ_RB; ++q) {
                    up[q] = dn[q] = t0[q] = t1[q] = 0.0;
                    if (f0 + q < nrow) {
                        const size_t rr = (size_t)rpos[f0 + q];
                        const double *pr = bf.fl + row_base(rr, max_nl);
                        if (lv) {
                            up[q] = pr[(size_t)(l - 1) * ROW_BLK];
                            dn[q] = pr[(size_t)(max_nl + l - 1) * ROW_BLK];
                        }
                        if (r == 0) {
                            const double *skp = bf.sc + sc_base(rr);
                            t0[q] = vis ? skp[0] - skp[ROW_BLK] : skp[0];
                            t1[q] = skp[2 * ROW_BLK];
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < FZ_RB; ++q) {
                    if (f0 + q < nrow) {
                        const double a = wa[f0 + q], b = wb[f0 + q], e = we[f0 + q];
                        auto wt = [&](double v) { return ((v * a) * b) * e; };
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
        __syncwarp();   // the row tables are rebuilt for the next family
    }
    __syncwarp();
    const double *plev = sg.plev + (size_t)c * LEV;
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
    __syncwarp();
}

// Next item of a warp from a shared counter (lane 0 takes it, all lanes get it).
__device__ __forceinline__ int fz_warp_item(int *ctr, int lane) {
    int it = 0;
    if (lane == 0) it = atomicAdd(ctr, 1);
    return __shfl_sync(0xffffffffu, it, 0);
}

template <bool F32, int TC, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
rt_fused(const SegTable *__restrict__ st, int ncols, int max_nl, unsigned char *__restrict__ scratch, size_t cta_bytes,
         size_t stride, const double *__restrict__ kv, const double *__restrict__ ki,
         const float *__restrict__ kvf, const double *__restrict__ planck, const RtConst K,
         unsigned int *tile_ctr, uint32_t *status, unsigned long long *nsys) {
    constexpr int WARPS = THREADS / 32;
    extern __shared__ __align__(16) unsigned char fz_smem[];
    int *lists = reinterpret_cast<int *>(fz_smem);   // [2][TC * NSYS]
    double *ws = reinterpret_cast<double *>(fz_smem + ((size_t)2 * TC * NSYS * sizeof(int) + 15) / 16 * 16) +
                 (size_t)(threadIdx.x >> 5) * FZ_WARP_DOUBLES;
    // s_cnt[b][f]: kept systems of buffer b, family f; s_solve, s_stage,
    // s_item: item counters of the phases; s_claim: the last tile claimed
    __shared__ int s_claim, s_cnt[2][2], s_solve, s_stage, s_item;
    const int tid = threadIdx.x, lane = tid & 31;
    const int total = min(st->total_cols, ncols);   // columns [0, ncols) of the table
    const size_t half = cta_bytes / 2;
    const size_t row = (size_t)2 * max_nl;
    auto buf = [&](int b, int tile) {
        FzBuf r;
        r.blocks = scratch + (size_t)blockIdx.x * cta_bytes + (size_t)b * half;
        r.fl = reinterpret_cast<double *>(r.blocks + (size_t)TC * stride);
        r.sc = r.fl + row_slots((size_t)TC * NSYS) * row;
        r.list = lists + (size_t)b * TC * NSYS;
        const long long g0 = (long long)tile * TC;
        r.g0 = g0 < total ? (int)g0 : 0;
        r.ng = g0 < total ? (int)min((long long)TC, total - g0) : 0;
        return r;
    };
    SysLocal w;
    unsigned int nsolved = 0;

    // prologue: stage and screen the first tile into buffer 0
    if (tid == 0) {
        s_claim = (int)atomicAdd(tile_ctr, 1u);
        s_cnt[0][0] = s_cnt[0][1] = s_cnt[1][0] = s_cnt[1][1] = 0;
        s_solve = s_stage = s_item = 0;
    }
    __syncthreads();
    int tc = s_claim;
    FzBuf bc = buf(0, tc);
    if (bc.ng > 0) {
        for (int it = fz_warp_item(&s_stage, lane); it < bc.ng; it = fz_warp_item(&s_stage, lane))
            fz_stage_column(st, K, planck, bc, it, max_nl, stride, status, lane);
        if (tid == 0) s_claim = (int)atomicAdd(tile_ctr, 1u);
        __syncthreads();
        int tn = s_claim;
        for (int it = fz_warp_item(&s_item, lane); it < bc.ng * SCREEN_GROUPS; it = fz_warp_item(&s_item, lane))
            fz_screen_item<F32, TC>(st, K, kv, ki, kvf, bc, it, max_nl, stride, w, nsolved, s_cnt[0], lane);
        if (tid == 0) s_stage = 0;
        __syncthreads();
        int cur = 0;
        for (;;) {
            const int nxt = cur ^ 1;
            bc = buf(cur, tc);
            const FzBuf bn = buf(nxt, tn);   // ng = 0 when the counter ran past the columns
            // phase X: solve tile cur; warps left without systems stage tile nxt
            const int nv = s_cnt[cur][0], ni = s_cnt[cur][1];
            if (tid == 0) {
                s_item = 0;
                s_cnt[nxt][0] = s_cnt[nxt][1] = 0;
                if (bn.ng > 0) s_claim = (int)atomicAdd(tile_ctr, 1u);
            }
            // a warp takes 32 consecutive systems at a time
            for (;;) {
                int b0 = 0;
                if (lane == 0) b0 = atomicAdd(&s_solve, 32);
                b0 = __shfl_sync(0xffffffffu, b0, 0);
                if (b0 >= nv + ni) break;
                if (b0 + lane < nv + ni)
                    fz_solve_one<F32, TC>(st, K, kv, ki, kvf, bc, b0 + lane, nv, max_nl, stride, w);
            }
            __syncwarp();
            for (int it = fz_warp_item(&s_stage, lane); it < bn.ng; it = fz_warp_item(&s_stage, lane))
                fz_stage_column(st, K, planck, bn, it, max_nl, stride, status, lane);
            __syncthreads();
            const int tnn = s_claim;
            // phase Y: reduce tile cur, screen tile nxt
            if (tid == 0) s_solve = s_stage = 0;
            const int nred = bc.ng, nitems = nred + bn.ng * SCREEN_GROUPS;
            for (int it = fz_warp_item(&s_item, lane); it < nitems; it = fz_warp_item(&s_item, lane)) {
                if (it < nred)
                    fz_reduce_column<TC>(st, K, bc, it, nv, max_nl, stride, ws, lane);
                else
                    fz_screen_item<F32, TC>(st, K, kv, ki, kvf, bn, it - nred, max_nl, stride, w, nsolved,
                                            s_cnt[nxt], lane);
            }
            __syncthreads();   // tile cur's buffer is free; tile nxt is screened
            if (bn.ng == 0) break;
            tc = tn;
            tn = tnn;
            cur = nxt;
        }
    }
    if (nsys) {
        unsigned int v = nsolved;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(nsys, (unsigned long long)v);
    }
}

#define FUSED_ARGS                                                                                     \
    const SegTable *__restrict__, int, int, unsigned char *__restrict__, size_t, size_t,              \
        const double *__restrict__, const double *__restrict__, const float *__restrict__,             \
        const double *__restrict__, const RtConst, unsigned int *, uint32_t *, unsigned long long *
#define FUSED_INST(TC, TH, MB)                                          \
    template __global__ void rt_fused<false, TC, TH, MB>(FUSED_ARGS);  \
    template __global__ void rt_fused<true, TC, TH, MB>(FUSED_ARGS);
FUSED_INST(2, 128, 8)
FUSED_INST(4, 128, 8)
FUSED_INST(8, 128, 8)
FUSED_INST(4, 128, 6)
FUSED_INST(4, 256, 4)
FUSED_INST(8, 256, 4)
FUSED_INST(16, 256, 4)
FUSED_INST(8, 512, 2)
FUSED_INST(8, 256, 3)
FUSED_INST(16, 384, 2)
FUSED_INST(16, 256, 3)
FUSED_INST(24, 384, 2)
FUSED_INST(16, 320, 2)
#undef FUSED_INST
#undef FUSED_ARGS

size_t fused_smem(int warps, int tc) { return fused_smem_bytes(warps, tc); }
size_t fused_scratch_per_cta(int tc, int max_nl, size_t stride) { return 2 * fused_buf_bytes(tc, max_nl, stride); }

}  // namespace mgcm
