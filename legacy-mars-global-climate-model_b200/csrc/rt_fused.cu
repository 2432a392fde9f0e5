// Persistent fused radiation kernel: one launch per call for any number of
// columns on any mix of vertical grids (the segments of a SegTable).
//
// Every CTA loops: it claims a tile of TC consecutive columns from a global
// counter (one atomicAdd), then runs the whole path on that tile --
//   stage   bins (tpindex), per-band opacity terms, Planck terms into the
//           tile's column blocks (code/tpindex.f90:72-134,
//           code/optcv.f90:103-124,182-247, code/optci.f90:113-131,182-220,
//           code/sfluxi.f90:51-62, code/gfluxi.f90:69-87);
//   screen  a warp per (column, screening group): optics sums, TLIMIT test,
//           DETAU and CUMTAUV (code/sfluxv.f90:60-75, code/sfluxi.f90:72-75,
//           code/getdetau.f90:29-56); kept systems appended to the CTA's
//           list in shared memory, each group's run in ascending order;
//   solve   a thread per kept system, visible and IR in one index space
//           (code/gfluxv.f90:108-280, code/gfluxi.f90:69-194,
//           code/dsolver.f90:54-103, code/dtridgl.f90:25-38), flux rows to
//           the CTA's scratch;
//   reduce  a warp per column: ordered sums over (band, Gauss), SUNTOT,
//           IRTOTAL, QRAD (code/sfluxv.f90:102-162, code/sfluxi.f90:95-143,
//           code/comp3.f:677-681,735-738,765-771)
// -- with CTA barriers between the phases.  CTAs never wait on one another,
// so no wait in the kernel can hang.  The CTA's scratch (column blocks, flux
// rows) is written and read back within the tile, while it sits in L2.
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

// Shared memory of a CTA of `warps` warps and TC columns per tile.
__host__ __device__ inline size_t fused_smem_bytes(int warps, int tc) {
    size_t b = 0;
    b += (size_t)tc * NSYS * sizeof(int);                        // kept-system lists (visible, then IR)
    b += (size_t)warps * FZ_WARP_DOUBLES * 8;                      // reduce: folded FZERO, FMNET, top values
    b += 64;
    return (b + 127) / 128 * 128;
}

// Global scratch of one CTA: TC column blocks and the flux rows of every
// system a tile can keep.
__host__ __device__ inline size_t fused_cta_bytes(int tc, int max_nl, size_t stride) {
    const size_t row = (size_t)2 * max_nl * 8;
    return (size_t)tc * stride + (size_t)tc * NSYS * (row + 32);
}

template <bool F32, int TC, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
rt_fused(const SegTable *__restrict__ st, int ncols, int max_nl, unsigned char *__restrict__ scratch, size_t cta_bytes,
         size_t stride, const double *__restrict__ kv, const double *__restrict__ ki,
         const float *__restrict__ kvf, const double *__restrict__ planck, const RtConst K,
         unsigned int *tile_ctr, uint32_t *status, unsigned long long *nsys) {
    constexpr int WARPS = THREADS / 32;
    extern __shared__ __align__(16) unsigned char fz_smem[];
    int *list = reinterpret_cast<int *>(fz_smem);                            // [TC * NSYS]
    double *rbase = reinterpret_cast<double *>(fz_smem + ((size_t)TC * NSYS * sizeof(int) + 15) / 16 * 16);
    __shared__ int s_tile, s_cnt[2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int total = min(st->total_cols, ncols);   // columns [0, ncols) of the table
    unsigned char *blocks = scratch + (size_t)blockIdx.x * cta_bytes;
    const size_t row = (size_t)2 * max_nl;   // doubles per flux row
    double *fl = reinterpret_cast<double *>(blocks + (size_t)TC * stride);   // [TC * NSYS][row]
    double *sc = fl + (size_t)TC * NSYS * row;                              // [TC * NSYS][4]
    SysLocal w;
    unsigned int nsolved = 0;
    for (;;) {
        if (tid == 0) {
            s_tile = (int)atomicAdd(tile_ctr, 1u);
            s_cnt[0] = s_cnt[1] = 0;
        }
        __syncthreads();
        const long long g0ll = (long long)s_tile * TC;
        if (g0ll >= total) break;
        const int g0 = (int)g0ll, ng = min(TC, total - g0);

        // ---- stage: level items of every column, then band items
        const int per_lev = 2 * max_nl + 1, per_band = (max_nl + 1) * (D_NV + D_NI) + D_NI;
        for (int it = tid; it < ng * per_lev; it += THREADS) {
            const int j = it / per_lev, k = 2 + it % per_lev, g = g0 + j;
            const SegDev &sg = st->seg[find_seg(st, g)];
            if (k > 2 * sg.L + 4) continue;
            ColSmem s = carve_smem(blocks + (size_t)j * stride, max_nl, nullptr, false);
            stage_level(sg, g - sg.col0, K, s, k);
        }
        __syncthreads();
        for (int it = tid; it < ng * per_band; it += THREADS) {
            const int j = it / per_band, q = it % per_band, g = g0 + j;
            const SegDev &sg = st->seg[find_seg(st, g)];
            if (q >= stage_band_items(sg.L)) continue;
            ColSmem s = carve_smem(blocks + (size_t)j * stride, max_nl, nullptr, false);
            stage_band(sg, g - sg.col0, K, planck, s, q, status);
        }
        __syncthreads();

        // ---- screen: a warp per (column, group); lists in shared memory,
        // visible entries from 0 up, IR entries from the top down
        for (int it = warp; it < ng * SCREEN_GROUPS; it += WARPS) {
            const int j = it / SCREEN_GROUPS, grp = it % SCREEN_GROUPS, g = g0 + j;
            const SegDev &sg = st->seg[find_seg(st, g)];
            const int c = g - sg.col0;
            ColSmem s = carve_smem(blocks + (size_t)j * stride, max_nl, nullptr, false);
            const bool vis = grp < SCREEN_GROUPS_V;
            const int t = group_first(grp) + lane;
            bool act = false;
            if (vis) {
                if (t < group_end(grp) && sg.acosz[c] >= R4(1.0e-5)) {
                    solve_vis<1, F32>(sg, c, t / D_NG + 1, t % D_NG + 1, t, s, K, kv, w, nsolved, nullptr, nullptr,
                                      nullptr, nullptr, nullptr, kvf);
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
                base = n ? atomicAdd(&s_cnt[vis ? 0 : 1], n) : 0;
                s.meta[2 * grp] = base;
                s.meta[2 * grp + 1] = n;
            }
            base = __shfl_sync(0xffffffffu, base, 0);
            const int pos = base + __popc(m & ((1u << lane) - 1u));
            if (act) list[vis ? pos : TC * NSYS - 1 - pos] = (j << 8) | t;
        }
        __syncthreads();

        // ---- solve: visible entries [0, nv), IR entries [nv, nv + ni)
        const int nv = s_cnt[0], ni = s_cnt[1];
        for (int i = tid; i < nv + ni; i += THREADS) {
            const bool vis = i < nv;
            const int li = vis ? i : i - nv;
            const int e = list[vis ? li : TC * NSYS - 1 - li];
            const int j = e >> 8, sidx = e & 255, g = g0 + j;
            const SegDev &sg = st->seg[find_seg(st, g)];
            const int c = g - sg.col0;
            ColSmem s = carve_smem(blocks + (size_t)j * stride, max_nl, nullptr, false);
            // rows: visible at [0, nv), IR at [TC * NSYS_V + li]
            const size_t r = vis ? (size_t)li : (size_t)TC * NSYS_V + li;
            double *fr = fl + r * row, *scr = sc + r * 4;
            unsigned int dummy = 0;
            if (vis) {
                solve_vis<2, F32>(sg, c, sidx / D_NG + 1, sidx % D_NG + 1, sidx, s, K, kv, w, dummy, fr,
                                  fr + max_nl, scr, scr + 1, scr + 2, kvf);
            } else {
                const int jj = sidx - NSYS_V;
                solve_ir<2>(sg, c, jj / D_NG + 1, jj % D_NG + 1, sidx, s, K, ki, w, dummy, fr, fr + max_nl, scr);
            }
        }
        __syncthreads();

        // ---- reduce: a warp per column, lanes over levels.  Each kept row
        // is weighted as the reference weights it: visible
        // (v*GWEIGHT)*(1-FZEROV), Gauss point 17 v*FZERO; IR
        // ((v*DWNI)*GWEIGHT)*(1-FZEROI), Gauss point 17 (v*DWNI)*FZERO, where
        // FZERO has the weights of the TLIMIT-skipped points folded in, in
        // ascending order (code/sfluxv.f90:72-75,102-162,
        // code/sfluxi.f90:72-75,95-143).  Per family the lanes first lay out
        // the kept rows' positions and weights in order; then each level's
        // sums run over the rows in that order, FZ_RB rows' loads issued
        // before they are added.
        double *fzf = rbase + (size_t)warp * FZ_WARP_DOUBLES;
        double *fmv = fzf + 12, *fmi = fmv + (D_MAXNL + 2), *misc = fmi + (D_MAXNL + 2);
        double *wa = misc + 4, *wb = wa + NSYS_V, *we = wb + NSYS_V;
        int *rpos = reinterpret_cast<int *>(we + NSYS_V);
        for (int j = warp; j < ng; j += WARPS) {
            const int g = g0 + j;
            const SegDev &sg = st->seg[find_seg(st, g)];
            const int c = g - sg.col0;
            const int NL = sg.L + 1, LEV = 2 * sg.L + 3;
            const ColSmem s = carve_smem(blocks + (size_t)j * stride, max_nl, nullptr, false);
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
                            const int sidx = list[vis ? li : TC * NSYS - 1 - li] & 255;
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
                            rpos[nrow + lane] = vis ? li : TC * NSYS_V + li;
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
                                const double *pr = fl + rr * row;
                                if (lv) {
                                    up[q] = pr[l - 1];
                                    dn[q] = pr[max_nl + l - 1];
                                }
                                if (r == 0) {
                                    const double *skp = sc + rr * 4;
                                    t0[q] = vis ? skp[0] - skp[1] : skp[0];
                                    t1[q] = skp[2];
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
        __syncthreads();   // the tile's lists, blocks and rows are free again
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
#undef FUSED_INST
#undef FUSED_ARGS

size_t fused_smem(int warps, int tc) { return fused_smem_bytes(warps, tc); }
size_t fused_scratch_per_cta(int tc, int max_nl, size_t stride) { return fused_cta_bytes(tc, max_nl, stride); }

}  // namespace mgcm
