// Column prep on the device: what COMP3 assembles on the host before it
// calls the radiation, from the GCM state of each column.
//
//   PL            code/potemp1.f:95-106 (PTROP + SIGMA(K) P, PTROP/2 on top)
//   PLEV..TMID    code/fillpt.f90:30-72 (TSTRAT on levels 1-3, the layer
//                 temperatures on the even levels, log-pressure
//                 interpolation on the odd ones, GT at the bottom)
//   QH2O          code/comp3.f:576-589
//   TAUREF        prescribed dust only: the Conrath profile of
//                 code/dustprofile.f:32-114 on the PRDST grid, sampled by
//                 code/filltaucum.f:39-55 (JSRCHGT of code/jsrchgt.f90)
//
// One warp per column.  The lanes share the exponentials of the dust
// profile and the level pairs of the outputs (so the stores coalesce); the
// two running sums of the profile (its normalisation and TAUDST) stay
// serial in lane 0, in the reference's order.  Built with --fmad=false; the
// logarithms, powers and exponentials are the deterministic routines of
// include/mgcm_rt_math.h, which the CPU oracle calls too.
#include "rt_prep.cuh"
#include "rt_common.cuh"
#include "../../include/mgcm_rt_math.h"

namespace mgcm {

namespace {

constexpr int PREP_WARPS = PREP_THREADS / 32;
constexpr int PREP_MAXLEV = D_MAXLEV;

__device__ __forceinline__ double r4(double x) { return (double)(float)x; }

}  // namespace

__global__ void __launch_bounds__(PREP_THREADS)
rt_prep(const PrepSeg a) {
    __shared__ double prdst[PREP_NPDST];
    __shared__ int nstop_s;
    __shared__ double e_s[PREP_WARPS][PREP_NPDST], qr_s[PREP_WARPS][PREP_NPDST];
    __shared__ double td_s[PREP_WARPS][PREP_NPDST], tc_s[PREP_WARPS][PREP_MAXLEV];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int L = a.L, lev = 2 * L + 3, lev1 = lev + 1;
    const double ptrop = a.ptrop, rptau = a.rptau;
    if (a.prescribed_dust) {
        if (threadIdx.x == 0) {
            // code/dustprofile.f:32-37; the exponent is REAL*4 arithmetic
            const float ex = 1.0f / ((float)PREP_NPDST - 1.0f);
            const double refpr = mgcm_rt_pow(5.0 * a.psf / ptrop, (double)ex);
            prdst[0] = ptrop;
            for (int n = 1; n < PREP_NPDST; ++n) prdst[n] = refpr * prdst[n - 1];
            // the Fortran DO index where code/dustprofile.f:59-68 leaves its
            // sum loop: the first n with PRDST(n) >= RPTAU, else NPDST+1
            int ns = PREP_NPDST + 1;
            for (int n = 2; n <= PREP_NPDST; ++n)
                if (prdst[n - 1] >= rptau) {
                    ns = n;
                    break;
                }
            nstop_s = ns;
        }
        __syncthreads();
    }
#define PR(n) prdst[(n) - 1]
    double *E = e_s[wid], *QR = qr_s[wid], *TD = td_s[wid], *TC = tc_s[wid];
    const unsigned full = 0xffffffffu;
    for (long long cc = (long long)blockIdx.x * PREP_WARPS + wid; cc < a.ncol;
         cc += (long long)gridDim.x * PREP_WARPS) {
        const size_t c = (size_t)cc;
        const double p = a.pcol[c];
        const double *tl = a.t + c * L;
        if (a.prescribed_dust) {
            const double conr = a.conr[c], tautot = a.tautot[c];
            const int nstop = nstop_s;
            // exponentials of the sum terms n = 2 .. nstop-1 (= those of QRDST(n-1))
            for (int n = 2 + lane; n < nstop; n += 32) {
                const double pave = 0.5 * (PR(n) + PR(n - 1));
                E[n - 1] = mgcm_rt_exp(conr * (1.0 - (rptau / pave)));
            }
            __syncwarp();
            double qrdst0 = 0.0;
            if (lane == 0) {
                double sum = 0.0;
                for (int n = 2; n < nstop; ++n) sum = sum + E[n - 1] * (PR(n) - PR(n - 1));
                const double pave = 0.5 * (rptau + PR(nstop - 1));
                sum = sum + mgcm_rt_exp(conr * (1.0 - (rptau / pave))) * (rptau - PR(nstop - 1));
                qrdst0 = tautot / sum;
            }
            qrdst0 = __shfl_sync(full, qrdst0, 0);
            // QRDST(n), n = 1 .. NPDST-1 (code/dustprofile.f:79-105)
            for (int n = 1 + lane; n <= PREP_NPDST - 1; n += 32) {
                double q = 0.0;
                if (rptau > PR(n + 1)) {
                    double ex;
                    if (n + 1 < nstop) {
                        ex = E[n];
                    } else {
                        const double pave = 0.5 * (PR(n + 1) + PR(n));
                        ex = mgcm_rt_exp(conr * (1.0 - (rptau / pave)));
                    }
                    q = qrdst0 * ex;
                }
                if (rptau <= PR(n + 1) && rptau >= PR(n)) {
                    const double pave = 0.5 * (PR(n) + rptau);
                    const double pdif1 = rptau - PR(n), pdif2 = PR(n + 1) - rptau;
                    q = qrdst0 * (mgcm_rt_exp(conr * (1.0 - (rptau / pave))) * pdif1 + pdif2) /
                        (PR(n + 1) - PR(n));
                }
                if (rptau < PR(n)) q = qrdst0;
                QR[n - 1] = q;
            }
            __syncwarp();
            if (lane == 0) {   // TAUDST (code/dustprofile.f:109-114)
                double acc = 0.0;
                TD[0] = acc;
                for (int n = 2; n <= PREP_NPDST; ++n) {
                    acc = acc + QR[n - 2] * (PR(n) - PR(n - 1));
                    TD[n - 1] = acc;
                }
            }
            __syncwarp();
            // TAUCUM(K), K = 4 .. LEV (code/filltaucum.f:43-53)
            for (int k = lane; k < lev; k += 32) {
                const int K = k + 1;
                double tc = 0.0;
                if (K >= 4) {
                    const double pstar = p * a.sigma[K - 1] + ptrop;
                    const double pstar1 = pstar > PR(1) ? pstar : PR(1);
                    // JSRCHGT(NPDST-1, PRDST, 1, PSTAR1)
                    const int n = PREP_NPDST - 1;
                    int j;
                    if (pstar1 > PR(n)) {
                        j = n + 1;
                    } else if (pstar1 < PR(1)) {
                        j = 1;
                    } else {
                        int jl = 1, jh = n;
                        while (jh - jl > 1) {
                            const int jm = (jl + jh) / 2;
                            if (pstar1 > PR(jm)) jl = jm;
                            else jh = jm;
                        }
                        if (pstar1 == PR(jh)) jh = jh + 1;
                        j = jh;
                    }
                    // 1 <= NSTAR: PSTAR1 >= PRDST(1) gives j >= 2 (kept for NaN inputs)
                    const int ns = max(1, min(j - 1, PREP_NPDST - 1));
                    tc = TD[ns - 1] + (pstar1 - PR(ns)) * (TD[ns] - TD[ns - 1]) / (PR(ns + 1) - PR(ns));
                }
                TC[k] = tc;
            }
            __syncwarp();
            double *tr = a.tauref + c * lev1;
            for (int k = lane; k < lev1; k += 32)
                tr[k] = (k < 3 || k == lev1 - 1) ? 0.0 : TC[k] - TC[k - 1];
            __syncwarp();   // the buffers are reused by the next column
        }
        // level pairs (K = 2l+1, 2l+2); l = 0 is levels 1-2, l = L+1 level LEV
        double *plev = a.plev + c * lev, *tlev = a.tlev + c * lev;
        double *pmid = a.pmid + c * lev, *tmid = a.tmid + c * lev, *qh = a.qh2o + c * lev;
        const double qfix = r4(1.0E-7);
        auto qval = [&](int l) { return a.active_water ? a.mwratio * a.vapour[c * L + l - 1] : qfix; };
        for (int l = lane; l <= L + 1; l += 32) {
            if (l == 0) {
                const double pv = ptrop / 2.0, ts = a.tstrat[c];
                plev[0] = pv;
                plev[1] = pv;
                tlev[0] = ts;
                tlev[1] = ts;
                tmid[0] = ts;
                tmid[1] = ts;
                pmid[0] = pv;
                pmid[1] = pv;
                qh[0] = 0.0;
                qh[1] = 0.0;
            } else if (l <= L) {
                const int k0 = 2 * l;   // index of K = 2l+1
                const double po = ptrop + a.sigma[k0] * p, pe = ptrop + a.sigma[k0 + 1] * p;
                const double te = tl[l - 1];
                double to;
                if (l == 1) {
                    to = a.tstrat[c];
                } else {
                    const double pm = ptrop + a.sigma[k0 - 1] * p, tm = tl[l - 2];
                    to = te + (tm - te) * mgcm_rt_ln(po / pe) / mgcm_rt_ln(pm / pe);
                }
                plev[k0] = po;
                plev[k0 + 1] = pe;
                tlev[k0] = to;
                tlev[k0 + 1] = te;
                tmid[k0] = to;
                tmid[k0 + 1] = to;
                pmid[k0] = po;
                pmid[k0 + 1] = po;
                qh[k0] = l == 1 ? 0.0 : qval(l - 1);
                qh[k0 + 1] = qval(l);
            } else {
                const double ps = ptrop + p, tg = a.gt[c];
                plev[lev - 1] = ps;
                tlev[lev - 1] = tg;
                tmid[lev - 1] = tg;
                pmid[lev - 1] = ps;
                qh[lev - 1] = qval(L);
            }
        }
    }
#undef PR
}

}  // namespace mgcm
