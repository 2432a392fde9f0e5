// Phase 1 of a column: level bins and per-band opacity terms into shared memory.
// Restates the set-up loops of code/optcv.f90:103-124,182-247 and
// code/optci.f90:113-131,182-220 plus the Planck boundary terms of
// code/sfluxi.f90:51-62 and code/gfluxi.f90:69-87.
#pragma once
#include "rt_column.cuh"

namespace mgcm {

// Level item k (2..LEV+1) of column c: bins, U, DPR and the TAUREF ratios.
__device__ inline void stage_level(const SegDev &sg, int c, const RtConst &K, ColSmem &s, int k) {
    const int L = sg.L, LEV = 2 * L + 3, LEV1 = LEV + 1;
    const double *plev = sg.plev + (size_t)c * LEV;
    const double *tlev = sg.tlev + (size_t)c * LEV;
    const double *pmid = sg.pmid + (size_t)c * LEV;
    const double *tmid = sg.tmid + (size_t)c * LEV;
    const double *qh2o = sg.qh2o + (size_t)c * LEV;
    const double *tauref = sg.tauref + (size_t)c * LEV1;
    const double *db = sg.dust_band;   // prescribed dust: band constants
    const double *qxref = db ? nullptr : sg.qextrefdst + (size_t)c * LEV1;
    const double *qxv = db ? nullptr : sg.qxvdst + (size_t)c * D_NV * LEV1;
    const bool cld = sg.taurefcld != nullptr;
    const double *taucld = cld ? sg.taurefcld + (size_t)c * LEV1 : nullptr;
    const double *qxcld = cld ? sg.qextrefcld + (size_t)c * LEV1 : nullptr;

    {
        if (k <= LEV) {
            int mt, mp, nh;
            double wr, lk[4];
            tpindex_dev(K, pmid[k - 1], tmid[k - 1], qh2o[k - 1], mt, mp, nh, wr, lk);
            const int nh1 = nh < D_NH ? nh + 1 : D_NH;   // WRATIO = 0 when NH2O = 10
            KLevel &kl = s.klev[k];
            kl.kofs = (((mt - 1) * D_NP + (mp - 1)) * D_NH + (nh - 1)) * D_NGK;
            kl.kdh = (nh1 - nh) * D_NGK;
            kl.wr = wr;
            kl.lk[0] = lk[0];
            kl.lk[1] = lk[1];
            kl.lk[2] = lk[2];
            kl.lk[3] = lk[3];
            const double dpr = plev[k - 1] - plev[k - 2];
            s.dpr[k] = dpr;
            kl.u = 3.51e22 * dpr;
            s.tref_v[k] = tauref[k - 1] / (db ? db[NREFV_IDX] : qxv[(size_t)(NREFV_IDX)*LEV1 + k - 1]);
            s.tref_i[k] = tauref[k - 1] / (db ? db[NREFV_IDX] : qxref[k - 1]);
            s.tref_c[k] = cld ? taucld[k - 1] / qxcld[k - 1] : 0.0 / 1.0;
        } else {
            s.tref_i[k] = db ? 0.0 : tauref[k - 1];
            s.tref_c[k] = cld ? taucld[k - 1] : 0.0;
        }
    }
}

// Band items of a column: nitem_v = (NL+1)*7 visible (layer l = 0..NL: level 2
// for l = 0), nitem_i = (NL+1)*5 IR with the Planck terms, then 5 IR boundary
// items.  Needs every level item of the column staged first.
__device__ __forceinline__ int stage_band_items(int L) { return (L + 2) * (D_NV + D_NI) + D_NI; }

__device__ inline void stage_band(const SegDev &sg, int c, const RtConst &K,
                                  const double *__restrict__ planck, ColSmem &s, int it,
                                  uint32_t *status) {
    const int L = sg.L, NL = L + 1, LEV = 2 * L + 3, LEV1 = LEV + 1;
    const double *tlev = sg.tlev + (size_t)c * LEV;
    const bool cld = sg.taurefcld != nullptr;
    const int nitem_v = (NL + 1) * D_NV, nitem_i = (NL + 1) * D_NI;
    {
        if (it < nitem_v) {
            const int l = it / D_NV, nw = it % D_NV + 1;
            // dust properties of level k at qx[(k - 1) * ks] (ks = 0: band constants)
            const double *db = sg.dust_band;
            const int ks = db ? 0 : 1;
            const double *qx = db ? db + nw - 1 : sg.qxvdst + ((size_t)c * D_NV + nw - 1) * LEV1;
            const double *qs = db ? db + D_NV + nw - 1 : sg.qsvdst + ((size_t)c * D_NV + nw - 1) * LEV1;
            const double *gv = db ? db + 2 * D_NV + nw - 1 : sg.gvdst + ((size_t)c * D_NV + nw - 1) * LEV1;
            const double *qxc = cld ? sg.qxvcld + ((size_t)c * D_NV + nw - 1) * LEV1 : nullptr;
            const double *qsc = cld ? sg.qsvcld + ((size_t)c * D_NV + nw - 1) * LEV1 : nullptr;
            const double *gc = cld ? sg.gvcld + ((size_t)c * D_NV + nw - 1) * LEV1 : nullptr;
            const double tr0 = K.tauray[nw - 1];
            auto lvl = [&](int k, double &tr, double &tl, double &tc, double &g1, double &g2) {
                tr = tr0 * s.dpr[k];
                const double taeros = s.tref_v[k] * qx[(k - 1) * ks];
                const double tcloud = s.tref_c[k] * (cld ? qxc[k - 1] : 0.0);
                s.trayaer[k * D_NV + nw - 1] = tr + taeros + tcloud;
                tl = s.tref_v[k] * qs[(k - 1) * ks];
                tc = s.tref_c[k] * (cld ? qsc[k - 1] : 0.0);
                g1 = gv[(k - 1) * ks];
                g2 = cld ? gc[k - 1] : 0.0;
            };
            double tra, tla, tca, ga, gca;
            if (l == 0) {
                lvl(2, tra, tla, tca, ga, gca);
            } else if (l <= L) {
                const int k = 2 * l + 1;
                double trb, tlb, tcb, gb, gcb;
                lvl(k, tra, tla, tca, ga, gca);
                lvl(k + 1, trb, tlb, tcb, gb, gcb);
                const double cb = (ga * tla + gb * tlb + gca * tca + gcb * tcb) / (tra + trb + tla + tlb + tca + tcb);
                s.cosb_v[l * D_NV + nw - 1] = cb;
                s.cbs_v[l * D_NV + nw - 1] = cb / (1.0 + cb);   // code/getdetau.f90:29-56
                s.wnum_v[l * D_NV + nw - 1] = tla + tlb + tca + tcb + (tra + trb) * R4(0.9999);
            } else {
                const int k = LEV;
                lvl(k, tra, tla, tca, ga, gca);
                const double cb = (ga * tla + gca * tca) / (tra + tla + tca);
                s.cosb_v[l * D_NV + nw - 1] = cb;
                s.cbs_v[l * D_NV + nw - 1] = cb / (1.0 + cb);
                s.wnum_v[l * D_NV + nw - 1] = tla + tca + tra * R4(0.9999);
            }
        } else if (it < nitem_v + nitem_i) {
            const int j = it - nitem_v;
            const int l = j / D_NI, nw = j % D_NI + 1;
            const double *db = sg.dust_band;
            const int ks = db ? 0 : 1;
            const double *qx = db ? db + 3 * D_NV + nw - 1 : sg.qxidst + ((size_t)c * D_NI + nw - 1) * LEV1;
            const double *qs = db ? db + 3 * D_NV + D_NI + nw - 1
                                  : sg.qsidst + ((size_t)c * D_NI + nw - 1) * LEV1;
            const double *gi = db ? db + 3 * D_NV + 2 * D_NI + nw - 1
                                  : sg.gidst + ((size_t)c * D_NI + nw - 1) * LEV1;
            const double *qxc = cld ? sg.qxicld + ((size_t)c * D_NI + nw - 1) * LEV1 : nullptr;
            const double *qsc = cld ? sg.qsicld + ((size_t)c * D_NI + nw - 1) * LEV1 : nullptr;
            const double *gc = cld ? sg.gicld + ((size_t)c * D_NI + nw - 1) * LEV1 : nullptr;
            auto ext = [&](int k) {   // TAEROS, TCLOUD at level k <= LEV
                s.taer_i[k * D_NI + nw - 1] = s.tref_i[k] * qx[(k - 1) * ks];
                s.tcld_i[k * D_NI + nw - 1] = s.tref_c[k] * (cld ? qxc[k - 1] : 0.0);
            };
            if (l == 0) {
                ext(2);
            } else {
                const int k = 2 * l + 1;
                ext(k);
                if (k + 1 <= LEV) ext(k + 1);
                const double tla = s.tref_i[k] * qs[(k - 1) * ks], tlb = s.tref_i[k + 1] * qs[k * ks];
                const double tca = s.tref_c[k] * (cld ? qsc[k - 1] : 0.0);
                const double tcb = s.tref_c[k + 1] * (cld ? qsc[k] : 0.0);
                const double tauac = tla + tlb + tca + tcb;
                s.wnum_i[l * D_NI + nw - 1] = tauac;
                double cb = 0.0;
                if (tauac > 0.0)
                    cb = (gi[(k - 1) * ks] * tla + gi[k * ks] * tlb + (cld ? gc[k - 1] : 0.0) * tca +
                          (cld ? gc[k] : 0.0) * tcb) /
                         (tla + tlb + tca + tcb);
                s.cosb_i[l * D_NI + nw - 1] = cb;
                // Planck source terms (gfluxi.f90:219-239)
                int nta, ntb;
                if (l < NL) {
                    ntb = planck_index(tlev[2 * l + 2 - 1], status);
                    nta = planck_index(tlev[2 * l - 1], status);
                    s.pdif_i[l * D_NI + nw - 1] = planck[(ntb - 1) * D_NI + nw - 1] - planck[(nta - 1) * D_NI + nw - 1];
                    s.b0_i[l * D_NI + nw - 1] = planck[(nta - 1) * D_NI + nw - 1];
                } else {
                    nta = planck_index(tlev[2 * l + 1 - 1], status);
                    ntb = planck_index(tlev[2 * l - 1], status);
                    s.pdif_i[l * D_NI + nw - 1] = planck[(nta - 1) * D_NI + nw - 1] - planck[(ntb - 1) * D_NI + nw - 1];
                    s.b0_i[l * D_NI + nw - 1] = planck[(ntb - 1) * D_NI + nw - 1];
                }
            }
        } else {
            // IR boundary terms (sfluxi.f90:51-62)
            const int nw = it - nitem_v - nitem_i + 1;
            const int nts = planck_index(tlev[LEV - 1], status);
            const int ntt = planck_index(tlev[2 - 1], status);
            s.bsurf_i[nw - 1] = (1.0 - sg.albi[c]) * planck[(nts - 1) * D_NI + nw - 1];
            s.pltop_i[nw - 1] = planck[(ntt - 1) * D_NI + nw - 1];
        }
    }
}

// The whole column by one CTA (the fused kernel).
__device__ inline void stage_column(const SegDev &sg, int c, const RtConst &K,
                                    const double *__restrict__ planck, ColSmem &s,
                                    uint32_t *status) {
    const int LEV1 = 2 * sg.L + 4;
    for (int k = 2 + (int)threadIdx.x; k <= LEV1; k += blockDim.x) stage_level(sg, c, K, s, k);
    __syncthreads();
    const int n = stage_band_items(sg.L);
    for (int it = threadIdx.x; it < n; it += blockDim.x) stage_band(sg, c, K, planck, s, it, status);
}

}  // namespace mgcm
