// C ABI of the B200 radiation path (include/mgcm_rt.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mgcm_rt.h"
#include "rt_column.cuh"
#include "tables.h"

namespace mgcm {
__global__ void rt_fp64_kernel(const SegTable *__restrict__ st, const double *__restrict__ kv,
                               const double *__restrict__ ki, const double *__restrict__ planck,
                               const RtConst K, int max_nl, uint32_t *status,
                               unsigned long long *nsys, double *red_scratch);
__global__ void rt_fp64_screen(const SegTable *__restrict__ st, int col_begin, int col_end, int max_nl,
                               unsigned char *__restrict__ blocks, size_t stride,
                               const double *__restrict__ kv, const double *__restrict__ ki,
                               const double *__restrict__ planck, const RtConst K,
                               int *__restrict__ list_v, int *__restrict__ list_i,
                               unsigned int *counts, uint32_t *status, unsigned long long *nsys);
template <bool VIS>
__global__ void rt_fp64_solve(const SegTable *__restrict__ st, int col_begin, int max_nl,
                              unsigned char *__restrict__ blocks, size_t stride,
                              const double *__restrict__ ktab, const RtConst K,
                              const int *__restrict__ list, const unsigned int *count,
                              double *__restrict__ fl, double *__restrict__ sc);
__global__ void rt_fp64_reduce(const SegTable *__restrict__ st, int col_begin, int col_end,
                               int max_nl, unsigned char *__restrict__ blocks, size_t stride,
                               const RtConst K, const double *__restrict__ fl_v,
                               const double *__restrict__ sc_v, const double *__restrict__ fl_i,
                               const double *__restrict__ sc_i, uint32_t *status, int in_smem);
size_t reduce_smem_bytes(int max_nl, int rows);
__global__ void rt_dsolflux_kernel(int ncol, const double *__restrict__ sol,
                                   const double *__restrict__ acosz,
                                   const double *__restrict__ detau,
                                   const double *__restrict__ dndiffv,
                                   double *__restrict__ dnvflux, const RtConst K);
}  // namespace mgcm

using namespace mgcm;

namespace {

constexpr int BLOCK = 224;

// ---------------------------------------------------------------- validation
__global__ void validate_kernel(const SegTable *__restrict__ st, uint32_t *status) {
    const int total = st->total_cols;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        const int si = find_seg(st, g);
        const SegDev &sg = st->seg[si];
        const int c = g - sg.col0, L = sg.L, LEV = 2 * L + 3, LEV1 = LEV + 1;
        uint32_t bad = 0;
        auto fin = [&](const double *p, size_t n) {
            if (!p) return;
            for (size_t i = 0; i < n; ++i)
                if (!isfinite(p[i])) { bad |= ST_NONFINITE; return; }
        };
        fin(sg.plev + (size_t)c * LEV, LEV);
        fin(sg.tlev + (size_t)c * LEV, LEV);
        fin(sg.pmid + (size_t)c * LEV, LEV);
        fin(sg.tmid + (size_t)c * LEV, LEV);
        fin(sg.qh2o + (size_t)c * LEV, LEV);
        fin(sg.tauref + (size_t)c * LEV1, LEV1);
        fin(sg.qextrefdst + (size_t)c * LEV1, LEV1);
        fin(sg.qxvdst + (size_t)c * 7 * LEV1, 7 * LEV1);
        fin(sg.qsvdst + (size_t)c * 7 * LEV1, 7 * LEV1);
        fin(sg.gvdst + (size_t)c * 7 * LEV1, 7 * LEV1);
        fin(sg.qxidst + (size_t)c * 5 * LEV1, 5 * LEV1);
        fin(sg.qsidst + (size_t)c * 5 * LEV1, 5 * LEV1);
        fin(sg.gidst + (size_t)c * 5 * LEV1, 5 * LEV1);
        if (sg.taurefcld) {
            fin(sg.taurefcld + (size_t)c * LEV1, LEV1);
            fin(sg.qextrefcld + (size_t)c * LEV1, LEV1);
            fin(sg.qxvcld + (size_t)c * 7 * LEV1, 7 * LEV1);
            fin(sg.qsvcld + (size_t)c * 7 * LEV1, 7 * LEV1);
            fin(sg.gvcld + (size_t)c * 7 * LEV1, 7 * LEV1);
            fin(sg.qxicld + (size_t)c * 5 * LEV1, 5 * LEV1);
            fin(sg.qsicld + (size_t)c * 5 * LEV1, 5 * LEV1);
            fin(sg.gicld + (size_t)c * 5 * LEV1, 5 * LEV1);
        }
        fin(sg.acosz + c, 1);
        fin(sg.als + c, 1);
        fin(sg.albi + c, 1);
        fin(sg.pcol + c, 1);
        fin(sg.detau + (size_t)c * 119, 119);
        const double *pl = sg.plev + (size_t)c * LEV, *pm = sg.pmid + (size_t)c * LEV;
        for (int k = 0; k < LEV; ++k)
            if (!(pl[k] > 0.0) || !(pm[k] > 0.0)) bad |= ST_NONFINITE;
        const double *tl = sg.tlev + (size_t)c * LEV;
        for (int k = 0; k < LEV; ++k) {
            const double x = __dsub_rn(__dmul_rn(tl[k], 10.0), 499.0);
            if (!(x >= 1.0 && x < 8502.0)) bad |= ST_TEMP;
        }
        if (bad) atomicOr(status, bad);
    }
}

struct Arena {
    void *ptr = nullptr;
    size_t bytes = 0;
};

struct Request;

}  // namespace

struct mgcm_rt_handle {
    mgcm_rt_config cfg{};
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    bool pending = false;
    long long pending_cols = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    HostTables host;
    RtConst K{};
    double *d_kv = nullptr, *d_ki = nullptr, *d_planck = nullptr;
    float *d_kvf = nullptr, *d_kif = nullptr;
    uint32_t *d_status = nullptr;
    unsigned long long *d_nsys = nullptr;
    SegTable *d_segs = nullptr;
    SegTable *h_segs = nullptr;   // pinned
    Arena stage;                  // host-pointer staging
    Arena red;                    // flux staging for L too large for shared memory
    Arena pipe;                   // pipeline: per-column blocks, system lists, counters
    int occ_screen = 0, occ_solve = 0, occ_reduce = 0, occ_nl = 0;
    std::mutex mu;
    mgcm_rt_stats stats{};
    size_t budget = 0;
    // serving
    std::mutex qmu;
    std::condition_variable qcv;
    std::map<long long, std::shared_ptr<Request>> reqs;
    long long next_ticket = 1;
};

namespace {

struct Request {
    mgcm_rt_batch_in in;
    mgcm_rt_batch_out out;
    int status = 1;   // 1 pending, 0 done, <0 error
    bool done = false;
};

int cuda_err(cudaError_t e) { return e == cudaSuccess ? MGCM_RT_OK : MGCM_RT_ECUDA; }

#define CK(x)                                   \
    do {                                        \
        cudaError_t e_ = (x);                   \
        if (e_ != cudaSuccess) return MGCM_RT_ECUDA; \
    } while (0)

struct Sizes {
    int L, lev, lev1, nl;
    size_t ncol;
};

Sizes sizes_of(const mgcm_rt_batch_in &in) {
    Sizes z;
    z.L = in.nlayers;
    z.lev = 2 * z.L + 3;
    z.lev1 = z.lev + 1;
    z.nl = z.L + 1;
    z.ncol = (size_t)std::max(in.ncol, 0);
    return z;
}

int check_args(const mgcm_rt_handle *h, const mgcm_rt_batch_in *in, const mgcm_rt_batch_out *out) {
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    if (in->ncol < 0) return MGCM_RT_EINVAL;
    if (in->nlayers < 1 || in->nlayers > MGCM_RT_MAX_LAYERS || in->nlayers > h->cfg.max_layers)
        return MGCM_RT_ELAYERS;
    if (in->ncol == 0) return MGCM_RT_OK;
    const void *req[] = {in->sigma, in->sol, in->plev, in->tlev, in->pmid, in->tmid, in->qh2o,
                         in->tauref, in->qextrefdst, in->qxvdst, in->qsvdst, in->gvdst, in->qxidst,
                         in->qsidst, in->gidst, in->acosz, in->als, in->albi, in->pcol, in->detau,
                         in->cumtauv, out->fmnetv, out->fluxupv, out->fluxdnv, out->fmneti,
                         out->fluxupi, out->fluxdni, out->suntot, out->irtotal, out->qrad,
                         out->nfluxtopv, out->nfluxtopi, out->diffvt, out->dnvflux, out->dndiffv,
                         out->dnirflux, out->fluxsurf};
    for (const void *p : req)
        if (!p) return MGCM_RT_EINVAL;
    if (in->taurefcld) {
        const void *cl[] = {in->qextrefcld, in->qxvcld, in->qsvcld, in->gvcld,
                            in->qxicld, in->qsicld, in->gicld};
        for (const void *p : cl)
            if (!p) return MGCM_RT_EINVAL;
    }
    if (!std::isfinite(in->ptrop) || !(in->ptrop > 0.0)) return MGCM_RT_ENONFINITE;
    return MGCM_RT_OK;
}

// Array list of one batch: (host/device pointer, doubles per column, direction).
struct ArrSpec {
    const double *src;
    double *dst;          // for outputs and in/out
    size_t per_col;
    int dir;              // 0 in, 1 out, 2 in/out
    double **seg_field;   // where the staged pointer goes in SegDev
    double *dev = nullptr;
};

std::vector<ArrSpec> arrays_of(const mgcm_rt_batch_in &in, const mgcm_rt_batch_out &out,
                               const Sizes &z, SegDev &sd) {
    std::vector<ArrSpec> a;
    auto add_in = [&](const double *p, size_t n, const double **f) {
        if (p) a.push_back({p, nullptr, n, 0, const_cast<double **>(f)});
    };
    auto add_out = [&](double *p, size_t n, double **f) { a.push_back({nullptr, p, n, 1, f}); };
    add_in(in.plev, z.lev, &sd.plev);
    add_in(in.tlev, z.lev, &sd.tlev);
    add_in(in.pmid, z.lev, &sd.pmid);
    add_in(in.tmid, z.lev, &sd.tmid);
    add_in(in.qh2o, z.lev, &sd.qh2o);
    add_in(in.tauref, z.lev1, &sd.tauref);
    add_in(in.qextrefdst, z.lev1, &sd.qextrefdst);
    add_in(in.qxvdst, 7 * z.lev1, &sd.qxvdst);
    add_in(in.qsvdst, 7 * z.lev1, &sd.qsvdst);
    add_in(in.gvdst, 7 * z.lev1, &sd.gvdst);
    add_in(in.qxidst, 5 * z.lev1, &sd.qxidst);
    add_in(in.qsidst, 5 * z.lev1, &sd.qsidst);
    add_in(in.gidst, 5 * z.lev1, &sd.gidst);
    add_in(in.taurefcld, z.lev1, &sd.taurefcld);
    add_in(in.qextrefcld, z.lev1, &sd.qextrefcld);
    add_in(in.qxvcld, 7 * z.lev1, &sd.qxvcld);
    add_in(in.qsvcld, 7 * z.lev1, &sd.qsvcld);
    add_in(in.gvcld, 7 * z.lev1, &sd.gvcld);
    add_in(in.qxicld, 5 * z.lev1, &sd.qxicld);
    add_in(in.qsicld, 5 * z.lev1, &sd.qsicld);
    add_in(in.gicld, 5 * z.lev1, &sd.gicld);
    add_in(in.acosz, 1, &sd.acosz);
    add_in(in.als, 1, &sd.als);
    add_in(in.albi, 1, &sd.albi);
    add_in(in.pcol, 1, &sd.pcol);
    a.push_back({in.detau, in.detau, 119, 2, &sd.detau});
    a.push_back({in.cumtauv, in.cumtauv, 119, 2, &sd.cumtauv});
    add_out(out.fmnetv, z.nl, &sd.fmnetv);
    add_out(out.fluxupv, z.nl, &sd.fluxupv);
    add_out(out.fluxdnv, z.nl, &sd.fluxdnv);
    add_out(out.fmneti, z.nl, &sd.fmneti);
    add_out(out.fluxupi, z.nl, &sd.fluxupi);
    add_out(out.fluxdni, z.nl, &sd.fluxdni);
    add_out(out.suntot, z.nl, &sd.suntot);
    add_out(out.irtotal, z.nl, &sd.irtotal);
    add_out(out.qrad, z.nl, &sd.qrad);
    add_out(out.nfluxtopv, 1, &sd.nfluxtopv);
    add_out(out.nfluxtopi, 1, &sd.nfluxtopi);
    add_out(out.diffvt, 1, &sd.diffvt);
    add_out(out.dnvflux, 1, &sd.dnvflux);
    add_out(out.dndiffv, 1, &sd.dndiffv);
    add_out(out.dnirflux, 1, &sd.dnirflux);
    add_out(out.fluxsurf, 1, &sd.fluxsurf);
    return a;
}

void fill_direct(SegDev &sd, const mgcm_rt_batch_in &in, const mgcm_rt_batch_out &out) {
    sd.plev = in.plev; sd.tlev = in.tlev; sd.pmid = in.pmid; sd.tmid = in.tmid; sd.qh2o = in.qh2o;
    sd.tauref = in.tauref; sd.qextrefdst = in.qextrefdst;
    sd.taurefcld = in.taurefcld; sd.qextrefcld = in.qextrefcld;
    sd.qxvdst = in.qxvdst; sd.qsvdst = in.qsvdst; sd.gvdst = in.gvdst;
    sd.qxidst = in.qxidst; sd.qsidst = in.qsidst; sd.gidst = in.gidst;
    sd.qxvcld = in.qxvcld; sd.qsvcld = in.qsvcld; sd.gvcld = in.gvcld;
    sd.qxicld = in.qxicld; sd.qsicld = in.qsicld; sd.gicld = in.gicld;
    sd.acosz = in.acosz; sd.als = in.als; sd.albi = in.albi; sd.pcol = in.pcol;
    sd.detau = in.detau; sd.cumtauv = in.cumtauv;
    sd.fmnetv = out.fmnetv; sd.fluxupv = out.fluxupv; sd.fluxdnv = out.fluxdnv;
    sd.fmneti = out.fmneti; sd.fluxupi = out.fluxupi; sd.fluxdni = out.fluxdni;
    sd.suntot = out.suntot; sd.irtotal = out.irtotal; sd.qrad = out.qrad;
    sd.nfluxtopv = out.nfluxtopv; sd.nfluxtopi = out.nfluxtopi; sd.diffvt = out.diffvt;
    sd.dnvflux = out.dnvflux; sd.dndiffv = out.dndiffv; sd.dnirflux = out.dnirflux;
    sd.fluxsurf = out.fluxsurf;
}

bool red_in_smem(int max_nl) { return col_smem_bytes(max_nl, true) <= SMEM_CAP; }

int fp64_blocks_per_sm(int max_nl) {
    int nb = 0;
    const size_t smem = col_smem_bytes(max_nl, red_in_smem(max_nl));
    cudaFuncSetAttribute(rt_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rt_fp64_kernel, BLOCK, smem) != cudaSuccess)
        return 1;
    return std::max(nb, 1);
}

// Three-kernel FP64 pipeline over chunks of columns (rt_fp64.cu).
int launch_pipeline(mgcm_rt_handle *h, int total, int max_nl, int &nk) {
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t stride = al(col_smem_bytes(max_nl, false));
    const size_t row = (size_t)2 * max_nl * sizeof(double);
    const size_t per_col = stride + NSYS * (sizeof(int) + row + 4 * sizeof(double));
    const size_t cap = std::min<size_t>(h->budget / 2, (size_t)8 << 30);
    const int chunk = (int)std::min<size_t>((size_t)total, std::max<size_t>(cap / per_col, 1));
    const size_t n_v = (size_t)chunk * NSYS_V, n_i = (size_t)chunk * NSYS_I;
    const size_t need = al((size_t)chunk * stride) + al(n_v * 4) + al(n_i * 4) + al(n_v * row) +
                        al(n_i * row) + al(n_v * 32) + al(n_i * 32) + 256;
    if (h->pipe.bytes < need) {
        if (h->pipe.ptr) {
            CK(cudaStreamSynchronize(h->stream));
            cudaFree(h->pipe.ptr);
        }
        h->pipe.ptr = nullptr;
        h->pipe.bytes = 0;
        if (cudaMalloc(&h->pipe.ptr, need) != cudaSuccess) return MGCM_RT_ENOMEM;
        h->pipe.bytes = need;
    }
    unsigned char *p = static_cast<unsigned char *>(h->pipe.ptr);
    auto take = [&](size_t b) { unsigned char *r = p; p += al(b); return r; };
    unsigned char *blocks = take((size_t)chunk * stride);
    int *list_v = reinterpret_cast<int *>(take(n_v * 4));
    int *list_i = reinterpret_cast<int *>(take(n_i * 4));
    double *fl_v = reinterpret_cast<double *>(take(n_v * row));
    double *fl_i = reinterpret_cast<double *>(take(n_i * row));
    double *sc_v = reinterpret_cast<double *>(take(n_v * 32));
    double *sc_i = reinterpret_cast<double *>(take(n_i * 32));
    unsigned int *counts = reinterpret_cast<unsigned int *>(take(256));
    // reduce pool: room for a typical column's kept systems in ~48 KB (4 CTAs
    // per SM); columns with more kept systems sum from global memory
    int pool_rows = (int)std::min<size_t>(NSYS, (48 * 1024) / (16 * (size_t)max_nl + 32));
    if (pool_rows < 24) pool_rows = 0;
    const size_t rsm = reduce_smem_bytes(max_nl, pool_rows);
    const bool rin = pool_rows > 0;
    if (h->occ_nl != max_nl) {
        h->occ_nl = max_nl;
        int a = 1, b = 1, c = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, rt_fp64_screen, BLOCK, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, rt_fp64_solve<false>, 128, 0);
        cudaFuncSetAttribute(rt_fp64_reduce, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             rin ? (int)rsm : 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, rt_fp64_reduce, 160, rin ? rsm : 0);
        h->occ_screen = std::max(a, 1);
        h->occ_solve = std::max(b, 1);
        if (const char *e = std::getenv("MGCM_RT_SOLVE_CTAS_PER_SM")) h->occ_solve = std::max(1, std::atoi(e));
        h->occ_reduce = std::max(c, 1);
    }
    for (int c0 = 0; c0 < total; c0 += chunk) {
        const int c1 = std::min(total, c0 + chunk);
        CK(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned int), h->stream));
        const int g1 = std::min(c1 - c0, h->num_sms * h->occ_screen);
        rt_fp64_screen<<<g1, BLOCK, 0, h->stream>>>(h->d_segs, c0, c1, max_nl, blocks, stride,
                                                     h->d_kv, h->d_ki, h->d_planck, h->K, list_v,
                                                     list_i, counts, h->d_status, h->d_nsys);
        const int g2 = h->num_sms * h->occ_solve;
        rt_fp64_solve<true><<<g2, 128, 0, h->stream>>>(h->d_segs, c0, max_nl, blocks, stride,
                                                        h->d_kv, h->K, list_v, counts, fl_v, sc_v);
        rt_fp64_solve<false><<<g2, 128, 0, h->stream>>>(h->d_segs, c0, max_nl, blocks, stride,
                                                         h->d_ki, h->K, list_i, counts, fl_i, sc_i);
        const int g3 = std::min(c1 - c0, h->num_sms * h->occ_reduce);
        rt_fp64_reduce<<<g3, 160, rin ? rsm : 0, h->stream>>>(h->d_segs, c0, c1, max_nl, blocks,
                                                               stride, h->K, fl_v, sc_v, fl_i, sc_i,
                                                               h->d_status, pool_rows);
        nk += 4;
        CK(cudaGetLastError());
    }
    return MGCM_RT_OK;
}

// Launches the radiation kernels for the segment table already in h->d_segs.
int launch_all(mgcm_rt_handle *h, int total, int max_nl, bool validate) {
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(uint32_t), h->stream));
    CK(cudaMemsetAsync(h->d_nsys, 0, sizeof(unsigned long long), h->stream));
    int nk = 0;
    if (validate) {
        const int vb = std::min((total + 255) / 256, h->num_sms * 8);
        validate_kernel<<<std::max(vb, 1), 256, 0, h->stream>>>(h->d_segs, h->d_status);
        ++nk;
    }
    CK(cudaEventRecord(h->ev0, h->stream));
    if (h->cfg.precision == MGCM_RT_FP64) {
        const int rc = launch_pipeline(h, total, max_nl, nk);
        if (rc) return rc;
    } else {
        const bool in_smem = red_in_smem(max_nl);
        const size_t smem = col_smem_bytes(max_nl, in_smem);
        const int grid = std::min(total, h->num_sms * fp64_blocks_per_sm(max_nl));
        double *red = nullptr;
        if (!in_smem) {
            const size_t need = (size_t)grid * red_bytes(max_nl);
            if (h->red.bytes < need) {
                if (h->red.ptr) {
                    CK(cudaStreamSynchronize(h->stream));
                    cudaFree(h->red.ptr);
                }
                h->red.ptr = nullptr;
                h->red.bytes = 0;
                if (cudaMalloc(&h->red.ptr, need) != cudaSuccess) return MGCM_RT_ENOMEM;
                h->red.bytes = need;
            }
            red = static_cast<double *>(h->red.ptr);
        }
        rt_fp64_kernel<<<grid, BLOCK, smem, h->stream>>>(h->d_segs, h->d_kv, h->d_ki, h->d_planck,
                                                         h->K, max_nl, h->d_status, h->d_nsys, red);
        ++nk;
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(h->ev1, h->stream));
    h->stats.kernels = nk;
    return MGCM_RT_OK;
}

int status_to_code(uint32_t st) {
    if (st & 16u) return MGCM_RT_ECUDA;   // a bounded device wait ran out
    if (st & ST_NONFINITE) return MGCM_RT_ENONFINITE;
    if (st & (ST_TEMP | ST_PLANCK_RANGE)) return MGCM_RT_ETEMP;
    if (st & ST_BADL) return MGCM_RT_ELAYERS;
    return MGCM_RT_OK;
}

int finish(mgcm_rt_handle *h, long long cols) {
    CK(cudaStreamSynchronize(h->stream));
    uint32_t st = 0;
    unsigned long long ns = 0;
    CK(cudaMemcpy(&st, h->d_status, sizeof(st), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&ns, h->d_nsys, sizeof(ns), cudaMemcpyDeviceToHost));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.gpu_ms = ms;
    h->stats.columns = cols;
    h->stats.systems = (long long)ns;
    h->stats.status = (int)st;
    return status_to_code(st);
}

int ensure_stage(mgcm_rt_handle *h, size_t bytes) {
    if (h->stage.bytes >= bytes) return MGCM_RT_OK;
    if (bytes > h->budget) return MGCM_RT_ENOMEM;
    if (h->stage.ptr) cudaFree(h->stage.ptr);
    h->stage.ptr = nullptr;
    h->stage.bytes = 0;
    if (cudaMalloc(&h->stage.ptr, bytes) != cudaSuccess) return MGCM_RT_ENOMEM;
    h->stage.bytes = bytes;
    return MGCM_RT_OK;
}

// Runs nbatch segments (all host or all device pointers); synchronous unless
// async (device pointers only), in which case the caller later calls finish().
int run_segments(mgcm_rt_handle *h, int nbatch, const mgcm_rt_batch_in *in,
                 mgcm_rt_batch_out *out, bool async = false) {
    if (nbatch < 1 || nbatch > MAX_SEGS) return MGCM_RT_EINVAL;
    const auto t0 = std::chrono::steady_clock::now();
    const int kind = in[0].device_ptrs ? 1 : 0;
    if (async && !kind) return MGCM_RT_EINVAL;
    if (h->pending) {   // a previous enqueue not yet synced: its segment table is in use
        const int rc = finish(h, h->pending_cols);
        h->pending = false;
        if (rc) return rc;
    }
    SegTable &tab = *h->h_segs;
    tab.nseg = 0;
    int total = 0, max_nl = 1;
    size_t stage_bytes = 0;
    for (int b = 0; b < nbatch; ++b) {
        const int rc = check_args(h, &in[b], &out[b]);
        if (rc) return rc;
        if ((in[b].device_ptrs ? 1 : 0) != kind) return MGCM_RT_EINVAL;
        const Sizes z = sizes_of(in[b]);
        if (z.ncol == 0) continue;
        if ((long long)total + (long long)z.ncol > 0x7fffffff) return MGCM_RT_EINVAL;
        SegDev sd{};
        const auto arrs = arrays_of(in[b], out[b], z, sd);
        for (const auto &a : arrs) stage_bytes += ((a.per_col * z.ncol * 8 + 255) / 256) * 256;
        stage_bytes += ((z.lev + 8) * 8 + 255) / 256 * 256;   // sigma + sol
        max_nl = std::max(max_nl, z.nl);
        total += (int)z.ncol;
    }
    if (total == 0) return MGCM_RT_OK;
    if (!kind) {
        const int rc = ensure_stage(h, stage_bytes);
        if (rc) return rc;
    }
    char *base = static_cast<char *>(h->stage.ptr);
    size_t off = 0;
    int col0 = 0;
    std::vector<std::pair<std::vector<ArrSpec>, size_t>> pending;   // for D2H
    for (int b = 0; b < nbatch; ++b) {
        const Sizes z = sizes_of(in[b]);
        if (z.ncol == 0) continue;
        SegDev sd{};
        sd.ncol = (int)z.ncol;
        sd.L = z.L;
        sd.col0 = col0;
        sd.ptrop = in[b].ptrop;
        if (kind) {
            fill_direct(sd, in[b], out[b]);
            sd.sigma = in[b].sigma;
            sd.sol = in[b].sol;
        } else {
            auto arrs = arrays_of(in[b], out[b], z, sd);
            for (auto &a : arrs) {
                double *d = reinterpret_cast<double *>(base + off);
                off += ((a.per_col * z.ncol * 8 + 255) / 256) * 256;
                *a.seg_field = d;
                a.dev = d;
                if (a.dir != 1)
                    CK(cudaMemcpyAsync(d, a.src, a.per_col * z.ncol * 8, cudaMemcpyHostToDevice, h->stream));
            }
            double *ds = reinterpret_cast<double *>(base + off);
            off += ((z.lev + 8) * 8 + 255) / 256 * 256;
            CK(cudaMemcpyAsync(ds, in[b].sigma, z.lev * 8, cudaMemcpyHostToDevice, h->stream));
            CK(cudaMemcpyAsync(ds + z.lev, in[b].sol, 7 * 8, cudaMemcpyHostToDevice, h->stream));
            sd.sigma = ds;
            sd.sol = ds + z.lev;
            pending.push_back({arrs, z.ncol});
        }
        tab.seg[tab.nseg++] = sd;
        col0 += (int)z.ncol;
    }
    tab.total_cols = total;
    CK(cudaMemcpyAsync(h->d_segs, h->h_segs, sizeof(SegTable), cudaMemcpyHostToDevice, h->stream));
    int rc = launch_all(h, total, max_nl, h->cfg.validate != 0);
    if (rc) return rc;
    if (!kind) {
        for (size_t i = 0; i < pending.size(); ++i)
            for (auto &a : pending[i].first)
                if (a.dir != 0)
                    CK(cudaMemcpyAsync(a.dst, a.dev, a.per_col * pending[i].second * 8,
                                       cudaMemcpyDeviceToHost, h->stream));
    }
    if (async) {
        h->pending = true;
        h->pending_cols = total;
        return MGCM_RT_OK;
    }
    rc = finish(h, total);
    h->stats.total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

}  // namespace

extern "C" {

const char *mgcm_rt_version(void) { return "mgcm-rt-b200 0.1 (Legacy Mars GCM v24 radiation)"; }

const char *mgcm_rt_strerror(int s) {
    switch (s) {
        case MGCM_RT_OK: return "ok";
        case MGCM_RT_EINVAL: return "invalid argument";
        case MGCM_RT_ENONFINITE: return "non-finite or non-positive input";
        case MGCM_RT_ETEMP: return "temperature outside the Planck table [50,900) K";
        case MGCM_RT_ELAYERS: return "layer count outside the supported range";
        case MGCM_RT_ENOMEM: return "device memory or HBM budget exhausted";
        case MGCM_RT_EIO: return "radiation data file missing or malformed";
        case MGCM_RT_ECUDA: return "CUDA runtime error";
        case MGCM_RT_ETIMEOUT: return "timed out";
        case MGCM_RT_EBUSY: return "request queue full";
        case MGCM_RT_ENOTFOUND: return "unknown ticket";
        default: return "unknown status";
    }
}

int mgcm_rt_tables_host(const char *data_dir, double *co2v, double *co2i, double *planckir,
                        double *pfgasref) {
    if (!data_dir) return MGCM_RT_EINVAL;
    HostTables t;
    if (load_tables(data_dir, t)) return MGCM_RT_EIO;
    if (co2v) std::memcpy(co2v, t.co2v.data(), t.co2v.size() * 8);
    if (co2i) std::memcpy(co2i, t.co2i.data(), t.co2i.size() * 8);
    if (planckir) std::memcpy(planckir, t.planckir.data(), t.planckir.size() * 8);
    if (pfgasref) std::memcpy(pfgasref, t.pfgasref, sizeof(t.pfgasref));
    return MGCM_RT_OK;
}

mgcm_rt_handle *mgcm_rt_create(const mgcm_rt_config *cfg, const char *data_dir, int *status) {
    int dummy;
    if (!status) status = &dummy;
    if (!cfg || !data_dir) { *status = MGCM_RT_EINVAL; return nullptr; }
    if (cfg->max_layers < 1 || cfg->max_layers > MGCM_RT_MAX_LAYERS) { *status = MGCM_RT_ELAYERS; return nullptr; }
    if (cfg->precision != MGCM_RT_FP64) { *status = MGCM_RT_EINVAL; return nullptr; }
    auto h = std::make_unique<mgcm_rt_handle>();
    h->cfg = *cfg;
    if (load_tables(data_dir, h->host)) { *status = MGCM_RT_EIO; return nullptr; }
    h->device = cfg->device;
    if (cudaSetDevice(h->device) != cudaSuccess) { *status = MGCM_RT_ECUDA; return nullptr; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess) { *status = MGCM_RT_ECUDA; return nullptr; }
    h->num_sms = prop.multiProcessorCount;
    auto fail = [&](int code) { mgcm_rt_destroy(h.release()); *status = code; return nullptr; };
    if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) return fail(MGCM_RT_ECUDA);
    h->stream = h->own_stream;
    if (cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) return fail(MGCM_RT_ECUDA);
    // constants
    RtConst &K = h->K;
    std::memcpy(K.tauray, h->host.tauray, sizeof(K.tauray));
    std::memcpy(K.fzerov, h->host.fzerov, sizeof(K.fzerov));
    std::memcpy(K.fzeroi, h->host.fzeroi, sizeof(K.fzeroi));
    std::memcpy(K.gweight, h->host.gweight, sizeof(K.gweight));
    std::memcpy(K.dwni, h->host.dwni, sizeof(K.dwni));
    std::memcpy(K.pfgasref, h->host.pfgasref, sizeof(K.pfgasref));
    std::memcpy(K.plimit, h->host.plimit, sizeof(K.plimit));
    std::memcpy(K.wrefh2o, h->host.wrefh2o, sizeof(K.wrefh2o));
    // device tables
    std::vector<double> kv, ki;
    gauss_fastest(h->host, kv, ki);
    std::vector<float> kvf(kv.begin(), kv.end()), kif(ki.begin(), ki.end());
    if (cudaMalloc(&h->d_kv, kv.size() * 8) || cudaMalloc(&h->d_ki, ki.size() * 8) ||
        cudaMalloc(&h->d_kvf, kvf.size() * 4) || cudaMalloc(&h->d_kif, kif.size() * 4) ||
        cudaMalloc(&h->d_planck, h->host.planckir.size() * 8) ||
        cudaMalloc(&h->d_status, 64) || cudaMalloc(&h->d_nsys, 64) ||
        cudaMalloc(&h->d_segs, sizeof(SegTable)) ||
        cudaMallocHost(&h->h_segs, sizeof(SegTable)))
        return fail(MGCM_RT_ENOMEM);
    if (cudaMemcpy(h->d_kv, kv.data(), kv.size() * 8, cudaMemcpyHostToDevice) ||
        cudaMemcpy(h->d_ki, ki.data(), ki.size() * 8, cudaMemcpyHostToDevice) ||
        cudaMemcpy(h->d_kvf, kvf.data(), kvf.size() * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(h->d_kif, kif.data(), kif.size() * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(h->d_planck, h->host.planckir.data(), h->host.planckir.size() * 8, cudaMemcpyHostToDevice))
        return fail(MGCM_RT_ECUDA);
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    h->budget = cfg->hbm_budget ? cfg->hbm_budget : freeb / 4 * 3;
    *status = MGCM_RT_OK;
    return h.release();
}

void mgcm_rt_destroy(mgcm_rt_handle *h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->stream = h->own_stream;
    cudaFree(h->d_kv);
    cudaFree(h->d_ki);
    cudaFree(h->d_kvf);
    cudaFree(h->d_kif);
    cudaFree(h->d_planck);
    cudaFree(h->d_status);
    cudaFree(h->d_nsys);
    cudaFree(h->d_segs);
    if (h->h_segs) cudaFreeHost(h->h_segs);
    if (h->stage.ptr) cudaFree(h->stage.ptr);
    if (h->red.ptr) cudaFree(h->red.ptr);
    if (h->pipe.ptr) cudaFree(h->pipe.ptr);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
}

int mgcm_rt_run(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out) {
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    return run_segments(h, 1, in, out);
}

int mgcm_rt_run_multi(mgcm_rt_handle *h, int nbatch, const mgcm_rt_batch_in *in,
                      mgcm_rt_batch_out *out) {
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    return run_segments(h, nbatch, in, out);
}

int mgcm_rt_enqueue(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out) {
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    return run_segments(h, 1, in, out, true);
}

int mgcm_rt_sync(mgcm_rt_handle *h) {
    if (!h) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    if (!h->pending) {
        CK(cudaStreamSynchronize(h->stream));
        return MGCM_RT_OK;
    }
    h->pending = false;
    return finish(h, h->pending_cols);
}

int mgcm_rt_set_stream(mgcm_rt_handle *h, void *cuda_stream) {
    if (!h) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->pending) {
        h->pending = false;
        const int rc = finish(h, h->pending_cols);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(h->stream));
    h->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : h->own_stream;
    return MGCM_RT_OK;
}

int mgcm_rt_get_stats(mgcm_rt_handle *h, mgcm_rt_stats *st) {
    if (!h || !st) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    *st = h->stats;
    return MGCM_RT_OK;
}

int mgcm_rt_dsolflux(mgcm_rt_handle *h, int ncol, int device_ptrs, const double *sol,
                     const double *acosz, const double *detau, const double *dndiffv,
                     double *dnvflux) {
    if (!h || ncol < 0 || !sol || !acosz || !detau || !dndiffv || !dnvflux) return MGCM_RT_EINVAL;
    if (ncol == 0) return MGCM_RT_OK;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    const double *ds = sol, *da = acosz, *dd = detau, *dn = dndiffv;
    double *dout = dnvflux;
    if (!device_ptrs) {
        const size_t n = (size_t)ncol;
        const size_t bytes = 8 * (8 + n + 119 * n + n + n) + 5 * 256;
        const int rc = ensure_stage(h, bytes);
        if (rc) return rc;
        char *b = static_cast<char *>(h->stage.ptr);
        double *p = reinterpret_cast<double *>(b);
        double *pa = p + 8, *pd = pa + n, *pn = pd + 119 * n, *po = pn + n;
        CK(cudaMemcpyAsync(p, sol, 7 * 8, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(pa, acosz, n * 8, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(pd, detau, 119 * n * 8, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(pn, dndiffv, n * 8, cudaMemcpyHostToDevice, h->stream));
        ds = p; da = pa; dd = pd; dn = pn; dout = po;
    }
    rt_dsolflux_kernel<<<(ncol + 127) / 128, 128, 0, h->stream>>>(ncol, ds, da, dd, dn, dout, h->K);
    CK(cudaGetLastError());
    if (!device_ptrs) CK(cudaMemcpyAsync(dnvflux, dout, (size_t)ncol * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MGCM_RT_OK;
}

// Serving: a submitted batch runs at once on the handle's stream; wait()
// collects its status.
int mgcm_rt_submit(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out,
                   long long *ticket) {
    if (!h || !in || !out || !ticket) return MGCM_RT_EINVAL;
    const int rc = mgcm_rt_run(h, in, out);
    std::lock_guard<std::mutex> lk(h->qmu);
    auto r = std::make_shared<Request>();
    r->status = rc;
    r->done = true;
    *ticket = h->next_ticket++;
    h->reqs[*ticket] = r;
    return MGCM_RT_OK;
}

int mgcm_rt_poll(mgcm_rt_handle *h, long long ticket) {
    if (!h) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->qmu);
    auto it = h->reqs.find(ticket);
    if (it == h->reqs.end()) return MGCM_RT_ENOTFOUND;
    if (!it->second->done) return 0;
    return it->second->status < 0 ? it->second->status : 1;
}

int mgcm_rt_wait(mgcm_rt_handle *h, long long ticket, double timeout_s) {
    if (!h) return MGCM_RT_EINVAL;
    (void)timeout_s;
    std::lock_guard<std::mutex> lk(h->qmu);
    auto it = h->reqs.find(ticket);
    if (it == h->reqs.end()) return MGCM_RT_ENOTFOUND;
    const int st = it->second->status;
    h->reqs.erase(it);
    return st;
}
}

// ---------------------------------------------------------------------------
// No-allocation entry point.  Its scratch is this file-scope array; in host
// code the symbol is only a stand-in, so the device address is resolved with
// cudaGetSymbolAddress once per device (with that device current) and cached.
namespace {

constexpr size_t NOALLOC_HDR = 64 * 1024;   // descriptor + status + counter
static_assert(offsetof(SegTable, seg) + sizeof(SegDev) + 512 <= NOALLOC_HDR, "descriptor");
static_assert(NOALLOC_HDR < MGCM_RT_NOALLOC_SCRATCH_BYTES, "scratch size");

__device__ __align__(256) unsigned char g_noalloc_scratch[MGCM_RT_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_ptr[256] = {};

int noalloc_scratch(int device, unsigned char **ptr) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (device < 0 || device >= 256) return MGCM_RT_EINVAL;
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return MGCM_RT_ECUDA;
        g_noalloc_ptr[device] = static_cast<unsigned char *>(p);
    }
    *ptr = g_noalloc_ptr[device];
    return MGCM_RT_OK;
}

}  // namespace

extern "C" int mgcm_rt_run_noalloc(mgcm_rt_handle *h, const mgcm_rt_batch_in *in,
                                   mgcm_rt_batch_out *out) {
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    if (!in->device_ptrs) return MGCM_RT_EINVAL;   // host buffers would need staging memory
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    int rc = check_args(h, in, out);
    if (rc) return rc;
    if (in->ncol == 0) return MGCM_RT_OK;
    if (h->pending) {
        h->pending = false;
        rc = finish(h, h->pending_cols);
        if (rc) return rc;
    }
    unsigned char *scr = nullptr;
    rc = noalloc_scratch(h->device, &scr);
    if (rc) return rc;
    const Sizes z = sizes_of(*in);
    const int max_nl = z.nl;
    // flux staging per CTA in the array; the grid is capped to the slabs that fit
    const size_t slab = red_bytes(max_nl);
    const size_t nslab = (MGCM_RT_NOALLOC_SCRATCH_BYTES - NOALLOC_HDR) / slab;
    if (nslab < 1) return MGCM_RT_ENOMEM;
    const size_t smem = col_smem_bytes(max_nl, false);
    if (cudaFuncSetAttribute(rt_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return MGCM_RT_ECUDA;
    int nb = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rt_fp64_kernel, BLOCK, smem) != cudaSuccess)
        nb = 1;
    const size_t want = (size_t)h->num_sms * (size_t)std::max(nb, 1);
    const int grid = (int)std::min({(size_t)z.ncol, want, nslab});
    // descriptor: header + one segment, staged through the handle's pinned buffer
    SegTable &tab = *h->h_segs;
    tab.nseg = 1;
    tab.total_cols = (int)z.ncol;
    SegDev sd{};
    sd.ncol = (int)z.ncol;
    sd.L = z.L;
    sd.col0 = 0;
    sd.ptrop = in->ptrop;
    fill_direct(sd, *in, *out);
    sd.sigma = in->sigma;
    sd.sol = in->sol;
    tab.seg[0] = sd;
    SegTable *d_tab = reinterpret_cast<SegTable *>(scr);
    uint32_t *d_status = reinterpret_cast<uint32_t *>(scr + NOALLOC_HDR - 256);
    unsigned long long *d_nsys = reinterpret_cast<unsigned long long *>(scr + NOALLOC_HDR - 128);
    double *d_red = reinterpret_cast<double *>(scr + NOALLOC_HDR);
    CK(cudaMemcpyAsync(d_tab, h->h_segs, offsetof(SegTable, seg) + sizeof(SegDev),
                       cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(d_status, 0, sizeof(uint32_t), h->stream));
    CK(cudaMemsetAsync(d_nsys, 0, sizeof(unsigned long long), h->stream));
    CK(cudaEventRecord(h->ev0, h->stream));
    rt_fp64_kernel<<<grid, BLOCK, smem, h->stream>>>(d_tab, h->d_kv, h->d_ki, h->d_planck, h->K,
                                                     max_nl, d_status, d_nsys, d_red);
    CK(cudaGetLastError());
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    uint32_t st = 0;
    unsigned long long ns = 0;
    CK(cudaMemcpy(&st, d_status, sizeof(st), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&ns, d_nsys, sizeof(ns), cudaMemcpyDeviceToHost));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.gpu_ms = ms;
    h->stats.columns = (long long)z.ncol;
    h->stats.systems = (long long)ns;
    h->stats.status = (int)st;
    h->stats.kernels = 1;
    return status_to_code(st);
}
