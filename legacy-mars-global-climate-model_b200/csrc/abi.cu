// C ABI of the B200 radiation path (include/mgcm_rt.h): handles, slots,
// the synchronous and asynchronous batch calls and the serving queue.
//
// A slot is one CUDA stream with its own staging (host-pointer batches),
// pipeline scratch, segment descriptor and status words.  A job is up to one
// slot's worth of columns from one batch.  Synchronous calls with host
// buffers run their jobs on two slots alternately so copies of one job
// overlap the kernels of the other; served requests are split into jobs that
// a worker thread admits onto free slots as memory and slots free up, so
// work from different requests overlaps on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstddef>
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
#include "rt_aerosol.cuh"
#include "rt_prep.cuh"
#include "rt_column.cuh"
#include "tables.h"
#include <nvtx3/nvToolsExt.h>

namespace mgcm {
__global__ void rt_fp64_kernel(const SegTable *__restrict__ st, const double *__restrict__ kv,
                               const double *__restrict__ ki, const double *__restrict__ planck,
                               const RtConst K, int max_nl, uint32_t *status,
                               unsigned long long *nsys, double *red_scratch);
__global__ void rt_stage(const SegTable *__restrict__ st, int col_begin, int col_end, int max_nl,
                         unsigned char *__restrict__ blocks, size_t stride,
                         const double *__restrict__ planck, const RtConst K, uint32_t *status);
template <bool F32>
__global__ void rt_fp64_screen(const SegTable *__restrict__ st, int col_begin, int col_end, int max_nl,
                               unsigned char *__restrict__ blocks, size_t stride,
                               const double *__restrict__ kv, const double *__restrict__ ki,
                               const RtConst K, int *__restrict__ list_v, int *__restrict__ list_i,
                               unsigned int *counts, unsigned long long *nsys,
                               const float *__restrict__ kvf);
template <bool VIS>
__global__ void rt_fp64_solve(const SegTable *__restrict__ st, int col_begin, int max_nl,
                              unsigned char *__restrict__ blocks, size_t stride,
                              const double *__restrict__ ktab, const RtConst K,
                              const int *__restrict__ list, const unsigned int *count,
                              double *__restrict__ fl, double *__restrict__ sc);
template <bool VIS, int R>
__global__ void rt_quad_solve(const SegTable *__restrict__ st, int col_begin, int max_nl,
                              unsigned char *__restrict__ blocks, size_t stride,
                              const double *__restrict__ ktab, const RtConst K, const int *__restrict__ list,
                              const unsigned int *count, double *__restrict__ fl, double *__restrict__ sc);
template <int R>
__global__ void rt_quad_mixed_vis(const SegTable *__restrict__ st, int col_begin, int max_nl,
                                  unsigned char *__restrict__ blocks, size_t stride,
                                  const float *__restrict__ ktabf, const double *__restrict__ ktab,
                                  const RtConst K, const int *__restrict__ list, const unsigned int *count,
                                  double *__restrict__ fl, double *__restrict__ sc);
__global__ void rt_mixed_solve_vis(const SegTable *__restrict__ st, int col_begin, int max_nl,
                                   unsigned char *__restrict__ blocks, size_t stride,
                                   const float *__restrict__ ktabf, const double *__restrict__ ktab,
                                   const RtConst K, const int *__restrict__ list,
                                   const unsigned int *count, double *__restrict__ fl,
                                   double *__restrict__ sc);
template <bool ONE_LEVEL, int RB>
__global__ void rt_fp64_reduce(const SegTable *__restrict__ st, int col_begin, int col_end,
                               int max_nl, unsigned char *__restrict__ blocks, size_t stride,
                               const RtConst K, const double *__restrict__ fl_v,
                               const double *__restrict__ sc_v, const double *__restrict__ fl_i,
                               const double *__restrict__ sc_i);
size_t reduce_smem_bytes(int max_nl, int rb);
const void *reduce_kernel(int max_nl, int rb);
constexpr int REDUCE_WARPS = 4, REDUCE_THREADS = 32 * REDUCE_WARPS;   // rt_fp64_reduce: warp per column
constexpr int STAGE_THREADS = 256, SCREEN_THREADS = 128;
int reduce_rows_per_chunk(int max_nl);
__global__ void rt_dsolflux_kernel(int ncol, const double *__restrict__ sol,
                                   const double *__restrict__ acosz,
                                   const double *__restrict__ detau,
                                   const double *__restrict__ dndiffv,
                                   double *__restrict__ dnvflux, const RtConst K);
template <bool VIS, bool F32, int T>
__global__ void rt_solve_oc(const SegTable *__restrict__ st, int col_begin, int max_nl,
                            unsigned char *__restrict__ blocks, size_t stride, const double *__restrict__ ktab,
                            const float *__restrict__ ktabf, const RtConst K, const int *__restrict__ list,
                            const unsigned int *count, double *__restrict__ fl, double *__restrict__ sc);
template <bool VIS, bool F32, int W>
__global__ void rt_solve_tm(const SegTable *__restrict__ st, int col_begin, int max_nl,
                            unsigned char *__restrict__ blocks, size_t stride, const double *__restrict__ ktab,
                            const float *__restrict__ ktabf, const RtConst K, const int *__restrict__ list,
                            const unsigned int *count, double *__restrict__ fl, double *__restrict__ sc);
template <bool F32, int TC, int THREADS, int MINB>
__global__ void rt_fused(const SegTable *__restrict__ st, int ncols, int max_nl, unsigned char *__restrict__ scratch,
                         size_t cta_bytes, size_t stride, const double *__restrict__ kv,
                         const double *__restrict__ ki, const float *__restrict__ kvf,
                         const double *__restrict__ planck, const RtConst K, unsigned int *tile_ctr,
                         uint32_t *status, unsigned long long *nsys);
size_t fused_smem(int warps, int tc);
size_t fused_scratch_per_cta(int tc, int max_nl, size_t stride);
__global__ void rt_bins_decode(const SegTable *__restrict__ st, int ncol, int max_nl,
                               const unsigned char *__restrict__ blocks, size_t stride,
                               uint32_t *status, int *__restrict__ mt, int *__restrict__ mp,
                               int *__restrict__ nh, int *__restrict__ npl, double *__restrict__ wr,
                               double *__restrict__ lk);
}  // namespace mgcm

using namespace mgcm;

namespace {

// NVTX range for the duration of a scope: each entry point, each job a slot
// issues and each graph replay shows up by name in a timeline profiler
// (header-only NVTX 3; a no-op when no tool is attached).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

constexpr int BLOCK = 224;
// Slots of the synchronous calls: host-buffer jobs rotate over the first
// JOB_SLOTS; a device-pointer call runs up to all of them at once.
constexpr int SYNC_SLOTS = 4;
#ifndef MGCM_JOB_SLOTS
#define MGCM_JOB_SLOTS 4
#endif
constexpr int JOB_SLOTS = MGCM_JOB_SLOTS;
static_assert(JOB_SLOTS >= 1 && JOB_SLOTS <= SYNC_SLOTS, "job slots");

// On-chip solve kernels by family and threads per CTA (rt_onchip.cu).
using OcKernel = void (*)(const SegTable *__restrict__, int, int, unsigned char *__restrict__, size_t,
                          const double *__restrict__, const float *__restrict__, const RtConst,
                          const int *__restrict__, const unsigned int *, double *__restrict__,
                          double *__restrict__);
constexpr int OC_NT = 8;   // T = 32, 64, ..., 256
#define OC_ROW(V, F) {rt_solve_oc<V, F, 32>, rt_solve_oc<V, F, 64>, rt_solve_oc<V, F, 96>,          \
                       rt_solve_oc<V, F, 128>, rt_solve_oc<V, F, 160>, rt_solve_oc<V, F, 192>,      \
                       rt_solve_oc<V, F, 224>, rt_solve_oc<V, F, 256>}
const OcKernel OC_KERNELS[3][OC_NT] = {OC_ROW(true, false), OC_ROW(true, true), OC_ROW(false, false)};
#undef OC_ROW


// Persistent fused kernel (rt_fused.cu) by precision and launch shape.
using FusedKernel = void (*)(const SegTable *__restrict__, int, int, unsigned char *__restrict__, size_t, size_t,
                             const double *__restrict__, const double *__restrict__, const float *__restrict__,
                             const double *__restrict__, const RtConst, unsigned int *, uint32_t *,
                             unsigned long long *);
struct FusedShape { int tc, threads, minb; };
constexpr int FUSED_NS = 13;
constexpr FusedShape FUSED_SHAPES[FUSED_NS] = {{2, 128, 8}, {4, 128, 8}, {8, 128, 8}, {4, 128, 6},
                                               {4, 256, 4}, {8, 256, 4}, {16, 256, 4}, {8, 512, 2},
                                               {8, 256, 3}, {16, 384, 2}, {16, 256, 3}, {24, 384, 2},
                                               {16, 320, 2}};
constexpr int FUSED_DEFAULT = 9;   // the tuner's choice for the 889,920-column ensemble
#define FZ_ROW(F) {rt_fused<F, 2, 128, 8>, rt_fused<F, 4, 128, 8>, rt_fused<F, 8, 128, 8>,  \
                   rt_fused<F, 4, 128, 6>, rt_fused<F, 4, 256, 4>, rt_fused<F, 8, 256, 4>,  \
                   rt_fused<F, 16, 256, 4>, rt_fused<F, 8, 512, 2>, rt_fused<F, 8, 256, 3>,   \
                   rt_fused<F, 16, 384, 2>, rt_fused<F, 16, 256, 3>, rt_fused<F, 24, 384, 2>, \
                   rt_fused<F, 16, 320, 2>}
const FusedKernel FUSED_KERNELS[2][FUSED_NS] = {FZ_ROW(false), FZ_ROW(true)};
#undef FZ_ROW

// Slots (doubles) per system of a family at NL layers: rt_onchip.cuh.
int oc_slots(bool vis, int nl) { return vis ? 8 * nl + 1 : 7 * nl; }
// Largest T (multiple of 32, <= 256) whose slices fit one CTA's shared memory; 0: none.
int oc_threads(bool vis, int nl) {
    const size_t per = (size_t)oc_slots(vis, nl) * sizeof(double);
    const int t = (int)std::min<size_t>(256, SMEM_CAP / per) / 32 * 32;
    return t;
}
// Tensor-memory forms by family and warps per CTA: W = 4, 6, 8, 9.
constexpr int TM_NW = 4;
constexpr int TM_WARPS[TM_NW] = {4, 6, 8, 9};
#define TM_ROW(V, F) {rt_solve_tm<V, F, 4>, rt_solve_tm<V, F, 6>, rt_solve_tm<V, F, 8>, rt_solve_tm<V, F, 9>}
const OcKernel TM_KERNELS[3][TM_NW] = {TM_ROW(true, false), TM_ROW(true, true), TM_ROW(false, false)};
#undef TM_ROW
// Tensor-memory doubles per thread with W warps (the 512 columns split
// between the warps of a lane quarter).
int tm_doubles(int w) { return (int)(((512u / (unsigned)((w + 3) / 4)) & ~1u) / 2); }
// Dynamic shared memory the tensor-memory forms may take: the cap less room
// for their static shared memory (the TMEM address word).
constexpr size_t TM_SMEM_CAP = SMEM_CAP - 1024;
// Index into TM_WARPS of the most warps whose shared-memory remainder fits; -1: none.
int tm_choice(bool vis, int nl) {
    for (int q = TM_NW - 1; q >= 0; --q) {
        const int w = TM_WARPS[q];
        const long long rest = std::max(0, oc_slots(vis, nl) - tm_doubles(w));
        if ((size_t)rest * 32 * w * 8 <= TM_SMEM_CAP) return q;
    }
    return -1;
}
#ifndef MGCM_SYNC_JOB_COLS
#define MGCM_SYNC_JOB_COLS 8192
#endif
constexpr int SYNC_JOB_COLS = MGCM_SYNC_JOB_COLS;   // columns per job of a synchronous host-buffer call
#ifndef MGCM_SYNC_RAMP
#define MGCM_SYNC_RAMP 2048
#endif
constexpr int SYNC_RAMP_COLS = MGCM_SYNC_RAMP;   // first (and last) job of a ramped host-buffer call
#ifndef MGCM_SERVE_JOB_COLS
#define MGCM_SERVE_JOB_COLS 16384
#endif
constexpr int SERVE_JOB_COLS = MGCM_SERVE_JOB_COLS;   // columns per job of a served request
constexpr int SERVE_SLOTS = 4;          // serving slots at most

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
        fin(sg.tauref + (size_t)c * LEV1, sg.dust_band ? LEV : LEV1);   // TAUREF(LEV+1) is 0 then
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

struct Request {
    std::vector<mgcm_rt_batch_in> in;
    std::vector<mgcm_rt_batch_out> out;
    int status = 0;
    int jobs_left = 0;
    int jobs = 0;          // jobs the request was split into
    int deferred = 0;      // admissions put back by the HBM budget
    bool done = false;
    std::chrono::steady_clock::time_point t_submit, t_done;
    // device time of the request's kernels, ms after the handle's epoch event
    double dev_begin = 1e300, dev_end = -1e300;
};

struct Job {
    std::shared_ptr<Request> req;
    int seg = 0, c0 = 0, c1 = 0;   // columns [c0, c1) of batch `seg`
};

// Launch shape of the pipeline; 0 = the built-in choice.  Picked per graph by
// the autotuner (mgcm_rt_graph_create).
struct Tune {
    int chunk = 0;        // columns per pipeline pass
    int solve_ctas = 0;   // solver CTAs per SM
    int rb = 0;           // reduce: kept-system rows per TMA chunk
    int fused = -1;       // fused kernel: index into FUSED_SHAPES (-1: the default shape)
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaStream_t aux = nullptr;   // the visible solve runs here, beside the IR solve
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, done = nullptr;
    cudaEvent_t after_legacy = nullptr;   // orders the slot after the legacy default stream
    SegTable *h_segs = nullptr, *d_segs = nullptr;
    uint32_t *d_status = nullptr, *h_status = nullptr;
    unsigned long long *d_nsys = nullptr, *h_nsys = nullptr;
    Arena stage, pipe, aero;   // aero: per-level aerosol arrays of tracer jobs
    int occ_nl = 0, occ_rb = 0, occ_stage = 1, occ_screen = 1, occ_solve = 1, occ_quad = 1, occ_reduce = 1;
    bool busy = false;
    Job job;
    int kernels = 0;
    Tune tune;
};

}  // namespace

struct mgcm_rt_handle {
    mgcm_rt_config cfg{};
    int device = 0;
    int num_sms = 0;
    HostTables host;
    RtConst K{};
    double *d_kv = nullptr, *d_ki = nullptr, *d_planck = nullptr;
    float *d_kvf = nullptr;   // FP32 visible table (Cmk*k) of the MIXED path
    bool quad = false;        // four-lane solvers for L <= 51 (mgcm_rt_config.solver)
    bool onchip = false;      // solvers with the per-system arrays on chip (mgcm_rt_config.solver)
    bool tmem = false;        // ... with tensor memory in front of shared memory
    bool fused = false;       // one persistent fused kernel per call (mgcm_rt_config.solver)
    AeroConst aero{};         // aerosol optics constants (mgcm_rt_run_tracers)
    double *d_mie = nullptr;  // Mie tables on the device; null when the files were absent
    std::mutex mu;                                  // serialises the synchronous API
    std::vector<std::unique_ptr<Slot>> slots;       // SYNC_SLOTS synchronous slots
    cudaStream_t user_stream = nullptr;             // mgcm_rt_set_stream
    cudaEvent_t fork = nullptr;
    bool pending = false;
    long long pending_cols = 0;
    int pending_parts = 1;                          // slots a pending device call runs on
    mgcm_rt_stats stats{};
    size_t budget = 0, used = 0;
    std::mutex mem_mu;
    // serving
    std::mutex qmu;
    std::condition_variable qcv, dcv;
    std::deque<Job> jobs;
    std::map<long long, std::shared_ptr<Request>> reqs;
    long long next_ticket = 1;
    std::vector<std::unique_ptr<Slot>> sslots;
    std::thread worker;
    bool stop = false;
    int max_jobs = 100000;                          // jobs accepted and not finished, at most
    int outstanding = 0;
    cudaEvent_t epoch = nullptr;                    // device time origin of the request timestamps
    std::chrono::steady_clock::time_point t_epoch;  // host time origin
};

namespace {

#define CK(x)                                        \
    do {                                             \
        cudaError_t e_ = (x);                        \
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


cudaStream_t sync_stream(mgcm_rt_handle *h) {
    return h->user_stream ? h->user_stream : h->slots[0]->stream;
}

// Device-pointer calls: the slots' streams are non-blocking, so they do not
// wait for work the caller queued on the legacy default stream (cudaMemcpy,
// a framework's default-stream fills of the very buffers passed in).  An
// event recorded there and waited on first orders the call after all of it.
int after_legacy_stream(Slot &sl, cudaStream_t st) {
    CK(cudaEventRecord(sl.after_legacy, cudaStreamLegacy));
    CK(cudaStreamWaitEvent(st, sl.after_legacy, 0));
    return MGCM_RT_OK;
}

// Grows an arena within the handle's HBM budget (arenas never shrink).
int arena_ensure(mgcm_rt_handle *h, Arena &a, size_t bytes, cudaStream_t s) {
    if (a.bytes >= bytes) return MGCM_RT_OK;
    std::lock_guard<std::mutex> lk(h->mem_mu);
    if (h->used - a.bytes + bytes > h->budget) return MGCM_RT_ENOMEM;
    if (a.ptr) {
        CK(cudaStreamSynchronize(s));
        cudaFree(a.ptr);
        h->used -= a.bytes;
    }
    a.ptr = nullptr;
    a.bytes = 0;
    if (cudaMalloc(&a.ptr, bytes) != cudaSuccess) return MGCM_RT_ENOMEM;
    a.bytes = bytes;
    h->used += bytes;
    return MGCM_RT_OK;
}

int slot_init(Slot &s) {
    CK(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&s.aux, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&s.fork_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&s.join_ev, cudaEventDisableTiming));
    CK(cudaEventCreate(&s.ev0));
    CK(cudaEventCreate(&s.ev1));
    CK(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&s.after_legacy, cudaEventDisableTiming));
    CK(cudaMallocHost(&s.h_segs, sizeof(SegTable)));
    CK(cudaMalloc(&s.d_segs, sizeof(SegTable)));
    CK(cudaMalloc(&s.d_status, 256));
    CK(cudaMallocHost(&s.h_status, 64));
    s.d_nsys = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(s.d_status) + 128);
    s.h_nsys = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(s.h_status) + 32);
    *s.h_status = 0;
    *s.h_nsys = 0;
    return MGCM_RT_OK;
}

void slot_free(mgcm_rt_handle *h, Slot &s) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    for (Arena *a : {&s.stage, &s.pipe, &s.aero})
        if (a->ptr) {
            cudaFree(a->ptr);
            h->used -= a->bytes;
            a->ptr = nullptr;
            a->bytes = 0;
        }
    if (s.h_segs) cudaFreeHost(s.h_segs);
    if (s.d_segs) cudaFree(s.d_segs);
    if (s.d_status) cudaFree(s.d_status);
    if (s.h_status) cudaFreeHost(s.h_status);
    if (s.ev0) cudaEventDestroy(s.ev0);
    if (s.ev1) cudaEventDestroy(s.ev1);
    if (s.done) cudaEventDestroy(s.done);
    if (s.after_legacy) cudaEventDestroy(s.after_legacy);
    if (s.aux) cudaStreamSynchronize(s.aux);
    if (s.fork_ev) cudaEventDestroy(s.fork_ev);
    if (s.join_ev) cudaEventDestroy(s.join_ev);
    if (s.aux) cudaStreamDestroy(s.aux);
    if (s.stream) cudaStreamDestroy(s.stream);
}

// Function attributes are process-wide per device, so they are set once, to
// the largest value any layer count or handle needs, never per launch: a
// per-launch value set by one slot or handle would undercut another's launch.
int configure_kernels(int device) {
    static std::mutex mu;
    static bool done[256] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 256) return MGCM_RT_EINVAL;
    if (done[device]) return MGCM_RT_OK;
    for (int nl : {32, 33})
        for (int rb : {1, 2, 4, 8})
            CK(cudaFuncSetAttribute(reduce_kernel(nl, rb), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)SMEM_CAP));
    CK(cudaFuncSetAttribute(rt_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_CAP));
    for (int f = 0; f < 3; ++f)
        for (int q = 0; q < OC_NT; ++q)
            CK(cudaFuncSetAttribute((const void *)OC_KERNELS[f][q], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)SMEM_CAP));
    for (int f = 0; f < 2; ++f)
        for (int q = 0; q < FUSED_NS; ++q)
            CK(cudaFuncSetAttribute((const void *)FUSED_KERNELS[f][q], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(SMEM_CAP - 1024)));
    for (int f = 0; f < 3; ++f)
        for (int q = 0; q < TM_NW; ++q)
            CK(cudaFuncSetAttribute((const void *)TM_KERNELS[f][q], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)TM_SMEM_CAP));
    // the solvers use no shared memory: the whole unified L1 goes to the
    // per-system arrays
    for (const void *f : {(const void *)rt_fp64_solve<true>, (const void *)rt_fp64_solve<false>,
                          (const void *)rt_mixed_solve_vis})
        CK(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 0));
    done[device] = true;
    return MGCM_RT_OK;
}

size_t pipe_bytes_per_col(int max_nl, size_t *stride_out = nullptr) {
    const size_t stride = (col_smem_bytes(max_nl, false) + 255) / 256 * 256;
    if (stride_out) *stride_out = stride;
    const size_t row = (size_t)2 * max_nl * sizeof(double);
    return stride + NSYS * (sizeof(int) + row + 4 * sizeof(double));
}

// Three-kernel pipeline (rt_fp64.cu; MIXED swaps in rt_mixed.cu's solver)
// over chunks of the columns in the slot's segment table.
int launch_pipeline(mgcm_rt_handle *h, Slot &sl, cudaStream_t st, int total, int max_nl, int &nk,
                    int max_chunk) {
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    size_t stride = 0;
    const size_t per_col = pipe_bytes_per_col(max_nl, &stride);
    const size_t row = (size_t)2 * max_nl * sizeof(double);
    int chunk = std::min(total, max_chunk);
    if (sl.tune.chunk > 0) chunk = std::min(chunk, sl.tune.chunk);
    const size_t n_v = (size_t)chunk * NSYS_V, n_i = (size_t)chunk * NSYS_I;
    // flux rows and scalars in whole blocks of ROW_BLK list positions
    const size_t r_v = row_slots(n_v), r_i = row_slots(n_i);
    const size_t need = al((size_t)chunk * stride) + al(n_v * 4) + al(n_i * 4) + al(r_v * row) +
                        al(r_i * row) + al(r_v * 32) + al(r_i * 32) + 256;
    (void)per_col;
    int rc = arena_ensure(h, sl.pipe, need, st);
    if (rc) return rc;
    unsigned char *p = static_cast<unsigned char *>(sl.pipe.ptr);
    auto take = [&](size_t b) { unsigned char *r = p; p += al(b); return r; };
    unsigned char *blocks = take((size_t)chunk * stride);
    int *list_v = reinterpret_cast<int *>(take(n_v * 4));
    int *list_i = reinterpret_cast<int *>(take(n_i * 4));
    double *fl_v = reinterpret_cast<double *>(take(r_v * row));
    double *fl_i = reinterpret_cast<double *>(take(r_i * row));
    double *sc_v = reinterpret_cast<double *>(take(r_v * 32));
    double *sc_i = reinterpret_cast<double *>(take(r_i * 32));
    unsigned int *counts = reinterpret_cast<unsigned int *>(take(256));
    const int rb = sl.tune.rb > 0 ? sl.tune.rb : reduce_rows_per_chunk(max_nl);
    const size_t rsm = reduce_smem_bytes(max_nl, rb);
    const bool mixed = h->cfg.precision == MGCM_RT_MIXED;
    if (sl.occ_nl != max_nl || sl.occ_rb != rb) {
        sl.occ_nl = max_nl;
        sl.occ_rb = rb;
        int a = 1, b = 1, c = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, mixed ? rt_fp64_screen<true> : rt_fp64_screen<false>,
                                                      SCREEN_THREADS, 0);
        int e = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e, rt_stage, STAGE_THREADS, 0);
        sl.occ_stage = std::max(e, 1);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, rt_fp64_solve<false>, 128, 0);
        int qo = 1;
        const int qr = quad_r_for(max_nl);
        if (qr == 7) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&qo, rt_quad_solve<false, 7>, 128, 0);
        else if (qr == 10) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&qo, rt_quad_solve<false, 10>, 128, 0);
        else if (qr == 13) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&qo, rt_quad_solve<false, 13>, 128, 0);
        sl.occ_quad = std::max(qo, 1);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, reduce_kernel(max_nl, rb), REDUCE_THREADS, rsm);
        sl.occ_screen = std::max(a, 1);
        sl.occ_solve = std::max(b, 1);
        sl.occ_reduce = std::max(c, 1);
    }
    for (int c0 = 0; c0 < total; c0 += chunk) {
        const int c1 = std::min(total, c0 + chunk);
        CK(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned int), st));
        const int g0 = std::min((c1 - c0 + 3) / 4, h->num_sms * sl.occ_stage);   // 4 columns per CTA
        rt_stage<<<g0, STAGE_THREADS, 0, st>>>(sl.d_segs, c0, c1, max_nl, blocks, stride, h->d_planck, h->K,
                                               sl.d_status);
        const long long items = (long long)(c1 - c0) * SCREEN_GROUPS;
        const int warps = SCREEN_THREADS / 32;
        const int g1 = (int)std::min<long long>((items + warps - 1) / warps, (long long)h->num_sms * sl.occ_screen);
        if (mixed)
            rt_fp64_screen<true><<<g1, SCREEN_THREADS, 0, st>>>(sl.d_segs, c0, c1, max_nl, blocks, stride,
                                                                h->d_kv, h->d_ki, h->K, list_v, list_i,
                                                                counts, sl.d_nsys, h->d_kvf);
        else
            rt_fp64_screen<false><<<g1, SCREEN_THREADS, 0, st>>>(sl.d_segs, c0, c1, max_nl, blocks, stride,
                                                                 h->d_kv, h->d_ki, h->K, list_v, list_i,
                                                                 counts, sl.d_nsys, nullptr);
        const int g2 = h->num_sms * (sl.tune.solve_ctas > 0 ? sl.tune.solve_ctas : sl.occ_solve);
        // MIXED: FP32 visible opacities; the IR family is FP64 in both modes.
        // The visible solve runs on the slot's second stream beside the IR
        // solve, so each kernel's last wave overlaps the other's.
        CK(cudaEventRecord(sl.fork_ev, st));
        CK(cudaStreamWaitEvent(sl.aux, sl.fork_ev, 0));
        cudaStream_t vst = sl.aux;
        const int qr = h->quad ? quad_r_for(max_nl) : 0;
        const bool oc = h->onchip || h->tmem;
        const int tv = oc ? oc_threads(true, max_nl) : 0, ti = oc ? oc_threads(false, max_nl) : 0;
        // tensor-memory forms: every system of the launch on one layer count
        bool one_l = true;
        for (int q = 1; q < sl.h_segs->nseg; ++q) one_l = one_l && sl.h_segs->seg[q].L == sl.h_segs->seg[0].L;
        const int qv = h->tmem && one_l ? tm_choice(true, max_nl) : -1;
        const int qi = h->tmem && one_l ? tm_choice(false, max_nl) : -1;
        if (qv >= 0 && qi >= 0) {
            const int wv = TM_WARPS[qv], wi = TM_WARPS[qi];
            // at least 116 KB of shared memory each: no two CTAs that hold the
            // SM's 512 TMEM columns ever share an SM (a second allocation
            // would wait for the first CTA to finish)
            const size_t floor_b = 116 * 1024;
            const size_t smv = std::max(floor_b, (size_t)std::max(0, oc_slots(true, max_nl) - tm_doubles(wv)) * 32 * wv * 8);
            const size_t smi = std::max(floor_b, (size_t)std::max(0, oc_slots(false, max_nl) - tm_doubles(wi)) * 32 * wi * 8);
            TM_KERNELS[mixed ? 1 : 0][qv]<<<h->num_sms, 32 * wv, smv, vst>>>(
                sl.d_segs, c0, max_nl, blocks, stride, h->d_kv, h->d_kvf, h->K, list_v, counts, fl_v, sc_v);
            TM_KERNELS[2][qi]<<<h->num_sms, 32 * wi, smi, st>>>(
                sl.d_segs, c0, max_nl, blocks, stride, h->d_ki, nullptr, h->K, list_i, counts, fl_i, sc_i);
        } else if (tv > 0 && ti > 0) {
            const size_t smv = (size_t)tv * oc_slots(true, max_nl) * 8, smi = (size_t)ti * oc_slots(false, max_nl) * 8;
            OC_KERNELS[mixed ? 1 : 0][tv / 32 - 1]<<<h->num_sms, tv, smv, vst>>>(
                sl.d_segs, c0, max_nl, blocks, stride, h->d_kv, h->d_kvf, h->K, list_v, counts, fl_v, sc_v);
            OC_KERNELS[2][ti / 32 - 1]<<<h->num_sms, ti, smi, st>>>(
                sl.d_segs, c0, max_nl, blocks, stride, h->d_ki, nullptr, h->K, list_i, counts, fl_i, sc_i);
        } else if (qr) {
            const int gq = h->num_sms * (sl.tune.solve_ctas > 0 ? sl.tune.solve_ctas : sl.occ_quad);
#define MGCM_QUAD(R)                                                                                        \
    do {                                                                                                    \
        if (mixed)                                                                                          \
            rt_quad_mixed_vis<R><<<gq, 128, 0, vst>>>(sl.d_segs, c0, max_nl, blocks, stride, h->d_kvf,       \
                                                     h->d_kv, h->K, list_v, counts, fl_v, sc_v);             \
        else                                                                                                \
            rt_quad_solve<true, R><<<gq, 128, 0, vst>>>(sl.d_segs, c0, max_nl, blocks, stride, h->d_kv, h->K,\
                                                       list_v, counts, fl_v, sc_v);                          \
        rt_quad_solve<false, R><<<gq, 128, 0, st>>>(sl.d_segs, c0, max_nl, blocks, stride, h->d_ki, h->K,    \
                                                    list_i, counts, fl_i, sc_i);                             \
    } while (0)
            if (qr == 7) MGCM_QUAD(7);
            else if (qr == 10) MGCM_QUAD(10);
            else MGCM_QUAD(13);
#undef MGCM_QUAD
        } else {
            if (mixed)
                rt_mixed_solve_vis<<<g2, 128, 0, vst>>>(sl.d_segs, c0, max_nl, blocks, stride, h->d_kvf, h->d_kv,
                                                        h->K, list_v, counts, fl_v, sc_v);
            else
                rt_fp64_solve<true><<<g2, 128, 0, vst>>>(sl.d_segs, c0, max_nl, blocks, stride, h->d_kv, h->K,
                                                         list_v, counts, fl_v, sc_v);
            rt_fp64_solve<false><<<g2, 128, 0, st>>>(sl.d_segs, c0, max_nl, blocks, stride, h->d_ki, h->K,
                                                     list_i, counts, fl_i, sc_i);
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(sl.join_ev, sl.aux));
        CK(cudaStreamWaitEvent(st, sl.join_ev, 0));
        const int g3 = std::min((c1 - c0 + REDUCE_WARPS - 1) / REDUCE_WARPS, h->num_sms * sl.occ_reduce);
        {
            const SegTable *segs = sl.d_segs;
            const RtConst &K = h->K;
            void *args[] = {(void *)&segs, (void *)&c0, (void *)&c1, (void *)&max_nl, (void *)&blocks,
                            (void *)&stride, (void *)&K, (void *)&fl_v, (void *)&sc_v, (void *)&fl_i,
                            (void *)&sc_i};
            CK(cudaLaunchKernel(reduce_kernel(max_nl, rb), dim3(g3), dim3(REDUCE_THREADS), args, rsm, st));
        }
        nk += 5;
        CK(cudaGetLastError());
    }
    return MGCM_RT_OK;
}

// One persistent fused kernel over every column of the slot's segment table:
// grid = the CTAs that fit the SMs at once, each with its own scratch; a tile
// counter (cleared first) hands out the columns.  No chunking: the scratch
// does not grow with the number of columns.
int launch_fused(mgcm_rt_handle *h, Slot &sl, cudaStream_t st, int ncols, int max_nl, int &nk) {
    const int si = sl.tune.fused >= 0 && sl.tune.fused < FUSED_NS ? sl.tune.fused : FUSED_DEFAULT;
    const FusedShape sh = FUSED_SHAPES[si];
    const bool mixed = h->cfg.precision == MGCM_RT_MIXED;
    const FusedKernel kern = FUSED_KERNELS[mixed ? 1 : 0][si];
    const size_t smem = fused_smem(sh.threads / 32, sh.tc);
    int occ = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, sh.threads, smem) != cudaSuccess || occ < 1)
        occ = 1;
    const int grid = h->num_sms * occ;
    size_t stride = 0;
    pipe_bytes_per_col(max_nl, &stride);
    const size_t cta = (fused_scratch_per_cta(sh.tc, max_nl, stride) + 255) / 256 * 256;
    const int rc = arena_ensure(h, sl.pipe, cta * grid + 256, st);
    if (rc) return rc;
    unsigned char *scr = static_cast<unsigned char *>(sl.pipe.ptr);
    unsigned int *ctr = reinterpret_cast<unsigned int *>(scr + cta * grid);
    CK(cudaMemsetAsync(ctr, 0, sizeof(unsigned int), st));
    kern<<<grid, sh.threads, smem, st>>>(sl.d_segs, ncols, max_nl, scr, cta, stride, h->d_kv, h->d_ki, h->d_kvf,
                                         h->d_planck, h->K, ctr, sl.d_status, sl.d_nsys);
    CK(cudaGetLastError());
    nk += 1;
    return MGCM_RT_OK;
}

// The radiation kernels of a call: the persistent fused kernel or the
// multi-kernel pipeline, per the handle's form.
int launch_body(mgcm_rt_handle *h, Slot &sl, cudaStream_t st, int total, int max_nl, int &nk, int max_chunk) {
    return h->fused ? launch_fused(h, sl, st, total, max_nl, nk)
                    : launch_pipeline(h, sl, st, total, max_nl, nk, max_chunk);
}

// Status words cleared, optional validation, kernels between ev0 and ev1.
int launch_all(mgcm_rt_handle *h, Slot &sl, cudaStream_t st, int total, int max_nl, int max_chunk) {
    CK(cudaMemsetAsync(sl.d_status, 0, 256, st));
    int nk = 0;
    if (h->cfg.validate) {
        const int vb = std::min((total + 255) / 256, h->num_sms * 8);
        validate_kernel<<<std::max(vb, 1), 256, 0, st>>>(sl.d_segs, sl.d_status);
        ++nk;
    }
    CK(cudaEventRecord(sl.ev0, st));
    const int rc = launch_body(h, sl, st, total, max_nl, nk, max_chunk);
    if (rc) return rc;
    CK(cudaEventRecord(sl.ev1, st));
    sl.kernels = nk;
    return MGCM_RT_OK;
}

int status_to_code(uint32_t st) {
    if (st & ST_NONFINITE) return MGCM_RT_ENONFINITE;
    if (st & (ST_TEMP | ST_PLANCK_RANGE)) return MGCM_RT_ETEMP;
    if (st & ST_BADL) return MGCM_RT_ELAYERS;
    return MGCM_RT_OK;
}

// Copies the slot's status words to pinned host memory on its stream.
int post_status(Slot &sl, cudaStream_t st) {
    CK(cudaMemcpyAsync(sl.h_status, sl.d_status, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(sl.h_nsys, sl.d_nsys, 8, cudaMemcpyDeviceToHost, st));
    return MGCM_RT_OK;
}

// Issues one job on a slot: staging of host arrays (column range [c0,c1) of
// batch in/out), the kernels and the copies back; records sl.done.
int issue_job(mgcm_rt_handle *h, Slot &sl, cudaStream_t st, const mgcm_rt_batch_in &in,
              const mgcm_rt_batch_out &out, int c0, int c1) {
    NvtxRange nvtx_range("mgcm_rt job");
    const Sizes z = sizes_of(in);
    const size_t n = (size_t)(c1 - c0);
    SegDev sd{};
    sd.ncol = (int)n;
    sd.L = z.L;
    sd.col0 = 0;
    sd.ptrop = in.ptrop;
    std::vector<ArrSpec> arrs;
    if (in.device_ptrs) {
        if (const int rc = after_legacy_stream(sl, st)) return rc;
        fill_direct(sd, in, out);
        // shift every per-column pointer to the job's first column
        arrs = arrays_of(in, out, z, sd);
        for (auto &a : arrs) *a.seg_field = const_cast<double *>(a.src ? a.src : a.dst) + (size_t)c0 * a.per_col;
        sd.sigma = in.sigma;
        sd.sol = in.sol;
    } else {
        arrs = arrays_of(in, out, z, sd);
        size_t bytes = ((z.lev + 8) * 8 + 255) / 256 * 256;
        for (const auto &a : arrs) bytes += ((a.per_col * n * 8 + 255) / 256) * 256;
        const int rc = arena_ensure(h, sl.stage, bytes, st);
        if (rc) return rc;
        char *base = static_cast<char *>(sl.stage.ptr);
        size_t off = 0;
        for (auto &a : arrs) {
            double *d = reinterpret_cast<double *>(base + off);
            off += ((a.per_col * n * 8 + 255) / 256) * 256;
            *a.seg_field = d;
            a.dev = d;
            if (a.dir != 1)
                CK(cudaMemcpyAsync(d, a.src + (size_t)c0 * a.per_col, a.per_col * n * 8,
                                   cudaMemcpyHostToDevice, st));
        }
        double *ds = reinterpret_cast<double *>(base + off);
        CK(cudaMemcpyAsync(ds, in.sigma, z.lev * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ds + z.lev, in.sol, 7 * 8, cudaMemcpyHostToDevice, st));
        sd.sigma = ds;
        sd.sol = ds + z.lev;
    }
    SegTable &tab = *sl.h_segs;
    tab.nseg = 1;
    tab.total_cols = (int)n;
    tab.seg[0] = sd;
    CK(cudaMemcpyAsync(sl.d_segs, sl.h_segs, offsetof(SegTable, seg) + sizeof(SegDev),
                       cudaMemcpyHostToDevice, st));
    int rc = launch_all(h, sl, st, (int)n, z.nl, 1 << 30);
    if (rc) return rc;
    if (!in.device_ptrs)
        for (auto &a : arrs)
            if (a.dir != 0)
                CK(cudaMemcpyAsync(a.dst + (size_t)c0 * a.per_col, a.dev, a.per_col * n * 8,
                                   cudaMemcpyDeviceToHost, st));
    rc = post_status(sl, st);
    if (rc) return rc;
    CK(cudaEventRecord(sl.done, st));
    return MGCM_RT_OK;
}

// Device-pointer batches.  The columns are split into up to SYNC_SLOTS parts
// of at least SPLIT_COLS columns that run concurrently on the synchronous
// slots -- the first on the caller's stream, the others on their slots'
// streams, forked from and joined back into it -- so the parts' kernels share
// the SMs, which these latency-bound kernels use better than one call's
// kernels (64,800 columns: 12.66 ms in one call; as 2 / 3 / 4 concurrent
// calls 12.2 / 12.0 / 11.9 ms).  The fused form, a persistent kernel that
// fills the GPU by itself, runs unsplit.
constexpr int SPLIT_COLS = 12288;

// Segment table of the global columns [b0, b1) of the batches, every
// per-column pointer shifted to the segment's first column in the range;
// returns the table's columns.
int table_of_range(SegTable &tab, int nbatch, const mgcm_rt_batch_in *in, const mgcm_rt_batch_out *out,
                   int b0, int b1, int &max_nl) {
    tab.nseg = 0;
    int gcol = 0, pc = 0;
    for (int b = 0; b < nbatch; ++b) {
        const Sizes z = sizes_of(in[b]);
        if (z.ncol == 0) continue;
        const int lo = std::max(b0, gcol), hi = std::min(b1, gcol + (int)z.ncol);
        if (lo < hi) {
            SegDev sd{};
            sd.ncol = hi - lo;
            sd.L = z.L;
            sd.col0 = pc;
            sd.ptrop = in[b].ptrop;
            fill_direct(sd, in[b], out[b]);
            for (auto &a : arrays_of(in[b], out[b], z, sd))
                *a.seg_field = const_cast<double *>(a.src ? a.src : a.dst) + (size_t)(lo - gcol) * a.per_col;
            sd.sigma = in[b].sigma;
            sd.sol = in[b].sol;
            tab.seg[tab.nseg++] = sd;
            max_nl = std::max(max_nl, z.nl);
            pc += hi - lo;
        }
        gcol += (int)z.ncol;
    }
    tab.total_cols = pc;
    return pc;
}

int finish_pending(mgcm_rt_handle *h);

// Synchronous batch of device-pointer segments (async: leave it pending).
int run_device(mgcm_rt_handle *h, int nbatch, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out,
               bool async) {
    int total = 0;
    for (int b = 0; b < nbatch; ++b) {
        const Sizes z = sizes_of(in[b]);
        if ((long long)total + (long long)z.ncol > 0x7fffff) return MGCM_RT_EINVAL;
        total += (int)z.ncol;
    }
    if (total == 0) return MGCM_RT_OK;
    cudaStream_t st = sync_stream(h);
    Slot &s0 = *h->slots[0];
    if (!h->user_stream) {
        if (const int rc = after_legacy_stream(s0, st)) return rc;
    }
    const int nparts = h->fused ? 1 : std::max(1, std::min(SYNC_SLOTS, total / SPLIT_COLS));
    if (nparts > 1) {
        CK(cudaEventRecord(h->fork, st));
        for (int p = 1; p < nparts; ++p) CK(cudaStreamWaitEvent(h->slots[p]->stream, h->fork, 0));
    }
    // a part that fails to launch leaves the ones issued before it running on
    // the caller's buffers and the slots' scratch: wait for them
    auto drain = [&](int rc, int issued) {
        cudaStreamSynchronize(st);
        for (int q = 1; q <= issued && q < nparts; ++q) cudaStreamSynchronize(h->slots[q]->stream);
        return rc;
    };
    for (int p = 0; p < nparts; ++p) {
        Slot &sl = *h->slots[p];
        cudaStream_t ps = p == 0 ? st : sl.stream;
        const int b0 = (int)((long long)total * p / nparts), b1 = (int)((long long)total * (p + 1) / nparts);
        int max_nl = 1;
        const int n = table_of_range(*sl.h_segs, nbatch, in, out, b0, b1, max_nl);
        if (cudaMemcpyAsync(sl.d_segs, sl.h_segs, sizeof(SegTable), cudaMemcpyHostToDevice, ps) != cudaSuccess)
            return drain(MGCM_RT_ECUDA, p);
        // pipeline chunk: the parts' scratch together within half the budget
        // (one part: a quarter)
        const size_t per_col = pipe_bytes_per_col(max_nl);
        const size_t share = h->budget / (nparts > 1 ? 2 * nparts : 4);
        const int chunk = (int)std::max<size_t>(1, std::min<size_t>(n, share / per_col));
        int rc = launch_all(h, sl, ps, n, max_nl, chunk);
        if (!rc) rc = post_status(sl, ps);
        if (rc) return drain(rc, p);
    }
    if (nparts > 1) {
        for (int p = 1; p < nparts; ++p) {
            CK(cudaEventRecord(h->slots[p]->done, h->slots[p]->stream));
            CK(cudaStreamWaitEvent(st, h->slots[p]->done, 0));
        }
        CK(cudaEventRecord(s0.ev1, st));   // the call ends when every part has
    }
    h->pending = true;
    h->pending_cols = total;
    h->pending_parts = nparts;
    if (async) return MGCM_RT_OK;
    return finish_pending(h);
}

int finish_pending(mgcm_rt_handle *h) {
    if (!h->pending) return MGCM_RT_OK;
    Slot &s0 = *h->slots[0];
    CK(cudaStreamSynchronize(sync_stream(h)));
    h->pending = false;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s0.ev0, s0.ev1);
    uint32_t stw = *s0.h_status;
    unsigned long long nsys = *s0.h_nsys;
    int nk = s0.kernels;
    for (int p = 1; p < h->pending_parts; ++p) {
        const Slot &sp = *h->slots[p];
        stw |= *sp.h_status;
        nsys += *sp.h_nsys;
        nk += sp.kernels;
    }
    h->stats.gpu_ms = ms;
    h->stats.columns = h->pending_cols;
    h->stats.systems = (long long)nsys;
    h->stats.status = (int)stw;
    h->stats.kernels = nk;
    return status_to_code(stw);
}

// Column ranges (ends) of a synchronous host-buffer call over n columns: jobs
// of up to max_job columns.  With first > 0 the jobs ramp up (first, 2 first,
// ... below max_job) and back down at the end, so the first host-to-device
// copy and the last device-to-host copy, which no kernel overlaps, are short;
// the middle is split evenly.
std::vector<int> job_ends(int n, int max_job, int first) {
    std::vector<int> ramp, ends;
    int ramp_cols = 0;
    for (int sz = first; first > 0 && sz < max_job; sz *= 2) {
        ramp.push_back(sz);
        ramp_cols += sz;
    }
    int c = 0;
    if (!ramp.empty() && n >= 2 * ramp_cols + max_job) {
        for (int sz : ramp) ends.push_back(c += sz);
        const int mid = n - 2 * ramp_cols, nj = (mid + max_job - 1) / max_job;
        for (int j = 0; j < nj; ++j) ends.push_back(c += mid / nj + (j < mid % nj ? 1 : 0));
        for (auto it = ramp.rbegin(); it != ramp.rend(); ++it) ends.push_back(c += *it);
    } else {
        while (c < n) ends.push_back(c = std::min(n, c + max_job));
    }
    return ends;
}

// Synchronous batch of host-pointer segments: jobs rotate over JOB_SLOTS
// synchronous slots, forked from and joined back into the caller's stream.
int run_host(mgcm_rt_handle *h, int nbatch, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out) {
    cudaStream_t ust = sync_stream(h);
    if (!h->user_stream) {
        if (const int rc = after_legacy_stream(*h->slots[0], ust)) return rc;
    }
    CK(cudaEventRecord(h->fork, ust));
    for (auto &s : h->slots) CK(cudaStreamWaitEvent(s->stream, h->fork, 0));
    uint32_t acc = 0;
    long long cols = 0, systems = 0;
    int nk = 0, k = 0;
    bool used[JOB_SLOTS] = {};
    for (int b = 0; b < nbatch; ++b) {
        const Sizes z = sizes_of(in[b]);
        int c0 = 0;
        for (const int c1 : job_ends((int)z.ncol, SYNC_JOB_COLS, SYNC_RAMP_COLS)) {
            Slot &sl = *h->slots[k % JOB_SLOTS];
            if (used[k % JOB_SLOTS]) {   // the slot's previous job must finish before its buffers are reused
                CK(cudaEventSynchronize(sl.done));
                acc |= *sl.h_status;
                systems += (long long)*sl.h_nsys;
            }
            const int rc = issue_job(h, sl, sl.stream, in[b], out[b], c0, c1);
            if (rc) {   // jobs already issued may still copy to or from the caller's buffers
                for (auto &s : h->slots) cudaStreamSynchronize(s->stream);
                return rc;
            }
            used[k % JOB_SLOTS] = true;
            nk += sl.kernels;
            cols += c1 - c0;
            c0 = c1;
            ++k;
        }
    }
    for (int i = 0; i < JOB_SLOTS; ++i) {
        Slot &sl = *h->slots[i];
        if (used[i]) {
            CK(cudaEventSynchronize(sl.done));
            acc |= *sl.h_status;
            systems += (long long)*sl.h_nsys;
            CK(cudaStreamWaitEvent(ust, sl.done, 0));
        }
    }
    float ms = 0.f;
    if (used[0]) cudaEventElapsedTime(&ms, h->slots[0]->ev0, h->slots[0]->ev1);
    h->stats.gpu_ms = ms;
    h->stats.columns = cols;
    h->stats.systems = systems;
    h->stats.status = (int)acc;
    h->stats.kernels = nk;
    return status_to_code(acc);
}

// ---------------------------------------------------------------- tracer inputs
int check_tracers(const mgcm_rt_handle *h, const mgcm_rt_batch_tracers *in, const mgcm_rt_batch_out *out) {
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    if (in->ncol < 0) return MGCM_RT_EINVAL;
    if (in->nlayers < 1 || in->nlayers > MGCM_RT_MAX_LAYERS || in->nlayers > h->cfg.max_layers)
        return MGCM_RT_ELAYERS;
    if (in->ncol == 0) return MGCM_RT_OK;
    const void *req[] = {in->sigma, in->sol, in->plev, in->tlev, in->pmid, in->tmid, in->qh2o,
                         in->acosz, in->als, in->albi, in->pcol, in->detau, in->cumtauv,
                         out->fmnetv, out->fluxupv, out->fluxdnv, out->fmneti, out->fluxupi,
                         out->fluxdni, out->suntot, out->irtotal, out->qrad, out->nfluxtopv,
                         out->nfluxtopi, out->diffvt, out->dnvflux, out->dndiffv, out->dnirflux,
                         out->fluxsurf};
    for (const void *p : req)
        if (!p) return MGCM_RT_EINVAL;
    if (in->active_dust ? (!in->dust_mass || !in->dust_number) : !in->tauref) return MGCM_RT_EINVAL;
    if (in->cloudon && (!in->ice_mass || !in->ice_core_mass || !in->ice_number)) return MGCM_RT_EINVAL;
    if (!std::isfinite(in->ptrop) || !(in->ptrop > 0.0)) return MGCM_RT_ENONFINITE;
    if (!h->d_mie) return MGCM_RT_EIO;
    return MGCM_RT_OK;
}

// A state batch as the tracer batch it becomes once rt_prep has filled the
// level arrays (those pointers stay NULL here).
mgcm_rt_batch_tracers tracers_of_state(const mgcm_rt_batch_state &s) {
    mgcm_rt_batch_tracers t{};
    t.ncol = s.ncol;
    t.nlayers = s.nlayers;
    t.device_ptrs = s.device_ptrs;
    t.active_dust = s.active_dust;
    t.cloudon = s.cloudon;
    t.ptrop = s.ptrop;
    t.sigma = s.sigma;
    t.sol = s.sol;
    t.dust_mass = s.dust_mass;
    t.dust_number = s.dust_number;
    t.ice_mass = s.ice_mass;
    t.ice_core_mass = s.ice_core_mass;
    t.ice_number = s.ice_number;
    t.acosz = s.acosz;
    t.als = s.als;
    t.albi = s.albi;
    t.pcol = s.pcol;
    t.detau = s.detau;
    t.cumtauv = s.cumtauv;
    return t;
}

int check_state(const mgcm_rt_handle *h, const mgcm_rt_batch_state *in, const mgcm_rt_batch_out *out) {
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    if (in->ncol < 0) return MGCM_RT_EINVAL;
    if (in->nlayers < 1 || in->nlayers > MGCM_RT_MAX_LAYERS || in->nlayers > h->cfg.max_layers)
        return MGCM_RT_ELAYERS;
    if (in->ncol == 0) return MGCM_RT_OK;
    const void *req[] = {in->sigma, in->sol, in->pcol, in->t, in->tstrat, in->gt, in->acosz, in->als,
                         in->albi, in->detau, in->cumtauv, out->fmnetv, out->fluxupv, out->fluxdnv,
                         out->fmneti, out->fluxupi, out->fluxdni, out->suntot, out->irtotal, out->qrad,
                         out->nfluxtopv, out->nfluxtopi, out->diffvt, out->dnvflux, out->dndiffv,
                         out->dnirflux, out->fluxsurf};
    for (const void *p : req)
        if (!p) return MGCM_RT_EINVAL;
    if (in->active_water && !in->vapour) return MGCM_RT_EINVAL;
    if (in->active_dust ? (!in->dust_mass || !in->dust_number) : (!in->tautot || !in->conr))
        return MGCM_RT_EINVAL;
    if (in->cloudon && (!in->ice_mass || !in->ice_core_mass || !in->ice_number)) return MGCM_RT_EINVAL;
    if (!std::isfinite(in->ptrop) || !(in->ptrop > 0.0)) return MGCM_RT_ENONFINITE;
    if (!in->active_dust && (!std::isfinite(in->psf) || !(in->psf > 0.0) || !std::isfinite(in->rptau) ||
                             !(in->rptau > 0.0)))
        return MGCM_RT_ENONFINITE;
    if (in->active_water && !std::isfinite(in->mwratio)) return MGCM_RT_ENONFINITE;
    if (!h->d_mie) return MGCM_RT_EIO;
    return MGCM_RT_OK;
}

// One job of a tracer batch on a slot: compact inputs staged (host) or
// offset (device), the aerosol arrays filled by rt_aerosol, the pipeline,
// outputs copied back (host); records sl.done.  With a state batch (stt) the
// level arrays and the prescribed TAUREF are not inputs: rt_prep builds them
// from the column state first (into the caller's optional outputs, or the
// slot's aerosol arena).
int issue_tracer_job(mgcm_rt_handle *h, Slot &sl, cudaStream_t st, const mgcm_rt_batch_tracers &in,
                     const mgcm_rt_batch_out &out, int c0, int c1,
                     const mgcm_rt_batch_state *stt = nullptr) {
    NvtxRange nvtx_range("mgcm_rt tracer job");
    const size_t n = (size_t)(c1 - c0);
    const int L = in.nlayers, lev = 2 * L + 3, lev1 = lev + 1, nl = L + 1;
    SegDev sd{};
    sd.ncol = (int)n;
    sd.L = L;
    sd.col0 = 0;
    sd.ptrop = in.ptrop;
    AeroSeg as{};
    as.ncol = (int)n;
    as.L = L;
    as.active_dust = in.active_dust ? 1 : 0;
    as.cloudon = in.cloudon ? 1 : 0;
    std::vector<ArrSpec> arrs;
    auto add_in = [&](const double *p, size_t per, const double **f) {
        if (p) arrs.push_back({p, nullptr, per, 0, const_cast<double **>(f)});
    };
    auto add_out = [&](double *p, size_t per, double **f) { arrs.push_back({nullptr, p, per, 1, f}); };
    PrepSeg ps{};
    // prepared arrays the caller asked for (the others go to the arena below)
    double *prep_want[6] = {};
    double **prep_field[6] = {const_cast<double **>(&sd.plev), const_cast<double **>(&sd.tlev),
                              const_cast<double **>(&sd.pmid), const_cast<double **>(&sd.tmid),
                              const_cast<double **>(&sd.qh2o), const_cast<double **>(&as.tauref_in)};
    if (!stt) {
        add_in(in.plev, lev, &sd.plev);
        add_in(in.tlev, lev, &sd.tlev);
        add_in(in.pmid, lev, &sd.pmid);
        add_in(in.tmid, lev, &sd.tmid);
        add_in(in.qh2o, lev, &sd.qh2o);
        if (!in.active_dust) add_in(in.tauref, lev1, &as.tauref_in);
    } else {
        ps.ncol = (int)n;
        ps.L = L;
        ps.active_water = stt->active_water ? 1 : 0;
        ps.prescribed_dust = stt->active_dust ? 0 : 1;
        ps.ptrop = stt->ptrop;
        ps.psf = stt->psf;
        ps.rptau = stt->rptau;
        ps.mwratio = stt->mwratio;
        add_in(stt->t, L, &ps.t);
        add_in(stt->tstrat, 1, &ps.tstrat);
        add_in(stt->gt, 1, &ps.gt);
        if (ps.active_water) add_in(stt->vapour, L, &ps.vapour);
        if (ps.prescribed_dust) {
            add_in(stt->tautot, 1, &ps.tautot);
            add_in(stt->conr, 1, &ps.conr);
        }
        double *want[6] = {stt->plev, stt->tlev, stt->pmid, stt->tmid, stt->qh2o,
                           ps.prescribed_dust ? stt->tauref : nullptr};
        for (int i = 0; i < 6; ++i)
            if (want[i]) {
                prep_want[i] = want[i];
                add_out(want[i], i == 5 ? lev1 : lev, prep_field[i]);
            }
    }
    if (in.active_dust) {
        add_in(in.dust_mass, L, &as.dust_mass);
        add_in(in.dust_number, L, &as.dust_number);
    }
    if (in.cloudon) {
        add_in(in.ice_mass, L, &as.ice_mass);
        add_in(in.ice_core_mass, L, &as.ice_core);
        add_in(in.ice_number, L, &as.ice_number);
    }
    add_in(in.acosz, 1, &sd.acosz);
    add_in(in.als, 1, &sd.als);
    add_in(in.albi, 1, &sd.albi);
    add_in(in.pcol, 1, &sd.pcol);
    arrs.push_back({in.detau, in.detau, 119, 2, &sd.detau});
    arrs.push_back({in.cumtauv, in.cumtauv, 119, 2, &sd.cumtauv});
    add_out(out.fmnetv, nl, &sd.fmnetv);
    add_out(out.fluxupv, nl, &sd.fluxupv);
    add_out(out.fluxdnv, nl, &sd.fluxdnv);
    add_out(out.fmneti, nl, &sd.fmneti);
    add_out(out.fluxupi, nl, &sd.fluxupi);
    add_out(out.fluxdni, nl, &sd.fluxdni);
    add_out(out.suntot, nl, &sd.suntot);
    add_out(out.irtotal, nl, &sd.irtotal);
    add_out(out.qrad, nl, &sd.qrad);
    add_out(out.nfluxtopv, 1, &sd.nfluxtopv);
    add_out(out.nfluxtopi, 1, &sd.nfluxtopi);
    add_out(out.diffvt, 1, &sd.diffvt);
    add_out(out.dnvflux, 1, &sd.dnvflux);
    add_out(out.dndiffv, 1, &sd.dndiffv);
    add_out(out.dnirflux, 1, &sd.dnirflux);
    add_out(out.fluxsurf, 1, &sd.fluxsurf);
    if (in.device_ptrs) {
        for (auto &a : arrs) *a.seg_field = const_cast<double *>(a.src ? a.src : a.dst) + (size_t)c0 * a.per_col;
        sd.sigma = in.sigma;
        sd.sol = in.sol;
    } else {
        size_t bytes = ((lev + 8) * 8 + 255) / 256 * 256;
        for (const auto &a : arrs) bytes += ((a.per_col * n * 8 + 255) / 256) * 256;
        const int rc = arena_ensure(h, sl.stage, bytes, st);
        if (rc) return rc;
        char *base = static_cast<char *>(sl.stage.ptr);
        size_t off = 0;
        for (auto &a : arrs) {
            double *d = reinterpret_cast<double *>(base + off);
            off += ((a.per_col * n * 8 + 255) / 256) * 256;
            *a.seg_field = d;
            a.dev = d;
            if (a.dir != 1)
                CK(cudaMemcpyAsync(d, a.src + (size_t)c0 * a.per_col, a.per_col * n * 8,
                                   cudaMemcpyHostToDevice, st));
        }
        double *ds = reinterpret_cast<double *>(base + off);
        CK(cudaMemcpyAsync(ds, in.sigma, lev * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ds + lev, in.sol, 7 * 8, cudaMemcpyHostToDevice, st));
        sd.sigma = ds;
        sd.sol = ds + lev;
    }
    // the per-level aerosol arrays of the ABI, on the device (+ the prepared
    // level arrays of a state batch that the caller does not take)
    // (prescribed dust needs no per-level arrays: the stage reads the band
    // constants, SegDev::dust_band, and TAUREF as given)
    const size_t per = (size_t)lev1 * (2 + 3 * (AERO_NV + AERO_NI));
    const size_t prep_per = stt ? (size_t)5 * lev + lev1 : 0;
    const size_t abytes = n * (per * ((in.active_dust ? 1 : 0) + (in.cloudon ? 1 : 0)) + prep_per) * 8;
    int rc = arena_ensure(h, sl.aero, abytes, st);
    if (rc) return rc;
    double *ap = static_cast<double *>(sl.aero.ptr);
    auto take = [&](size_t per_col) { double *r = ap; ap += per_col * n; return r; };
    if (stt) {
        for (int i = 0; i < 6; ++i) {
            double *d = take(i == 5 ? lev1 : lev);
            if (!prep_want[i]) *prep_field[i] = d;
        }
        ps.sigma = sd.sigma;
        ps.pcol = sd.pcol;
        ps.plev = const_cast<double *>(sd.plev);
        ps.tlev = const_cast<double *>(sd.tlev);
        ps.pmid = const_cast<double *>(sd.pmid);
        ps.tmid = const_cast<double *>(sd.tmid);
        ps.qh2o = const_cast<double *>(sd.qh2o);
        ps.tauref = const_cast<double *>(as.tauref_in);
    }
    if (in.active_dust) {
        as.tauref = take(lev1);
        as.qextrefdst = take(lev1);
        as.qxvdst = take((size_t)AERO_NV * lev1);
        as.qsvdst = take((size_t)AERO_NV * lev1);
        as.gvdst = take((size_t)AERO_NV * lev1);
        as.qxidst = take((size_t)AERO_NI * lev1);
        as.qsidst = take((size_t)AERO_NI * lev1);
        as.gidst = take((size_t)AERO_NI * lev1);
    }
    if (in.cloudon) {
        as.taurefcld = take(lev1);
        as.qextrefcld = take(lev1);
        as.qxvcld = take((size_t)AERO_NV * lev1);
        as.qsvcld = take((size_t)AERO_NV * lev1);
        as.gvcld = take((size_t)AERO_NV * lev1);
        as.qxicld = take((size_t)AERO_NI * lev1);
        as.qsicld = take((size_t)AERO_NI * lev1);
        as.gicld = take((size_t)AERO_NI * lev1);
    }
    as.plev = sd.plev;
    if (!in.active_dust) {
        sd.dust_band = h->d_mie + AERO_MIE_SIZE;
        as.tauref = nullptr;   // rt_aerosol leaves the dust alone
    }
    sd.tauref = in.active_dust ? as.tauref : as.tauref_in;
    sd.qextrefdst = as.qextrefdst;
    sd.qxvdst = as.qxvdst;
    sd.qsvdst = as.qsvdst;
    sd.gvdst = as.gvdst;
    sd.qxidst = as.qxidst;
    sd.qsidst = as.qsidst;
    sd.gidst = as.gidst;
    sd.taurefcld = as.taurefcld;
    sd.qextrefcld = as.qextrefcld;
    sd.qxvcld = as.qxvcld;
    sd.qsvcld = as.qsvcld;
    sd.gvcld = as.gvcld;
    sd.qxicld = as.qxicld;
    sd.qsicld = as.qsicld;
    sd.gicld = as.gicld;
    SegTable &tab = *sl.h_segs;
    tab.nseg = 1;
    tab.total_cols = (int)n;
    tab.seg[0] = sd;
    CK(cudaMemcpyAsync(sl.d_segs, sl.h_segs, offsetof(SegTable, seg) + sizeof(SegDev),
                       cudaMemcpyHostToDevice, st));
    if (stt) {
        const int pg = (int)std::min<long long>(((long long)n + PREP_THREADS / 32 - 1) / (PREP_THREADS / 32),
                                                (long long)h->num_sms * 16);
        rt_prep<<<pg, PREP_THREADS, 0, st>>>(ps);
        CK(cudaGetLastError());
    }
    // a warp per column, AERO_WARPS columns per CTA, up to 8 CTAs per SM resident
    const int ag = (int)std::min<long long>(((long long)n + AERO_WARPS - 1) / AERO_WARPS,
                                            (long long)h->num_sms * 8);
    rt_aerosol<<<ag, 32 * AERO_WARPS, 0, st>>>(as, h->aero, h->d_mie);
    CK(cudaGetLastError());
    rc = launch_all(h, sl, st, (int)n, nl, 1 << 30);
    if (rc) return rc;
    sl.kernels += stt ? 2 : 1;   // rt_aerosol (+ rt_prep)
    if (!in.device_ptrs)
        for (auto &a : arrs)
            if (a.dir != 0)
                CK(cudaMemcpyAsync(a.dst + (size_t)c0 * a.per_col, a.dev, a.per_col * n * 8,
                                   cudaMemcpyDeviceToHost, st));
    rc = post_status(sl, st);
    if (rc) return rc;
    CK(cudaEventRecord(sl.done, st));
    return MGCM_RT_OK;
}

// Synchronous tracer (or state) batch: jobs alternate between the two
// synchronous slots.
int run_tracers(mgcm_rt_handle *h, const mgcm_rt_batch_tracers &in, mgcm_rt_batch_out &out,
                const mgcm_rt_batch_state *stt = nullptr) {
    cudaStream_t ust = sync_stream(h);
    if (!h->user_stream) {
        if (const int rc = after_legacy_stream(*h->slots[0], ust)) return rc;
    }
    CK(cudaEventRecord(h->fork, ust));
    for (auto &s : h->slots) CK(cudaStreamWaitEvent(s->stream, h->fork, 0));
    uint32_t acc = 0;
    long long systems = 0;
    int nk = 0, k = 0;
    bool used[JOB_SLOTS] = {};
    const std::vector<int> ends = in.device_ptrs ? job_ends(in.ncol, 4 * SYNC_JOB_COLS, 0)
                                                 : job_ends(in.ncol, SYNC_JOB_COLS, SYNC_RAMP_COLS);
    int c0 = 0;
    for (const int c1 : ends) {
        Slot &sl = *h->slots[k % JOB_SLOTS];
        if (used[k % JOB_SLOTS]) {
            CK(cudaEventSynchronize(sl.done));
            acc |= *sl.h_status;
            systems += (long long)*sl.h_nsys;
        }
        const int rc = issue_tracer_job(h, sl, sl.stream, in, out, c0, c1, stt);
        if (rc) {   // jobs already issued may still copy to or from the caller's buffers
            for (auto &s : h->slots) cudaStreamSynchronize(s->stream);
            return rc;
        }
        used[k % JOB_SLOTS] = true;
        nk += sl.kernels;
        c0 = c1;
        ++k;
    }
    for (int i = 0; i < JOB_SLOTS; ++i) {
        Slot &sl = *h->slots[i];
        if (used[i]) {
            CK(cudaEventSynchronize(sl.done));
            acc |= *sl.h_status;
            systems += (long long)*sl.h_nsys;
            CK(cudaStreamWaitEvent(ust, sl.done, 0));
        }
    }
    float ms = 0.f;
    if (used[0]) cudaEventElapsedTime(&ms, h->slots[0]->ev0, h->slots[0]->ev1);
    h->stats.gpu_ms = ms;
    h->stats.columns = in.ncol;
    h->stats.systems = systems;
    h->stats.status = (int)acc;
    h->stats.kernels = nk;
    return status_to_code(acc);
}

int run_batches(mgcm_rt_handle *h, int nbatch, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out,
                bool async) {
    if (nbatch < 1 || nbatch > MAX_SEGS) return MGCM_RT_EINVAL;
    const auto t0 = std::chrono::steady_clock::now();
    const int kind = in[0].device_ptrs ? 1 : 0;
    if (async && !kind) return MGCM_RT_EINVAL;
    for (int b = 0; b < nbatch; ++b) {
        const int rc = check_args(h, &in[b], &out[b]);
        if (rc) return rc;
        if ((in[b].device_ptrs ? 1 : 0) != kind) return MGCM_RT_EINVAL;
    }
    int rc = finish_pending(h);
    if (rc) return rc;
    rc = kind ? run_device(h, nbatch, in, out, async) : run_host(h, nbatch, in, out);
    h->stats.total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

// ---------------------------------------------------------------- serving
void finish_job(mgcm_rt_handle *h, Slot &sl) {
    std::shared_ptr<Request> r = sl.job.req;
    const int code = status_to_code(*sl.h_status);
    float b = 0.f, e = 0.f;
    const bool timed = cudaEventElapsedTime(&b, h->epoch, sl.ev0) == cudaSuccess &&
                       cudaEventElapsedTime(&e, h->epoch, sl.ev1) == cudaSuccess;
    sl.busy = false;
    sl.job = Job{};
    std::lock_guard<std::mutex> lk(h->qmu);
    --h->outstanding;
    if (timed) {
        r->dev_begin = std::min(r->dev_begin, (double)b);
        r->dev_end = std::max(r->dev_end, (double)e);
    }
    if (code && !r->status) r->status = code;
    if (--r->jobs_left == 0) {
        r->done = true;
        r->t_done = std::chrono::steady_clock::now();
        h->dcv.notify_all();
    }
}

void fail_job(mgcm_rt_handle *h, Job &j, int code) {
    std::lock_guard<std::mutex> lk(h->qmu);
    --h->outstanding;
    if (!j.req->status) j.req->status = code;
    if (--j.req->jobs_left == 0) {
        j.req->done = true;
        j.req->t_done = std::chrono::steady_clock::now();
        h->dcv.notify_all();
    }
}

void worker_main(mgcm_rt_handle *h) {
    cudaSetDevice(h->device);
    cudaEventRecord(h->epoch, nullptr);   // before any job of this worker
    for (;;) {
        bool any_busy = false;
        for (auto &s : h->sslots)
            if (s->busy) {
                if (cudaEventQuery(s->done) == cudaSuccess) finish_job(h, *s);
                else any_busy = true;
            }
        for (;;) {   // admit jobs onto free slots
            Job j;
            {
                std::lock_guard<std::mutex> lk(h->qmu);
                if (h->jobs.empty()) break;
                j = h->jobs.front();
            }
            Slot *free_slot = nullptr;
            for (auto &s : h->sslots)
                if (!s->busy) { free_slot = s.get(); break; }
            if (!free_slot && (int)h->sslots.size() < SERVE_SLOTS) {
                auto s = std::make_unique<Slot>();
                if (slot_init(*s) == MGCM_RT_OK) {
                    h->sslots.push_back(std::move(s));
                    free_slot = h->sslots.back().get();
                }
            }
            if (!free_slot) break;
            {
                std::lock_guard<std::mutex> lk(h->qmu);
                h->jobs.pop_front();
            }
            const int rc = issue_job(h, *free_slot, free_slot->stream, j.req->in[j.seg], j.req->out[j.seg],
                                     j.c0, j.c1);
            if (rc == MGCM_RT_ENOMEM && any_busy) {   // admitted later, when memory frees up
                std::lock_guard<std::mutex> lk(h->qmu);
                ++j.req->deferred;
                h->jobs.push_front(j);
                break;
            }
            if (rc) {
                fail_job(h, j, rc);
                continue;
            }
            free_slot->busy = true;
            free_slot->job = j;
            any_busy = true;
        }
        std::unique_lock<std::mutex> lk(h->qmu);
        if (h->stop && h->jobs.empty() && !any_busy) return;
        if (any_busy)
            h->qcv.wait_for(lk, std::chrono::microseconds(50));
        else
            h->qcv.wait(lk, [&] { return h->stop || !h->jobs.empty(); });
    }
}

}  // namespace

extern "C" {

const char *mgcm_rt_version(void) { return "mgcm-rt-b200 0.2 (Legacy Mars GCM v24 radiation)"; }

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

}  // extern "C"
namespace {
int noalloc_scratch(int device, unsigned char **ptr);
}  // namespace
extern "C" {

mgcm_rt_handle *mgcm_rt_create(const mgcm_rt_config *cfg, const char *data_dir, int *status) {
    int dummy;
    if (!status) status = &dummy;
    if (!cfg || !data_dir) { *status = MGCM_RT_EINVAL; return nullptr; }
    if (cfg->max_layers < 1 || cfg->max_layers > MGCM_RT_MAX_LAYERS) { *status = MGCM_RT_ELAYERS; return nullptr; }
    if (cfg->precision != MGCM_RT_FP64 && cfg->precision != MGCM_RT_MIXED) { *status = MGCM_RT_EINVAL; return nullptr; }
    auto h = std::make_unique<mgcm_rt_handle>();
    h->cfg = *cfg;
    if (load_tables(data_dir, h->host)) { *status = MGCM_RT_EIO; return nullptr; }
    h->device = cfg->device;
    if (cudaSetDevice(h->device) != cudaSuccess) { *status = MGCM_RT_ECUDA; return nullptr; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess) { *status = MGCM_RT_ECUDA; return nullptr; }
    if (const int rc = configure_kernels(h->device)) { *status = rc; return nullptr; }
    {   // the no-allocation entry point's static scratch: resolve its device
        // address now, while allocating is allowed, so that loading the
        // module that holds it never happens inside mgcm_rt_run_noalloc
        unsigned char *scr = nullptr;
        if (const int rc = noalloc_scratch(h->device, &scr)) { *status = rc; return nullptr; }
    }
    {   // The solve kernels keep per-system arrays in local memory, and the
        // driver grows a context's local-memory pool at the first launch
        // that needs more (about 2 GB here).  Reserve it now, while
        // allocating is allowed, through the per-thread stack limit, so that
        // no later call -- mgcm_rt_run_noalloc in particular -- allocates.
        size_t need = 0, cur = 0;
        for (const void *f : {(const void *)rt_fp64_kernel, (const void *)rt_fp64_solve<true>,
                              (const void *)rt_fp64_solve<false>, (const void *)rt_mixed_solve_vis,
                              (const void *)rt_fp64_screen<false>, (const void *)rt_fp64_screen<true>}) {
            cudaFuncAttributes fa{};
            if (cudaFuncGetAttributes(&fa, f) != cudaSuccess) { *status = MGCM_RT_ECUDA; return nullptr; }
            need = std::max(need, (size_t)fa.localSizeBytes);
        }
        need = (need + 1024 + 15) / 16 * 16;
        if (cudaDeviceGetLimit(&cur, cudaLimitStackSize) != cudaSuccess) { *status = MGCM_RT_ECUDA; return nullptr; }
        if (cur < need && cudaDeviceSetLimit(cudaLimitStackSize, need) != cudaSuccess) {
            *status = MGCM_RT_ENOMEM;
            return nullptr;
        }
    }
    if (cfg->solver < MGCM_RT_SOLVER_AUTO || cfg->solver > MGCM_RT_SOLVER_FUSED) { *status = MGCM_RT_EINVAL; return nullptr; }
    h->fused = cfg->solver == MGCM_RT_SOLVER_FUSED;
    h->tmem = cfg->solver == MGCM_RT_SOLVER_TMEM;
    h->quad = cfg->solver == MGCM_RT_SOLVER_QUAD;
    h->onchip = cfg->solver == MGCM_RT_SOLVER_ONCHIP;
    h->num_sms = prop.multiProcessorCount;
    auto fail = [&](int code) { mgcm_rt_destroy(h.release()); *status = code; return nullptr; };
    for (int i = 0; i < SYNC_SLOTS; ++i) {
        h->slots.push_back(std::make_unique<Slot>());
        if (slot_init(*h->slots.back())) return fail(MGCM_RT_ECUDA);
    }
    if (cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming)) return fail(MGCM_RT_ECUDA);
    RtConst &K = h->K;
    std::memcpy(K.tauray, h->host.tauray, sizeof(K.tauray));
    std::memcpy(K.fzerov, h->host.fzerov, sizeof(K.fzerov));
    std::memcpy(K.fzeroi, h->host.fzeroi, sizeof(K.fzeroi));
    std::memcpy(K.gweight, h->host.gweight, sizeof(K.gweight));
    std::memcpy(K.dwni, h->host.dwni, sizeof(K.dwni));
    std::memcpy(K.pfgasref, h->host.pfgasref, sizeof(K.pfgasref));
    std::memcpy(K.plimit, h->host.plimit, sizeof(K.plimit));
    std::memcpy(K.wrefh2o, h->host.wrefh2o, sizeof(K.wrefh2o));
    std::vector<double> kv, ki;
    gauss_fastest(h->host, kv, ki);
    // FP32 tables hold Cmk*k (optical depth per mbar): k itself reaches 1e-49,
    // below the FP32 range (code/optcv.f90:104-105,164, U = Cmk*DPR)
    std::vector<float> kvf(kv.size());
    for (size_t q = 0; q < kv.size(); ++q) kvf[q] = (float)(3.51e22 * kv[q]);
    if (cudaMalloc(&h->d_kv, kv.size() * 8) || cudaMalloc(&h->d_ki, ki.size() * 8) ||
        cudaMalloc(&h->d_kvf, kvf.size() * 4) ||
        cudaMalloc(&h->d_planck, h->host.planckir.size() * 8))
        return fail(MGCM_RT_ENOMEM);
    if (cudaMemcpy(h->d_kv, kv.data(), kv.size() * 8, cudaMemcpyHostToDevice) ||
        cudaMemcpy(h->d_ki, ki.data(), ki.size() * 8, cudaMemcpyHostToDevice) ||
        cudaMemcpy(h->d_kvf, kvf.data(), kvf.size() * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(h->d_planck, h->host.planckir.data(), h->host.planckir.size() * 8, cudaMemcpyHostToDevice))
        return fail(MGCM_RT_ECUDA);
    {   // aerosol optics tables: optional (mgcm_rt_run_tracers returns EIO without them)
        AerosolTables at;
        if (load_aerosol_tables(data_dir, at) == 0) {
            AeroConst &A = h->aero;
            std::memcpy(A.radb, at.radb, sizeof(A.radb));
            for (int j = 0; j < AERO_NRATIO; ++j) A.cor_ratio[j] = (float)at.cor_ratio[j];
            std::memcpy(A.qextv, at.qextv, sizeof(A.qextv));
            std::memcpy(A.qscatv, at.qscatv, sizeof(A.qscatv));
            std::memcpy(A.gv, at.gv, sizeof(A.gv));
            std::memcpy(A.qexti, at.qexti, sizeof(A.qexti));
            std::memcpy(A.qscati, at.qscati, sizeof(A.qscati));
            std::memcpy(A.gi, at.gi, sizeof(A.gi));
            std::vector<double> mie;
            mie.reserve(AERO_MIE_SIZE);
            for (int m = 0; m < 3; ++m)
                for (int i = 0; i < AERO_NBIN; ++i)
                    for (int l = 0; l < AERO_NV; ++l) mie.push_back(at.dst_v[m][i][l]);
            for (int m = 0; m < 3; ++m)
                for (int i = 0; i < AERO_NBIN; ++i)
                    for (int l = 0; l < AERO_NI; ++l) mie.push_back(at.dst_i[m][i][l]);
            for (int m = 0; m < 3; ++m)
                for (int j = 0; j < AERO_NRATIO; ++j)
                    for (int i = 0; i < AERO_NBIN; ++i)
                        for (int l = 0; l < AERO_NV; ++l) mie.push_back(at.cld_v[m][j][i][l]);
            for (int m = 0; m < 3; ++m)
                for (int j = 0; j < AERO_NRATIO; ++j)
                    for (int i = 0; i < AERO_NBIN; ++i)
                        for (int l = 0; l < AERO_NI; ++l) mie.push_back(at.cld_i[m][j][i][l]);
            // then the prescribed dust band properties (SegDev::dust_band order)
            for (const double *p : {A.qextv, A.qscatv, A.gv}) mie.insert(mie.end(), p, p + AERO_NV);
            for (const double *p : {A.qexti, A.qscati, A.gi}) mie.insert(mie.end(), p, p + AERO_NI);
            if (cudaMalloc(&h->d_mie, mie.size() * 8) ||
                cudaMemcpy(h->d_mie, mie.data(), mie.size() * 8, cudaMemcpyHostToDevice))
                return fail(MGCM_RT_ENOMEM);
        }
    }
    if (cfg->max_queued_jobs < 0) return fail(MGCM_RT_EINVAL);
    if (cfg->max_queued_jobs > 0) h->max_jobs = cfg->max_queued_jobs;
    if (cudaEventCreate(&h->epoch) != cudaSuccess) return fail(MGCM_RT_ECUDA);
    h->t_epoch = std::chrono::steady_clock::now();
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    h->budget = cfg->hbm_budget ? cfg->hbm_budget : freeb / 4 * 3;
    *status = MGCM_RT_OK;
    return h.release();
}

void mgcm_rt_destroy(mgcm_rt_handle *h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->worker.joinable()) {
        {
            std::lock_guard<std::mutex> lk(h->qmu);
            h->stop = true;
        }
        h->qcv.notify_all();
        h->worker.join();
    }
    for (auto &s : h->sslots) slot_free(h, *s);
    for (auto &s : h->slots) slot_free(h, *s);
    cudaFree(h->d_kv);
    cudaFree(h->d_ki);
    cudaFree(h->d_kvf);
    cudaFree(h->d_mie);
    cudaFree(h->d_planck);
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->epoch) cudaEventDestroy(h->epoch);
    delete h;
}

int mgcm_rt_run(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out) {
    NvtxRange nvtx_range("mgcm_rt_run");
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    return run_batches(h, 1, in, out, false);
}

int mgcm_rt_run_multi(mgcm_rt_handle *h, int nbatch, const mgcm_rt_batch_in *in,
                      mgcm_rt_batch_out *out) {
    NvtxRange nvtx_range("mgcm_rt_run_multi");
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    return run_batches(h, nbatch, in, out, false);
}

int mgcm_rt_enqueue(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out) {
    NvtxRange nvtx_range("mgcm_rt_enqueue");
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    return run_batches(h, 1, in, out, true);
}

int mgcm_rt_sync(mgcm_rt_handle *h) {
    if (!h) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    if (!h->pending) {
        CK(cudaStreamSynchronize(sync_stream(h)));
        return MGCM_RT_OK;
    }
    return finish_pending(h);
}

int mgcm_rt_set_stream(mgcm_rt_handle *h, void *cuda_stream) {
    if (!h) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    const int rc = finish_pending(h);
    if (rc) return rc;
    CK(cudaStreamSynchronize(sync_stream(h)));
    h->user_stream = static_cast<cudaStream_t>(cuda_stream);
    return MGCM_RT_OK;
}

int mgcm_rt_get_stats(mgcm_rt_handle *h, mgcm_rt_stats *st) {
    if (!h || !st) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    *st = h->stats;
    std::lock_guard<std::mutex> mk(h->mem_mu);
    st->hbm_used = (long long)h->used;
    st->hbm_budget = (long long)h->budget;
    return MGCM_RT_OK;
}

int mgcm_rt_dsolflux(mgcm_rt_handle *h, int ncol, int device_ptrs, const double *sol,
                     const double *acosz, const double *detau, const double *dndiffv,
                     double *dnvflux) {
    if (!h || ncol < 0 || !sol || !acosz || !detau || !dndiffv || !dnvflux) return MGCM_RT_EINVAL;
    if (ncol == 0) return MGCM_RT_OK;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    int rc = finish_pending(h);
    if (rc) return rc;
    Slot &sl = *h->slots[0];
    cudaStream_t st = sync_stream(h);
    if (device_ptrs && !h->user_stream) {
        if (const int rc = after_legacy_stream(*h->slots[0], st)) return rc;
    }
    const double *ds = sol, *da = acosz, *dd = detau, *dn = dndiffv;
    double *dout = dnvflux;
    if (!device_ptrs) {
        const size_t n = (size_t)ncol;
        const size_t bytes = 8 * (8 + n + 119 * n + n + n) + 5 * 256;
        rc = arena_ensure(h, sl.stage, bytes, st);
        if (rc) return rc;
        double *p = static_cast<double *>(sl.stage.ptr);
        double *pa = p + 8, *pd = pa + n, *pn = pd + 119 * n, *po = pn + n;
        CK(cudaMemcpyAsync(p, sol, 7 * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(pa, acosz, n * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(pd, detau, 119 * n * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(pn, dndiffv, n * 8, cudaMemcpyHostToDevice, st));
        ds = p; da = pa; dd = pd; dn = pn; dout = po;
    }
    rt_dsolflux_kernel<<<(ncol + 127) / 128, 128, 0, st>>>(ncol, ds, da, dd, dn, dout, h->K);
    CK(cudaGetLastError());
    if (!device_ptrs) CK(cudaMemcpyAsync(dnvflux, dout, (size_t)ncol * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return MGCM_RT_OK;
}

int mgcm_rt_debug_bins(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, int *mt, int *mp, int *nh2o,
                       int *nplanck, double *wratio, double *lcoef) {
    if (!h || !in || !mt || !mp || !nh2o || !nplanck || !wratio || !lcoef) return MGCM_RT_EINVAL;
    if (!in->device_ptrs) return MGCM_RT_EINVAL;
    mgcm_rt_batch_out none{};
    const int ac = check_args(h, in, &none);
    if (ac != MGCM_RT_OK && ac != MGCM_RT_EINVAL) return ac;
    if (in->ncol < 0 || !in->plev || !in->tlev || !in->pmid || !in->tmid || !in->qh2o || !in->tauref ||
        !in->qextrefdst || !in->qxvdst || !in->sigma || !in->sol)
        return MGCM_RT_EINVAL;
    if (in->taurefcld && !in->qextrefcld) return MGCM_RT_EINVAL;
    if (in->ncol == 0) return MGCM_RT_OK;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    if (int rc = finish_pending(h)) return rc;
    Slot &sl = *h->slots[0];
    cudaStream_t st = sync_stream(h);
    if (!h->user_stream) {
        if (const int rc0 = after_legacy_stream(sl, st)) return rc0;
    }
    const Sizes z = sizes_of(*in);
    SegDev sd{};
    sd.ncol = (int)z.ncol;
    sd.L = z.L;
    sd.col0 = 0;
    sd.ptrop = in->ptrop;
    fill_direct(sd, *in, none);
    sd.sigma = in->sigma;
    sd.sol = in->sol;
    SegTable &tab = *sl.h_segs;
    tab.nseg = 1;
    tab.total_cols = (int)z.ncol;
    tab.seg[0] = sd;
    size_t stride = 0;
    pipe_bytes_per_col(z.nl, &stride);
    unsigned char *blocks = nullptr;
    if (cudaMalloc(&blocks, z.ncol * stride) != cudaSuccess) return MGCM_RT_ENOMEM;
    int rc = MGCM_RT_OK;
    do {
        if (cudaMemcpyAsync(sl.d_segs, sl.h_segs, offsetof(SegTable, seg) + sizeof(SegDev),
                            cudaMemcpyHostToDevice, st) ||
            cudaMemsetAsync(sl.d_status, 0, 256, st)) { rc = MGCM_RT_ECUDA; break; }
        const int g0 = std::min<int>(((int)z.ncol + 3) / 4, h->num_sms * 4);
        rt_stage<<<g0, STAGE_THREADS, 0, st>>>(sl.d_segs, 0, (int)z.ncol, z.nl, blocks, stride, h->d_planck,
                                               h->K, sl.d_status);
        const long long items = (long long)z.ncol * z.lev;
        const int g1 = (int)std::min<long long>((items + 255) / 256, (long long)h->num_sms * 8);
        rt_bins_decode<<<g1, 256, 0, st>>>(sl.d_segs, (int)z.ncol, z.nl, blocks, stride, sl.d_status, mt, mp,
                                           nh2o, nplanck, wratio, lcoef);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(sl.h_status, sl.d_status, 4, cudaMemcpyDeviceToHost, st) ||
            cudaStreamSynchronize(st)) { rc = MGCM_RT_ECUDA; break; }
        rc = status_to_code(*sl.h_status);
    } while (0);
    cudaFree(blocks);
    return rc;
}

int mgcm_rt_run_state(mgcm_rt_handle *h, const mgcm_rt_batch_state *in, mgcm_rt_batch_out *out) {
    NvtxRange nvtx_range("mgcm_rt_run_state");
    const int rc = check_state(h, in, out);
    if (rc || in->ncol == 0) return rc;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    const int prc = finish_pending(h);
    if (prc) return prc;
    const mgcm_rt_batch_tracers t = tracers_of_state(*in);
    return run_tracers(h, t, *out, in);
}

int mgcm_rt_run_tracers(mgcm_rt_handle *h, const mgcm_rt_batch_tracers *in, mgcm_rt_batch_out *out) {
    NvtxRange nvtx_range("mgcm_rt_run_tracers");
    const int rc = check_tracers(h, in, out);
    if (rc || in->ncol == 0) return rc;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    const int prc = finish_pending(h);
    if (prc) return prc;
    return run_tracers(h, *in, *out);
}

int mgcm_rt_submit(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out,
                   long long *ticket) {
    if (!h || !in || !out || !ticket) return MGCM_RT_EINVAL;
    const int rc = check_args(h, in, out);
    if (rc) return rc;
    auto r = std::make_shared<Request>();
    r->in.push_back(*in);
    r->out.push_back(*out);
    r->t_submit = std::chrono::steady_clock::now();
    const int ncol = in->ncol;
    const int njobs = (ncol + SERVE_JOB_COLS - 1) / SERVE_JOB_COLS;
    std::lock_guard<std::mutex> lk(h->qmu);
    // queue full: the request's jobs would take the accepted-and-unfinished
    // jobs above the handle's limit (mgcm_rt_config.max_queued_jobs)
    if (h->outstanding + njobs > h->max_jobs) return MGCM_RT_EBUSY;
    if (!h->worker.joinable()) {
        h->stop = false;
        h->worker = std::thread(worker_main, h);
    }
    *ticket = h->next_ticket++;
    h->reqs[*ticket] = r;
    if (ncol == 0) {
        r->done = true;
        r->t_done = r->t_submit;
        return MGCM_RT_OK;
    }
    for (int c0 = 0; c0 < ncol; c0 += SERVE_JOB_COLS) {
        Job j;
        j.req = r;
        j.seg = 0;
        j.c0 = c0;
        j.c1 = std::min(ncol, c0 + SERVE_JOB_COLS);
        ++r->jobs_left;
        ++r->jobs;
        ++h->outstanding;
        h->jobs.push_back(j);
    }
    h->qcv.notify_all();
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

int mgcm_rt_get_request_info(mgcm_rt_handle *h, long long ticket, mgcm_rt_request_info *info) {
    if (!h || !info) return MGCM_RT_EINVAL;
    std::lock_guard<std::mutex> lk(h->qmu);
    auto it = h->reqs.find(ticket);
    if (it == h->reqs.end()) return MGCM_RT_ENOTFOUND;
    const Request &r = *it->second;
    auto ms = [&](std::chrono::steady_clock::time_point t) {
        return std::chrono::duration<double, std::milli>(t - h->t_epoch).count();
    };
    *info = mgcm_rt_request_info{};
    info->done = r.done ? 1 : 0;
    info->status = r.status;
    info->jobs = r.jobs;
    info->deferred = r.deferred;
    info->submit_ms = ms(r.t_submit);
    info->done_ms = r.done ? ms(r.t_done) : -1.0;
    const bool dev = r.dev_end >= r.dev_begin;
    info->device_begin_ms = dev ? r.dev_begin : -1.0;
    info->device_end_ms = dev ? r.dev_end : -1.0;
    return MGCM_RT_OK;
}

int mgcm_rt_wait(mgcm_rt_handle *h, long long ticket, double timeout_s) {
    if (!h) return MGCM_RT_EINVAL;
    std::unique_lock<std::mutex> lk(h->qmu);
    auto it = h->reqs.find(ticket);
    if (it == h->reqs.end()) return MGCM_RT_ENOTFOUND;
    std::shared_ptr<Request> r = it->second;
    if (timeout_s < 0) {
        h->dcv.wait(lk, [&] { return r->done; });
    } else if (!h->dcv.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->done; })) {
        return MGCM_RT_ETIMEOUT;
    }
    h->reqs.erase(ticket);
    return r->status;
}
}

// ---------------------------------------------------------------------------
// Captured uneven batches: segment tables built once, launch shape
// autotuned, the pipeline captured into a CUDA graph.  As for device-pointer
// calls, the columns are split into up to SYNC_SLOTS concurrent parts (part 0
// on the graph's slot, the others on their own slots, forked and joined
// inside the graph); the fused form runs as one part.
struct mgcm_rt_graph {
    mgcm_rt_handle *h = nullptr;
    Slot slot;                        // part 0
    Slot parts[SYNC_SLOTS - 1];       // parts 1 .. nparts-1
    int nparts = 1, ncols[SYNC_SLOTS] = {}, part_nl[SYNC_SLOTS] = {};
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int total = 0, max_nl = 1, max_chunk = 1;
    mgcm_rt_tune info{};
    Slot &part(int p) { return p == 0 ? slot : parts[p - 1]; }
};

namespace {

// One eager pass over the first `cols` columns with shape t; returns ms.
int time_shape(mgcm_rt_graph *g, const Tune &t, int cols, float &ms) {
    mgcm_rt_handle *h = g->h;
    Slot &sl = g->slot;
    cudaStream_t st = sl.stream;
    sl.tune = t;
    int nk = 0;
    float best = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
        CK(cudaMemsetAsync(sl.d_status, 0, 256, st));
        CK(cudaEventRecord(sl.ev0, st));
        int rc = launch_body(h, sl, st, cols, g->part_nl[0], nk, g->max_chunk);
        if (rc) return rc;
        CK(cudaEventRecord(sl.ev1, st));
        CK(cudaStreamSynchronize(st));
        float x = 0.f;
        cudaEventElapsedTime(&x, sl.ev0, sl.ev1);
        best = std::min(best, x);
    }
    ms = best;
    return MGCM_RT_OK;
}

void graph_free(mgcm_rt_graph *g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->fork) cudaEventDestroy(g->fork);
    if (g->h)
        for (int p = 0; p < g->nparts; ++p) slot_free(g->h, g->part(p));
    delete g;
}

}  // namespace

extern "C" {

int mgcm_rt_graph_create(mgcm_rt_handle *h, int nbatch, const mgcm_rt_batch_in *in,
                         mgcm_rt_batch_out *out, int autotune, mgcm_rt_graph **graph) {
    if (!h || !in || !out || !graph || nbatch < 1 || nbatch > MAX_SEGS) return MGCM_RT_EINVAL;
    *graph = nullptr;
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    for (int b = 0; b < nbatch; ++b) {
        const int rc = check_args(h, &in[b], &out[b]);
        if (rc) return rc;
        if (!in[b].device_ptrs) return MGCM_RT_EINVAL;
    }
    mgcm_rt_graph *g = new mgcm_rt_graph;
    g->h = h;
    auto fail = [&](int code) { graph_free(g); return code; };
    int total = 0, max_nl = 1;
    for (int b = 0; b < nbatch; ++b) {
        const Sizes z = sizes_of(in[b]);
        if ((long long)total + (long long)z.ncol > 0x7fffff) {
            delete g;
            return MGCM_RT_EINVAL;
        }
        total += (int)z.ncol;
        if (z.ncol) max_nl = std::max(max_nl, z.nl);
    }
    if (total == 0) {
        delete g;
        return MGCM_RT_EINVAL;
    }
    g->nparts = h->fused ? 1 : std::max(1, std::min(SYNC_SLOTS, total / SPLIT_COLS));
    for (int p = 0; p < g->nparts; ++p)
        if (slot_init(g->part(p))) {
            g->nparts = p + 1;   // slot_free the ones begun
            return fail(MGCM_RT_ECUDA);
        }
    if (cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming)) return fail(MGCM_RT_ECUDA);
    for (int p = 0; p < g->nparts; ++p) {
        Slot &ps = g->part(p);
        const int b0 = (int)((long long)total * p / g->nparts), b1 = (int)((long long)total * (p + 1) / g->nparts);
        int nl = 1;
        g->ncols[p] = table_of_range(*ps.h_segs, nbatch, in, out, b0, b1, nl);
        g->part_nl[p] = nl;
        if (cudaMemcpyAsync(ps.d_segs, ps.h_segs, sizeof(SegTable), cudaMemcpyHostToDevice, ps.stream) ||
            cudaStreamSynchronize(ps.stream))
            return fail(MGCM_RT_ECUDA);
    }
    Slot &sl = g->slot;
    g->total = total;
    g->max_nl = max_nl;
    // the parts' scratch together within a quarter of the budget, which the
    // handle's own calls can use beside the graph's
    const size_t per_col = pipe_bytes_per_col(max_nl);
    const size_t share = h->budget / (4 * g->nparts);
    const int most = *std::max_element(g->ncols, g->ncols + g->nparts);
    g->max_chunk = (int)std::max<size_t>(1, std::min<size_t>(most, share / per_col));

    // autotune: coordinate descent over chunk, solver CTAs per SM and reduce
    // rows per chunk, each shape timed (best of two) on the first columns
    Tune best{};
    // tuning sample: the first 131,072 columns for the pipeline; the whole
    // batch (up to 1M columns) for the fused kernel, whose best shape depends
    // on the mix of layer counts, which the first members need not represent
    const int sample = h->fused ? std::min(g->ncols[0], 1 << 20) : std::min(g->ncols[0], 131072);
    float t_def = 0.f;
    int rc = time_shape(g, best, sample, t_def);
    if (rc) return fail(rc);
    rc = time_shape(g, best, sample, t_def);   // the first pass also sized the scratch
    if (rc) return fail(rc);
    float t_best = t_def;
    int ncand = 1;
    if (autotune && h->fused) {   // fused kernel: columns per tile, threads per CTA, CTAs per SM
        for (int q = 0; q < FUSED_NS; ++q) {
            if (q == FUSED_DEFAULT) continue;
            Tune t = best;
            t.fused = q;
            float ms = 0.f;
            if ((rc = time_shape(g, t, sample, ms))) return fail(rc);
            ++ncand;
            if (ms < t_best) {
                t_best = ms;
                best = t;
            }
        }
    } else if (autotune) {
        auto consider = [&](Tune t) -> int {
            float ms = 0.f;
            const int r = time_shape(g, t, sample, ms);
            if (r) return r;
            ++ncand;
            if (ms < t_best) {
                t_best = ms;
                best = t;
            }
            return MGCM_RT_OK;
        };
        for (int c : {16384, 32768, 65536}) {
            if (c >= sample || c > g->max_chunk) continue;
            Tune t = best;
            t.chunk = c;
            if ((rc = consider(t))) return fail(rc);
        }
        for (int k : {2, 3, 4, 5, 6}) {
            Tune t = best;
            t.solve_ctas = k;
            if ((rc = consider(t))) return fail(rc);
        }
        for (int r : {1, 2, 4, 8}) {
            if (reduce_smem_bytes(max_nl, r) > SMEM_CAP) continue;
            if (r == reduce_rows_per_chunk(max_nl)) continue;
            Tune t = best;
            t.rb = r;
            if ((rc = consider(t))) return fail(rc);
        }
    }
    // one eager pass over every part's columns with the chosen shape sizes
    // the scratch for the capture (nothing may allocate while capturing)
    for (int p = 0; p < g->nparts; ++p) {
        Slot &ps = g->part(p);
        ps.tune = best;
        int nk0 = 0;
        if ((rc = launch_body(h, ps, ps.stream, g->ncols[p], g->part_nl[p], nk0, g->max_chunk))) return fail(rc);
        if (cudaStreamSynchronize(ps.stream) != cudaSuccess) return fail(MGCM_RT_ECUDA);
    }

    int nk = 0;
    cudaStream_t st = sl.stream;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return fail(MGCM_RT_ECUDA);
    int crc = MGCM_RT_OK;
    if (cudaMemsetAsync(sl.d_status, 0, 256, st) != cudaSuccess) crc = MGCM_RT_ECUDA;
    if (!crc && g->nparts > 1 && cudaEventRecord(g->fork, st) != cudaSuccess) crc = MGCM_RT_ECUDA;
    for (int p = 1; p < g->nparts && !crc; ++p) {
        Slot &ps = g->part(p);
        if (cudaStreamWaitEvent(ps.stream, g->fork, 0) != cudaSuccess ||
            cudaMemsetAsync(ps.d_status, 0, 256, ps.stream) != cudaSuccess)
            crc = MGCM_RT_ECUDA;
    }
    for (int p = 0; p < g->nparts && !crc; ++p) {
        Slot &ps = g->part(p);
        cudaStream_t pst = p == 0 ? st : ps.stream;
        crc = launch_body(h, ps, pst, g->ncols[p], g->part_nl[p], nk, g->max_chunk);
        if (!crc) crc = post_status(ps, pst);
    }
    for (int p = 1; p < g->nparts && !crc; ++p) {
        Slot &ps = g->part(p);
        if (cudaEventRecord(ps.done, ps.stream) != cudaSuccess || cudaStreamWaitEvent(st, ps.done, 0) != cudaSuccess)
            crc = MGCM_RT_ECUDA;
    }
    cudaGraph_t gr = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &gr);
    if (crc || ce != cudaSuccess || !gr) {
        if (gr) cudaGraphDestroy(gr);
        return fail(crc ? crc : MGCM_RT_ECUDA);
    }
    g->graph = gr;
    if (cudaGraphInstantiate(&g->exec, gr, 0) != cudaSuccess) return fail(MGCM_RT_ECUDA);
    mgcm_rt_tune &inf = g->info;
    inf.chunk_cols = best.chunk > 0 ? std::min(best.chunk, g->max_chunk) : std::min(total, g->max_chunk);
    inf.solve_ctas_per_sm = best.solve_ctas;
    inf.reduce_rows = best.rb > 0 ? best.rb : reduce_rows_per_chunk(max_nl);
    inf.candidates = ncand;
    inf.tuning_cols = sample;
    inf.default_ms = t_def;
    inf.best_ms = t_best;
    inf.kernels = nk;
    inf.columns = total;
    if (h->fused) {
        const FusedShape fs = FUSED_SHAPES[best.fused >= 0 ? best.fused : FUSED_DEFAULT];
        inf.chunk_cols = fs.tc;
        inf.solve_ctas_per_sm = fs.minb;
        inf.reduce_rows = 0;
        inf.threads_per_cta = fs.threads;
    }
    *graph = g;
    return MGCM_RT_OK;
}

int mgcm_rt_graph_launch(mgcm_rt_graph *g, void *stream) {
    NvtxRange nvtx_range("mgcm_rt_graph_launch");
    if (!g || !g->exec) return MGCM_RT_EINVAL;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g->slot.stream;
    CK(cudaGraphLaunch(g->exec, st));
    return MGCM_RT_OK;
}

int mgcm_rt_graph_status(mgcm_rt_graph *g) {
    if (!g) return MGCM_RT_EINVAL;
    uint32_t st = 0;
    for (int p = 0; p < g->nparts; ++p) st |= *g->part(p).h_status;
    return status_to_code(st);
}

int mgcm_rt_graph_info(const mgcm_rt_graph *g, mgcm_rt_tune *info) {
    if (!g || !info) return MGCM_RT_EINVAL;
    *info = g->info;
    return MGCM_RT_OK;
}

void mgcm_rt_graph_destroy(mgcm_rt_graph *g) {
    if (!g) return;
    std::lock_guard<std::mutex> lk(g->h->mu);
    cudaSetDevice(g->h->device);
    graph_free(g);
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
    NvtxRange nvtx_range("mgcm_rt_run_noalloc");
    if (!h || !in || !out) return MGCM_RT_EINVAL;
    if (!in->device_ptrs) return MGCM_RT_EINVAL;   // host buffers would need staging memory
    std::lock_guard<std::mutex> lk(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess) return MGCM_RT_ECUDA;
    int rc = check_args(h, in, out);
    if (rc) return rc;
    if (in->ncol == 0) return MGCM_RT_OK;
    rc = finish_pending(h);
    if (rc) return rc;
    Slot &sl = *h->slots[0];
    cudaStream_t stream = sync_stream(h);
    if (!h->user_stream) {
        if (const int rc2 = after_legacy_stream(sl, stream)) return rc2;
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
    int nb = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rt_fp64_kernel, BLOCK, smem) != cudaSuccess)
        nb = 1;
    const size_t want = (size_t)h->num_sms * (size_t)std::max(nb, 1);
    const int grid = (int)std::min({(size_t)z.ncol, want, nslab});
    // descriptor: header + one segment, staged through the handle's pinned buffer
    SegTable &tab = *sl.h_segs;
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
    CK(cudaMemcpyAsync(d_tab, sl.h_segs, offsetof(SegTable, seg) + sizeof(SegDev),
                       cudaMemcpyHostToDevice, stream));
    CK(cudaMemsetAsync(d_status, 0, sizeof(uint32_t), stream));
    CK(cudaMemsetAsync(d_nsys, 0, sizeof(unsigned long long), stream));
    if (h->cfg.validate) {   // the same input checks as the other entry points
        const int vb = std::min((int)((z.ncol + 255) / 256), h->num_sms * 8);
        validate_kernel<<<std::max(vb, 1), 256, 0, stream>>>(d_tab, d_status);
    }
    CK(cudaEventRecord(sl.ev0, stream));
    rt_fp64_kernel<<<grid, BLOCK, smem, stream>>>(d_tab, h->d_kv, h->d_ki, h->d_planck, h->K,
                                                     max_nl, d_status, d_nsys, d_red);
    CK(cudaGetLastError());
    CK(cudaEventRecord(sl.ev1, stream));
    CK(cudaStreamSynchronize(stream));
    uint32_t st = 0;
    unsigned long long ns = 0;
    CK(cudaMemcpy(&st, d_status, sizeof(st), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&ns, d_nsys, sizeof(ns), cudaMemcpyDeviceToHost));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, sl.ev0, sl.ev1);
    h->stats.gpu_ms = ms;
    h->stats.columns = (long long)z.ncol;
    h->stats.systems = (long long)ns;
    h->stats.status = (int)st;
    h->stats.kernels = h->cfg.validate ? 2 : 1;
    return status_to_code(st);
}
