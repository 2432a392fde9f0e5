/*
 * mgcm_rt.h -- C ABI of the B200 column radiative transfer for the NASA Ames
 * Legacy Mars GCM (v24).
 *
 * One batched call replaces the per-column radiation calls the reference
 * makes inside the physics column loop of COMP3 (code/comp3.f:411-1044):
 *
 *   code/comp3.f:658    CALL OPTCV   (visible opacities; code/optcv.f90:1)
 *   code/comp3.f:664    CUMTAUV store
 *   code/comp3.f:672    CALL SFLUXV  (visible two-stream; code/sfluxv.f90:1,
 *                                    code/gfluxv.f90:1, code/getdetau.f90:1,
 *                                    code/dsolver.f90:1, code/dtridgl.f90:1)
 *   code/comp3.f:677    SUNTOT divergences
 *   code/comp3.f:724    CALL OPTCI   (IR opacities; code/optci.f90:1)
 *   code/comp3.f:731    CALL SFLUXI  (IR two-stream; code/sfluxi.f90:1,
 *                                    code/gfluxi.f90:1)
 *   code/comp3.f:735    IRTOTAL divergences
 *   code/comp3.f:698-747 surface / top-of-atmosphere diagnostics
 *   code/comp3.f:765-771 QRAD heating rates (non-LTE factor included)
 *
 * Units are the reference's: pressures in mbar, temperatures in K, fluxes in
 * W/m^2, QRAD in K/s of potential temperature (QRAD*OM is dT/dt).
 *
 * Layout: every per-column array has the column index slowest, so a Fortran
 * host passes A(level, col) / A(level, band, col) / A(nw, ng, col) directly.
 *   LEV  = 2L+3 (L_LEVELS)        level arrays     [ncol][LEV]
 *   LEV1 = 2L+4 (L_LEVELS+1)      level+1 arrays   [ncol][LEV1]
 *   band arrays                   [ncol][NB][LEV1] (NB = 7 visible, 5 IR)
 *   NLAY = L+1 (L_NLAYRAD)        layer outputs    [ncol][NLAY]
 *   DETAU, CUMTAUV                [ncol][17][7]    (Fortran A(nw,ng,col))
 *
 * Device pointers: a call is ordered after all work already queued on the
 * legacy default stream (cudaMemcpy, a framework's default-stream kernels),
 * or, after mgcm_rt_set_stream, on the caller's stream; device buffers
 * written on any other stream must be complete before the call.
 *
 * Errors are negative return codes (never abort/exit; the reference STOPs,
 * code/gfluxi.f90:65).  A handle is thread-safe: calls on one handle are
 * serialised by an internal lock and run on the handle's own CUDA stream.
 */
#ifndef MGCM_RT_H
#define MGCM_RT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGCM_RT_NSPECTV 7    /* L_NSPECTV, code/modules.f90:225 */
#define MGCM_RT_NSPECTI 5    /* L_NSPECTI, code/modules.f90:224 */
#define MGCM_RT_NGAUSS 17    /* L_NGAUSS,  code/modules.f90:226 */
#define MGCM_RT_MAX_LAYERS 99 /* NLL <= NLP = 101, code/gfluxi.f90:43,65 */

/* precision modes */
#define MGCM_RT_FP64 0  /* plain FP64, operation order of the reference */
#define MGCM_RT_MIXED 1 /* FP32 opacities/optics, FP64 solves and flux sums */

/* status codes */
#define MGCM_RT_OK 0
#define MGCM_RT_EINVAL -1     /* null pointer, ncol < 0, bad config */
#define MGCM_RT_ENONFINITE -2 /* NaN/Inf or non-positive pressure in an input */
#define MGCM_RT_ETEMP -3      /* a temperature outside the Planck table [50,900) K */
#define MGCM_RT_ELAYERS -4    /* L outside 1..MGCM_RT_MAX_LAYERS or above max_layers */
#define MGCM_RT_ENOMEM -5     /* device memory or HBM budget exhausted */
#define MGCM_RT_EIO -6        /* data file missing or malformed */
#define MGCM_RT_ECUDA -7      /* CUDA runtime error */
#define MGCM_RT_ETIMEOUT -8   /* wait() ran out of time */
#define MGCM_RT_EBUSY -9      /* request queue full */
#define MGCM_RT_ENOTFOUND -10 /* unknown or already collected ticket */

typedef struct mgcm_rt_handle mgcm_rt_handle;

typedef struct {
    int max_layers;       /* largest L any batch will use (1..99) */
    int precision;        /* MGCM_RT_FP64 or MGCM_RT_MIXED */
    int device;           /* CUDA device ordinal */
    int validate;         /* nonzero: check inputs (finite, T range) before each launch */
    size_t hbm_budget;    /* device bytes for batch staging; 0 = 3/4 of free memory */
    int solver;           /* MGCM_RT_SOLVER_AUTO / _THREAD: one thread per (band, Gauss)
                             system; MGCM_RT_SOLVER_QUAD: four lanes per system with the
                             per-layer values in registers (L <= 51; same results) */
    int max_queued_jobs;  /* serving: jobs (of <= 16,384 columns) accepted and not yet
                             finished, at most; a submit beyond it returns MGCM_RT_EBUSY.
                             0 = 100,000 */
} mgcm_rt_config;

#define MGCM_RT_SOLVER_AUTO 0
#define MGCM_RT_SOLVER_THREAD 1
#define MGCM_RT_SOLVER_QUAD 2
#define MGCM_RT_SOLVER_ONCHIP 3   /* one thread per system, per-system arrays on chip */
#define MGCM_RT_SOLVER_TMEM 4     /* the same with tensor memory in front of shared memory */
#define MGCM_RT_SOLVER_FUSED 5    /* one persistent kernel per call: stage, screen, solve and
                                     reduce per tile of columns (thread-per-system solves) */

/* One batch of columns on one vertical grid. */
typedef struct {
    int ncol;             /* number of columns (>= 0) */
    int nlayers;          /* L: GCM layers of this grid */
    int device_ptrs;      /* nonzero: every array below is a device pointer */
    double ptrop;         /* PTROP, mbar */
    const double *sigma;  /* [LEV] SIGMA(K) of the grid (SIGMA(1)=SIGMA(2)=0) */
    const double *sol;    /* [7] SOLARF/RSDIST, W/m^2 (code/comp3.f:300-304) */
    const double *plev, *tlev, *pmid, *tmid, *qh2o;   /* [ncol][LEV]  (FILLPT, QH2O) */
    const double *tauref, *qextrefdst;                 /* [ncol][LEV1] dust */
    const double *qxvdst, *qsvdst, *gvdst;             /* [ncol][7][LEV1] */
    const double *qxidst, *qsidst, *gidst;             /* [ncol][5][LEV1] */
    const double *taurefcld, *qextrefcld;              /* [ncol][LEV1]; NULL = CLOUDON off */
    const double *qxvcld, *qsvcld, *gvcld;             /* [ncol][7][LEV1] (with cloud) */
    const double *qxicld, *qsicld, *gicld;             /* [ncol][5][LEV1] (with cloud) */
    const double *acosz;  /* [ncol] cos(solar zenith); day when >= 1.0e-5 (REAL*4) */
    const double *als;    /* [ncol] visible surface albedo */
    const double *albi;   /* [ncol] IR surface albedo = 1 - emissivity */
    const double *pcol;   /* [ncol] P(J,I) = surface pressure - PTROP, mbar */
    double *detau;        /* [ncol][17][7] in/out: delta-Eddington surface tau; kept for night */
    double *cumtauv;      /* [ncol][17][7] in/out: TAUCUMV(L_LEVELS); kept for night */
} mgcm_rt_batch_in;

typedef struct {
    double *fmnetv, *fluxupv, *fluxdnv;  /* [ncol][NLAY] visible net/up/down midpoint fluxes */
    double *fmneti, *fluxupi, *fluxdni;  /* [ncol][NLAY] IR */
    double *suntot, *irtotal;            /* [ncol][NLAY] SUNTOT(2l+1), IRTOTAL(2l+1) */
    double *qrad;                        /* [ncol][NLAY] QRAD(2l), K/s */
    double *nfluxtopv, *nfluxtopi;       /* [ncol] */
    double *diffvt;                      /* [ncol] diffuse visible down at the surface */
    double *dnvflux, *dndiffv;           /* [ncol] DNVFLUX = FLUXDNV(NLAY), DNDIFFV = DIFFVT */
    double *dnirflux, *fluxsurf;         /* [ncol] FLUXDNI(NLAY), (1-ALS)*FLUXDNV(NLAY) */
} mgcm_rt_batch_out;

/* Per-call statistics of the last completed run on a handle. */
typedef struct {
    double gpu_ms;          /* device time of the radiation kernels */
    double total_ms;        /* host wall time of the call */
    long long columns;      /* columns processed */
    long long systems;      /* two-stream systems solved (after TLIMIT and night skips) */
    int kernels;            /* kernels launched */
    int status;             /* device status word (0 = clean) */
    long long hbm_used;     /* device bytes the handle's staging arenas hold now */
    long long hbm_budget;   /* the handle's HBM budget for them */
} mgcm_rt_stats;

/* Reads CO2H2O_{V,IR}_12_95_INTEL from data_dir (code/laginterp.f90:59-69),
 * builds the k tables (code/setrad.f90, code/laginterp.f90), the Planck table
 * (code/setspi.f90:91-105) and the band constants (code/setspv.f90), and
 * uploads them.  Replaces RADSETUP (code/radsetup.f90:26-43).
 * Returns NULL and sets *status on failure. */
mgcm_rt_handle *mgcm_rt_create(const mgcm_rt_config *cfg, const char *data_dir, int *status);

/* Synchronous batched radiation (the block code/comp3.f:637-771 for every
 * column).  Host or device pointers per in->device_ptrs; outputs follow the
 * same kind.  Night columns leave DETAU and CUMTAUV unchanged and report
 * zero visible fluxes. */
int mgcm_rt_run(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out);

/* Asynchronous form for device pointers: enqueue the batch on the handle's
 * stream and return; mgcm_rt_sync() waits and returns the batch status.
 * Lets a C/C++/Python host overlap its own work or capture a CUDA graph. */
int mgcm_rt_enqueue(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out);
int mgcm_rt_sync(mgcm_rt_handle *h);

/* Run the handle's work on a caller-owned cudaStream_t (NULL restores the
 * handle's own stream). */
int mgcm_rt_set_stream(mgcm_rt_handle *h, void *cuda_stream);

/* Uneven batch: nbatch grids of different L and sizes in one persistent
 * launch.  Every batch must use the same pointer kind. */
int mgcm_rt_run_multi(mgcm_rt_handle *h, int nbatch, const mgcm_rt_batch_in *in,
                      mgcm_rt_batch_out *out);

/* Serving: queue a batch (pointers must stay valid until collected), get a
 * ticket.  Requests are split into jobs of <= 16,384 columns and admitted
 * onto up to four serving slots as slots and HBM budget free up; a job that
 * does not fit the budget while others run waits for them (a job that does
 * not fit an idle device fails with MGCM_RT_ENOMEM).  MGCM_RT_EBUSY when the
 * request would take the accepted-and-unfinished jobs above
 * mgcm_rt_config.max_queued_jobs. */
int mgcm_rt_submit(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out,
                   long long *ticket);
/* 1 = finished (result available), 0 = pending, < 0 = error for the ticket. */
int mgcm_rt_poll(mgcm_rt_handle *h, long long ticket);
/* Blocks until the ticket finishes or timeout_s passes (<0: no limit);
 * returns the request's status and releases the ticket. */
int mgcm_rt_wait(mgcm_rt_handle *h, long long ticket, double timeout_s);

/* Timeline of a request not yet released by mgcm_rt_wait (no counterpart in
 * the reference, which has no requests).  Host times are ms after the
 * handle's creation; device times are ms after an event the serving worker
 * records when it starts, taken from the CUDA events that bracket the
 * kernels of each of the request's jobs (earliest start, latest end), so
 * the device intervals of two requests show whether their kernels overlapped.
 * -1 where not yet known. */
typedef struct {
    int done;               /* 1 when every job has finished */
    int status;             /* request status so far (0 or a negative code) */
    int jobs;               /* jobs of <= 16,384 columns the request was split into */
    int deferred;           /* admissions put back because the HBM budget was full */
    double submit_ms, done_ms;                 /* host */
    double device_begin_ms, device_end_ms;     /* device */
} mgcm_rt_request_info;
int mgcm_rt_get_request_info(mgcm_rt_handle *h, long long ticket, mgcm_rt_request_info *info);

/* ---- tracer inputs: aerosol optics on the device -----------------------
 * The per-level dust and water-ice optical properties that COMP3 builds on
 * the host (code/comp3.f:592-630: OPT_DST from the dust tracers, or the
 * prescribed INI_OPTDST band properties with TAUREF from FILLTAUCUM; OPT_CLD
 * from the ice tracers) are computed on the device from the tracer mixing
 * ratios, then the radiation runs as in mgcm_rt_run.  The host passes about
 * 5 KB per column instead of ~35 KB (L = 24).  No reference counterpart as
 * one call; the outputs equal mgcm_rt_run on the host-computed arrays. */
typedef struct {
    int ncol, nlayers, device_ptrs;
    int active_dust;     /* 1: OPT_DST from dust_mass, dust_number; 0: prescribed dust, tauref given */
    int cloudon;         /* 1: OPT_CLD from ice_mass, ice_core_mass, ice_number; 0: no cloud */
    double ptrop;
    const double *sigma, *sol;
    const double *plev, *tlev, *pmid, *tmid, *qh2o;       /* [ncol][2L+3] */
    const double *tauref;                                 /* [ncol][2L+4] (active_dust = 0) */
    const double *dust_mass, *dust_number;                /* [ncol][L] QTRACE(J,I,L,iMa_dt/iNb_dt) */
    const double *ice_mass, *ice_core_mass, *ice_number;  /* [ncol][L] iMa_cld, iMa_cor, iNb_cld */
    const double *acosz, *als, *albi, *pcol;              /* [ncol] */
    double *detau, *cumtauv;                              /* [ncol][17][7] in/out */
} mgcm_rt_batch_tracers;
int mgcm_rt_run_tracers(mgcm_rt_handle *h, const mgcm_rt_batch_tracers *in, mgcm_rt_batch_out *out);

/* ---- GCM state inputs: column prep on the device ------------------------
 * COMP3's assembly of the radiation inputs runs on the device as well: the
 * level pressures PL (code/potemp1.f:95-106) and FILLPT's PLEV, TLEV, PMID,
 * TMID (code/fillpt.f90:30-72), QH2O (code/comp3.f:576-589) and, for
 * prescribed dust, TAUREF from the Conrath profile of DUSTPROFILE sampled by
 * FILLTAUCUM (code/dustprofile.f:32-114, code/filltaucum.f:39-55).  Then the
 * aerosol optics and the radiation run as in mgcm_rt_run_tracers.  The host
 * passes the model state itself: about 1.6 KB per column at L = 24 with
 * dust and ice tracers.  COLDAIR stays on the host (it changes the model
 * state); t, tstrat and gt are its results.  The prepared level arrays can
 * be returned through the optional pointers.  No reference counterpart as
 * one call; the outputs equal mgcm_rt_run_tracers on the same prepared
 * arrays. */
typedef struct {
    int ncol, nlayers, device_ptrs;
    int active_dust;     /* 1: OPT_DST from the dust tracers; 0: prescribed (Conrath) dust */
    int cloudon;         /* 1: OPT_CLD from the ice tracers; 0: no cloud */
    int active_water;    /* 1: QH2O = mwratio * vapour; 0: QH2O = 1.0E-7 (REAL*4) */
    double ptrop;        /* PTROP (mbar) */
    double psf;          /* PSF (mbar): sets the PRDST grid of the dust profile (active_dust = 0) */
    double rptau;        /* RPTAU (mbar): pressure tautot refers to (active_dust = 0) */
    double mwratio;      /* MWRATIO = MWCO2/MWH2O, code/input.f:180 (active_water = 1) */
    const double *sigma, *sol;                    /* [2L+3] SIGMA, [7] SOLARF/RSDIST */
    const double *pcol;                           /* [ncol] P(J,I) (mbar) */
    const double *t;                              /* [ncol][L] TL(2l+2) = T(J,I,l) after COLDAIR */
    const double *tstrat, *gt;                    /* [ncol] TSTRAT(J,I), GT(J,I) after COLDAIR */
    const double *vapour;                         /* [ncol][L] QTRACE(J,I,L,iMa_vap) (active_water = 1) */
    const double *tautot, *conr;                  /* [ncol] TAUTOTJI(J,I), Conrath nu (active_dust = 0) */
    const double *dust_mass, *dust_number;        /* [ncol][L] (active_dust = 1) */
    const double *ice_mass, *ice_core_mass, *ice_number; /* [ncol][L] (cloudon = 1) */
    const double *acosz, *als, *albi;             /* [ncol] */
    double *detau, *cumtauv;                      /* [ncol][17][7] in/out */
    double *plev, *tlev, *pmid, *tmid, *qh2o;     /* [ncol][2L+3] optional out (NULL: not returned) */
    double *tauref;                               /* [ncol][2L+4] optional out (active_dust = 0) */
} mgcm_rt_batch_state;
int mgcm_rt_run_state(mgcm_rt_handle *h, const mgcm_rt_batch_state *in, mgcm_rt_batch_out *out);

/* ---- captured uneven batches ------------------------------------------
 * A fixed set of device-resident batches (e.g. the members of an ensemble,
 * grids of different layer counts) captured once as a CUDA graph and
 * replayed every radiation step.  No reference counterpart: the reference
 * runs one grid per process.  Creation (optionally) autotunes the launch
 * shape on a sample of the columns, sizes the scratch, then captures;
 * launches of one graph must be ordered on one stream, and the batch
 * arrays it was created with must stay allocated. */
typedef struct mgcm_rt_graph mgcm_rt_graph;
typedef struct mgcm_rt_tune {
    int chunk_cols;        /* columns per pipeline pass (fused form: columns per tile) */
    int solve_ctas_per_sm; /* solver CTAs per SM (0 = as many as fit; fused form: CTAs per SM
                              the register budget allows) */
    int reduce_rows;       /* kept systems whose loads a reduce lane issues before summing */
    int candidates;        /* launch shapes timed by the autotuner */
    int tuning_cols;       /* columns of the tuning sample */
    double default_ms;     /* built-in shape on the sample */
    double best_ms;        /* chosen shape on the sample */
    int kernels;           /* kernel launches in the captured graph */
    int columns;           /* columns of all batches */
    int threads_per_cta;   /* fused form: threads per CTA (0 for the pipeline) */
} mgcm_rt_tune;
int mgcm_rt_graph_create(mgcm_rt_handle *h, int nbatch, const mgcm_rt_batch_in *in,
                         mgcm_rt_batch_out *out, int autotune, mgcm_rt_graph **graph);
/* Enqueues one replay on `stream` (a cudaStream_t; NULL: the graph's own). */
int mgcm_rt_graph_launch(mgcm_rt_graph *g, void *stream);
/* Status of the last replay; call after the replay's stream has completed. */
int mgcm_rt_graph_status(mgcm_rt_graph *g);
int mgcm_rt_graph_info(const mgcm_rt_graph *g, mgcm_rt_tune *info);
/* Destroy every graph before its handle. */
void mgcm_rt_graph_destroy(mgcm_rt_graph *g);

/* Partial radiation between full calls: DNVFLUX = DNDIFFV + direct beam from
 * DETAU (code/dsolflux.f:28-45, code/comp3.f:320-351). */
int mgcm_rt_dsolflux(mgcm_rt_handle *h, int ncol, int device_ptrs, const double *sol,
                     const double *acosz, const double *detau, const double *dndiffv,
                     double *dnvflux);

/* Debug export of the integer bins the device uses (device pointers only:
 * in->device_ptrs set, outputs device buffers [ncol][LEV], lcoef
 * [ncol][LEV][4]).  Runs the pipeline's staging kernel on the batch and
 * reads back, per level K = 2..LEV, the bins of TPINDEX (MT, MP, NH2O) with
 * WRATIO and LCOEF(1..4) (code/tpindex.f90:72-134, called per level at
 * code/optcv.f90:107 and code/optci.f90:117), and per level K = 1..LEV the
 * Planck table index INT(TLEV*10-499) (code/sfluxi.f90:54-55,
 * code/gfluxi.f90:73-74,86-87).  Level 1 has no TPINDEX call: zeros.
 * Allocates a temporary staging buffer. */
int mgcm_rt_debug_bins(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, int *mt, int *mp, int *nh2o,
                       int *nplanck, double *wratio, double *lcoef);

int mgcm_rt_get_stats(mgcm_rt_handle *h, mgcm_rt_stats *st);

/* Host copies of the set-up tables, laid out as the reference modules hold
 * them: co2v (7,51,10,7,17) and co2i (7,51,10,5,17) Fortran order, planckir
 * (5,8501), pfgasref (51).  Any pointer may be NULL.  No device needed. */
int mgcm_rt_tables_host(const char *data_dir, double *co2v, double *co2i, double *planckir,
                        double *pfgasref);

/* No-allocation run (no counterpart in the reference; the reference has no
 * device memory at all).  For callers that must not allocate device memory
 * once they are running: a host whose device memory is owned by another
 * allocator (a framework's caching pool), a time-stepping loop that forbids
 * allocation after start-up, a process under a hard device-memory quota.
 * Tables come from the handle (allocated once by mgcm_rt_create); inputs and
 * outputs are the caller's device buffers (in->device_ptrs must be set).  The
 * call itself allocates nothing: its scratch -- the batch descriptor, the
 * status word and the per-CTA flux staging of the FP64 kernel -- lives in one
 * file-scope static device array of MGCM_RT_NOALLOC_SCRATCH_BYTES.  The
 * array's device address is resolved by mgcm_rt_create on the handle's
 * device (once per device), so the array is committed on every device that
 * holds a handle, until the process exits.  mgcm_rt_create also reserves the
 * local memory the kernels need (the per-thread stack limit), so the call
 * itself never loads code or grows a device memory pool.  Always the FP64 kernel: the handle's
 * precision setting is ignored here.  The handle's validate setting is
 * honoured (the same NaN/Inf and temperature checks as mgcm_rt_run).  The
 * grid is capped by the per-CTA staging slabs that fit the array (about 200
 * at L = 24, 100 at L = 48), so the call is slower than mgcm_rt_run.  Runs on
 * the handle's stream and waits for it.  All calls share the one array and
 * each overwrites it, so calls that overlap on the GPU (different threads or
 * handles on the same device) race; serialise them.  Returns MGCM_RT_EINVAL
 * for host pointers and MGCM_RT_ENOMEM if one CTA's staging would not fit. */
#define MGCM_RT_NOALLOC_SCRATCH_BYTES (16u << 20)
int mgcm_rt_run_noalloc(mgcm_rt_handle *h, const mgcm_rt_batch_in *in, mgcm_rt_batch_out *out);

void mgcm_rt_destroy(mgcm_rt_handle *h);
const char *mgcm_rt_strerror(int status);
const char *mgcm_rt_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MGCM_RT_H */
