/*
 * mgcm_rt_oracle.h -- CPU oracle for the column radiative transfer of the
 * NASA Ames Legacy Mars GCM (v24).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against; it is never linked into the product library.  Only tests/,
 * __graft_entry__.smoke() and bench.py (its cpu_baseline leg and the
 * reference arm) load it.
 *
 * It restates, line by line and in FP64, the reference Fortran of the hot
 * path (code/tpindex.f90, optcv.f90, optci.f90, getdetau.f90, sfluxv.f90,
 * gfluxv.f90, sfluxi.f90, gfluxi.f90, dsolver.f90, dtridgl.f90, dsolflux.f,
 * the heating block of comp3.f:664-782) and its set-up (laginterp.f90,
 * lagrange.f90, setspv.f90, setspi.f90, setrad.f90), with the number of GCM
 * layers L a run-time value instead of the compile-time L_LAYERS.
 *
 * Array layout of a batch: the column index is slowest everywhere.
 *   level arrays      [ncol][2L+3]         PLEV TLEV PMID TMID QH2O
 *   level+1 arrays    [ncol][2L+4]         TAUREF QEXTREFDST TAUREFCLD QEXTREFCLD
 *   band arrays       [ncol][NB][2L+4]     QXVDST ... (Fortran A(level,band))
 *   layer outputs     [ncol][L+1]
 *   DETAU / CUMTAUV   [ncol][17][7]        (Fortran A(nw,ng), nw fastest)
 */
#ifndef MGCM_RT_ORACLE_H
#define MGCM_RT_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NSPECTV 7
#define ORC_NSPECTI 5
#define ORC_NGAUSS 17
#define ORC_NTREF 7
#define ORC_NPREF 11
#define ORC_PINT 51
#define ORC_REFH2O 10
#define ORC_NPLANCK 8501
#define ORC_MAXL 99

typedef struct {
    /* CO2V(nt,np,nh,nw,ng) in Fortran order: index nt + 7*(np + 51*(nh + 10*(nw + NB*ng))) */
    double co2v[ORC_NTREF * ORC_PINT * ORC_REFH2O * ORC_NSPECTV * ORC_NGAUSS];
    double co2i[ORC_NTREF * ORC_PINT * ORC_REFH2O * ORC_NSPECTI * ORC_NGAUSS];
    double fzerov[ORC_NSPECTV];
    double fzeroi[ORC_NSPECTI];
    double pfgasref[ORC_PINT];
    double tgasref[ORC_NTREF];
    double pgasref[ORC_NPREF];
    /* planckir(nw, it), it = 1..8501  ->  planckir[(it-1)*5 + nw-1] */
    double planckir[ORC_NSPECTI * ORC_NPLANCK];
    double wnov[ORC_NSPECTV], dwnv[ORC_NSPECTV], wavev[ORC_NSPECTV];
    double solarf[ORC_NSPECTV], tauray[ORC_NSPECTV];
    double wnoi[ORC_NSPECTI], dwni[ORC_NSPECTI], wavei[ORC_NSPECTI];
    double qextv[ORC_NSPECTV], qscatv[ORC_NSPECTV], gv[ORC_NSPECTV];
    double qexti[ORC_NSPECTI], qscati[ORC_NSPECTI], gi[ORC_NSPECTI];
    double gweight[ORC_NGAUSS];
    double wrefh2o[ORC_REFH2O];
} orc_tables;

/* Raw k-coefficient records as stored in the reference data files
 * (CO2H2O_V_12_95_INTEL, CO2H2O_IR_12_95_INTEL), before laginterp. */
int orc_read_ktables(const char *vis_path, const char *ir_path,
                     double *co2v8, double *fzerov, double *co2i8, double *fzeroi);

/* Build every table from raw k records (setspv, setspi, setrad/laginterp). */
void orc_build_tables(orc_tables *t, const double *co2v8, const double *fzerov,
                      const double *co2i8, const double *fzeroi);

/* Convenience: read + build.  Returns 0 or a negative error. */
int orc_tables_load(orc_tables *t, const char *vis_path, const char *ir_path);

size_t orc_tables_size(void);

/* tpindex.f90 restated: bins (1-based, as in Fortran) and weights. */
void orc_tpindex(const orc_tables *t, double pw, double tw, double qh2o,
                 double lcoef[4], int *mt, int *mp, int *nh2o, double *wratio);

/* Planck table index INT(T*10-499) (code/sfluxi.f90:54-55). */
int orc_planck_index(double t);

typedef struct {
    int ncol, L;
    /* inputs */
    const double *plev, *tlev, *pmid, *tmid, *qh2o;
    const double *tauref, *qextrefdst, *taurefcld, *qextrefcld;
    const double *qxvdst, *qsvdst, *gvdst, *qxidst, *qsidst, *gidst;
    const double *qxvcld, *qsvcld, *gvcld, *qxicld, *qsicld, *gicld; /* may be NULL */
    const double *acosz, *als, *albi, *pcol;
    const double *sol;   /* [7] */
    const double *sigma; /* [2L+3] */
    double ptrop;
    /* in/out */
    double *detau, *cumtauv;
    /* outputs */
    double *fmnetv, *fluxupv, *fluxdnv, *fmneti, *fluxupi, *fluxdni;
    double *suntot, *irtotal, *qrad;
    double *nfluxtopv, *nfluxtopi, *diffvt;
    double *dnvflux, *dndiffv, *dnirflux, *fluxsurf;
} orc_batch;

/* Full radiation block for every column of the batch; nthreads<=0 uses
 * all online cores (pthreads).  Returns 0 or a negative error. */
int orc_run_batch(const orc_tables *t, const orc_batch *b, int nthreads);

/* Debug access to the optical depths of one column (optcv/optci outputs).
 * dtauv [7][17][L+1], taucumv [7][17][2L+3], taugsurf [7][16] etc. */
void orc_optics_column(const orc_tables *t, const orc_batch *b, int col,
                       double *dtauv, double *wbarv, double *cosbv, double *taucumv,
                       double *taugsurfv, double *dtaui, double *wbari, double *cosbi,
                       double *taucumi, double *taugsurfi);

/* dsolflux.f: direct-beam surface flux from DETAU, per column. */
/* ---- aerosol optics (code/opt_dst.f, code/opt_cld.f, code/ini_optdst.f,
 * code/initcld.f:141-190, code/setrad.f90:73-105, code/comp3.f:592-630) */
#define ORC_NBIN 20
#define ORC_NRATIO 15
typedef struct {
    double radb[ORC_NBIN + 1];
    double dst_v[3][ORC_NBIN][ORC_NSPECTV], dst_i[3][ORC_NBIN][ORC_NSPECTI];
    double cld_v[3][ORC_NRATIO][ORC_NBIN][ORC_NSPECTV], cld_i[3][ORC_NRATIO][ORC_NBIN][ORC_NSPECTI];
    float cor_ratio[ORC_NRATIO];
    double qextv[ORC_NSPECTV], qscatv[ORC_NSPECTV], gv[ORC_NSPECTV];
    double qexti[ORC_NSPECTI], qscati[ORC_NSPECTI], gi[ORC_NSPECTI];
} orc_aero;

/* Reads the dust and water-ice Mie tables of `dir` and builds the size bins. */
int orc_aero_load(orc_aero *a, const char *dir);
size_t orc_aero_size(void);

/* Tracer inputs of a batch -> the full per-level aerosol arrays of orc_batch.
 * active_dust: opt_dst from the dust mass/number mixing ratios, else the
 * prescribed band properties with TAUREF copied from tauref_in;
 * cloudon: opt_cld from the ice mass, core mass and number mixing ratios.
 * Tracers are [ncol][L] (QTRACE(J,I,L,*)); outputs as in orc_batch. */
typedef struct {
    int ncol, L, active_dust, cloudon;
    const double *plev, *tauref_in;
    const double *dust_mass, *dust_number, *ice_mass, *ice_core, *ice_number;
    double *tauref, *qextrefdst, *qxvdst, *qsvdst, *gvdst, *qxidst, *qsidst, *gidst;
    double *taurefcld, *qextrefcld, *qxvcld, *qsvcld, *gvcld, *qxicld, *qsicld, *gicld;
} orc_tracers;
void orc_aerosols(const orc_aero *a, const orc_tracers *t);
/* The same over nthreads host threads (<= 0: all). */
void orc_aerosols_mt(const orc_aero *a, const orc_tracers *t, int nthreads);

/* TPINDEX bins/weights and Planck indices of every level of a batch
 * ([ncol][LEV], lcoef [ncol][LEV][4]; level 1: zero bins). */
void orc_bins_batch(const orc_tables *t, const orc_batch *b, int *mt, int *mp, int *nh2o, int *npl,
                    double *wratio, double *lcoef);

void orc_dsolflux(const orc_tables *t, int ncol, const double *sol, const double *acosz,
                  const double *detau, double *directsol);

/* Column prep: the radiation's level inputs from the GCM state of a column.
 *   PLEV/TLEV/PMID/TMID   PL of code/potemp1.f:95-106 through FILLPT
 *                         (code/fillpt.f90:30-72); t[l] is TL(2l+2), the
 *                         layer temperature after COLDAIR
 *   QH2O                  code/comp3.f:576-589 (MWRATIO * vapour, or the
 *                         REAL*4 1.0E-7 without active water); levels 1-3
 *                         are not set by COMP3 and are 0 here
 *   TAUREF (prescribed)   the Conrath profile of code/dustprofile.f:32-114
 *                         on the PRDST grid, sampled by FILLTAUCUM
 *                         (code/filltaucum.f:39-55, JSRCHGT of
 *                         code/jsrchgt.f90)
 * Per-column inputs [ncol] or [ncol][L]; outputs as in orc_batch. */
#define ORC_NPDST 100
typedef struct {
    int ncol, L, active_water, prescribed_dust;
    double ptrop, psf, rptau, mwratio;
    const double *sigma;                    /* [2L+3] */
    const double *pcol, *tstrat, *gt;       /* [ncol] P(J,I), TSTRAT, GT */
    const double *t;                        /* [ncol][L] */
    const double *vapour;                   /* [ncol][L] (active_water) */
    const double *tautot, *conr;            /* [ncol] (prescribed_dust) */
    double *plev, *tlev, *pmid, *tmid, *qh2o; /* [ncol][2L+3] */
    double *tauref;                         /* [ncol][2L+4] (prescribed_dust) */
} orc_prep_batch;
/* PRDST(1..NPDST) of code/dustprofile.f:32-37. */
void orc_dust_grid(double psf, double ptrop, double *prdst);
/* TAUDST(J,I,1..NPDST) of one column (code/dustprofile.f:59-114). */
void orc_dust_profile(const double *prdst, double rptau, double conr, double tautot, double *taudst);
/* JSRCHGT (code/jsrchgt.f90), 1-based result. */
int orc_jsrchgt(int n, const double *sx, double target);
void orc_prep(const orc_prep_batch *b);

#ifdef __cplusplus
}
#endif
#endif
