/*
 * shygpu.h -- C ABI of the B200 implementation of SHYFEM's semi-implicit
 * time step (zeta assembly + sparse Krylov solve + vertical momentum column
 * solve + 3D scalar transport).
 *
 * Two families of entry points:
 *
 *  1. The reference's own linear-system ("simsys") interface, with gfortran's
 *     by-reference calling convention and trailing-underscore names, so that
 *     SHYFEM's `hydro_zeta`/`hydro` link against this library instead of
 *     src/shyfem/simsys_spkaux.f90.  The element data that the reference
 *     passes through module globals (`mod_zeta_system :: kn(3), hia(3,3),
 *     hik(3)`, simsys_spkaux.f90:75-83) travels through the C-visible
 *     struct `shy_zeta_system` below, which a Fortran `bind(C)` interface
 *     names directly.
 *
 *  2. Whole-phase entries that keep every basin's state resident in device
 *     memory and advance whole time steps (`shyfem_run`'s loop body,
 *     src/shyfem/shyfem_subs.f90:569-658) for one or many basins per launch.
 *
 * All arrays use the reference's Fortran column-major layouts: `(nlv,nel)`
 * is `a[ie*nlv + l]`, `(3,nel)` is `a[ie*3 + ii]`, `(0:nlv,nkn)` is
 * `a[k*(nlv+1) + l]`.  Node and element numbers are 1-based.  Every function
 * returns 0 on success and a SHY_E* code otherwise; `shygpu_last_error()`
 * gives the message.  The library has no CPU fallback: without a usable
 * CUDA device every compute entry returns SHY_ECUDA.
 */
#ifndef SHYGPU_H
#define SHYGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SHY_EVDIM 19          /* entries of ev(evdim,nel), evgeom.f90:300-318 */
#define SHY_MAX_LAYERS 32     /* layers per column held by one warp segment  */
#define SHY_MAX_TIDE 4        /* harmonic constituents per level boundary    */
#define SHY_MAX_CONZ 8        /* passive tracers per basin                   */

enum shy_status {
  SHY_OK = 0,
  SHY_EARG = 1,       /* bad argument or size                            */
  SHY_ECUDA = 2,      /* CUDA runtime error / no device                  */
  SHY_ENOCONV = 3,    /* Krylov solve did not reach its tolerance        */
  SHY_ESINGULAR = 4,  /* zero pivot in a column or node solve            */
  SHY_EDEPTH = 5,     /* non-positive layer thickness                    */
  SHY_EISTOT = 6,     /* transport sub-step count above the limit        */
  SHY_ENAN = 7,       /* non-finite value in the state                   */
  SHY_ESTATE = 8,     /* call out of order (e.g. solve before initialize)*/
  SHY_ECAPACITY = 9   /* request does not fit the device memory budget   */
};

/* ------------------------------------------------------------------ */
/* Static description of one basin (host pointers, copied at create)   */
/* ------------------------------------------------------------------ */
typedef struct shy_basin {
  int32_t nkn, nel, nlv;        /* nodes, elements, layers (nlvdi == nlv)   */
  const int32_t *nen3v;         /* (3,nel) 1-based           basin::nen3v  */
  const float *xgv, *ygv;       /* (nkn) cartesian [m]       basin::xgv    */
  const float *hm3v;            /* (3,nel) depth at vertices basin::hm3v   */
  const float *hlv;             /* (nlv) bottom depth of z-layer l  levels  */
  const float *hldv;            /* (nlv) nominal layer thickness    levels  */
  const int32_t *ilhv;          /* (nel) layers in element          levels  */
  const int32_t *ilhkv;         /* (nkn) layers at node             levels  */
  const float *czv;             /* (nel) friction parameter  (chezy.f90)    */
  const float *fcorv;           /* (nel) Coriolis parameter [1/s]           */
  const float *visv;            /* (0:nlv,nkn) vertical viscosity           */
  const float *difv;            /* (0:nlv,nkn) vertical diffusivity         */
  const float *tauxnv, *tauynv; /* (nkn) wind stress / rho0  (mod_meteo)    */
  const float *ppv;             /* (nkn) atmospheric pressure term          */
  const float *rqv;             /* (nkn) discharge of flux boundaries and point */
                                /*   sources [m^3/s]: the zeta right-hand side  */
                                /*   (system_add_rhs) and, spread over the      */
                                /*   node's layers by volume (set_mass_flux,    */
                                /*   mfluxv), w and the transport               */
  const int32_t *bnd_index;     /* (nkn) 0 or the level-boundary number b>0 */
  int32_t nbnd, ntide;          /* level boundaries, constituents each      */
  const float *tide;            /* (4,ntide,nbnd): ampli, period, phase, zref
                                   (bnd_admin.f90:1304-1320, summed)        */
} shy_basin;

/* Parameters under their `.str` names (src/shyfem/def_para.f90).          */
typedef struct shy_params {
  double dt;                 /* time step [s]                               */
  double dtime0;             /* time of the initial state [s]               */
  float azpar, ampar, afpar; /* semi-implicit weights        :666-668       */
  float atpar, adpar, aapar; /* vertical implicit weights    :684-686       */
  float grav, rowass;        /*                              :782-784       */
  float vismol, difmol;      /* molecular viscosity/diffusivity :993-995    */
  float hzoff;               /* minimum depth for friction   :745           */
  float ahpar;               /* horizontal viscosity         :1023          */
  float rstol;               /* transport Courant limit      :1055          */
  float thpar, shpar, chpar; /* horizontal diffusivity T, S, tracers        */
  int32_t ireib;             /* friction type                :766           */
  int32_t ibarcl;            /* baroclinic pressure (1) or not (0)          */
  int32_t ilin;              /* 1: linear momentum; 0: explicit upwind      */
                             /*   advection (set_advective, itlin 0, avpar 0) */
  int32_t itemp, isalt;      /* transport temperature / salinity            */
  int32_t nconz;             /* passive tracers                             */
  int32_t istot_max;         /* transport sub-step limit (scal3sh: 1000)    */
  float solver_rtol;         /* Krylov stop ||r|| <= rtol*||r0|| + atol     */
  float solver_atol;         /*   (sparskit_admin.f90:270-277: 1e-8, 1e-8)  */
  int32_t solver_maxit;      /* iteration limit (sparskit_admin.f90:141)    */
  int32_t nsigma;            /* sigma layers (levels :: nsigma): 0 z-layers, */
                             /*   nlv pure sigma (hlv/hldv sigma values < 0),*/
                             /*   between: hybrid, z-layers below hsigma and */
                             /*   hlv(nsigma) = hsigma (initialize.f90:556)  */
  float hsigma;              /* depth limit of the sigma layers (hsigma)    */
  int32_t wetdry;            /* 1: wetting and drying of elements (setweg) */
  float hzmin, hzon, volmin; /* its thresholds       def_para.f90:744-746,1762 */
  float rlin;                /* strength of the advective terms (ilin 0) :590 */
  int32_t itvd;              /* horizontal transport: 0 upwind, 1 TVD with  */
                             /*   node gradients (superbee)     :1053       */
  int32_t itvdv;             /* vertical transport: 0 upwind, 1 TVD          */
                             /*   (superbee; needs aapar = 0)   :1054       */
  int32_t ihwadv;            /* vertical advection of momentum with ilin 0:  */
                             /*   0 none, 1 upwind, 2 centred   :1350       */
  int32_t nzadapt;           /* z-layers whose top layers follow the level  */
                             /*   (z-star, zadaptutil.f90): <= 1 plain z-   */
                             /*   layers, >= nlv all layers, between: the   */
                             /*   surface layers down to where the level    */
                             /*   reaches (nzadapt at rest); z-layers only, */
                             /*   no baroclinic terms, no wetting and drying */
  int32_t inohyd;            /* 1: non-hydrostatic pressure (nohydro.f90,   */
                             /*   def_para.f90:1933): a 3D Poisson system  */
                             /*   per step corrects level and transports;  */
                             /*   no wetting and drying, no z-adaptive     */
                             /*   layers                                   */
  float aqpar;               /* its semi-implicit weight (0.5)      :1935   */
  int32_t ivwadv;            /* vertical advection of w: 0 none, 1 upwind, */
                             /*   2 centred differences              :1939  */
  int32_t inhflx;            /* horizontal advection of w: 0 averaged, 1   */
                             /*   upwind fluxes                     :1940   */
} shy_params;

/* Host views of one basin's state, reference layouts.  NULL members are
 * skipped by set/get.                                                      */
typedef struct shy_state {
  float *znv;      /* (nkn) water level                         mod_hydro    */
  float *zenv;     /* (3,nel) water level at element vertices   mod_hydro    */
  float *utlnv;    /* (nlv,nel) transport in x                  mod_hydro    */
  float *vtlnv;    /* (nlv,nel) transport in y                  mod_hydro    */
  float *unv;      /* (nel) barotropic transport in x       mod_hydro_baro   */
  float *vnv;      /* (nel) barotropic transport in y                        */
  float *hdknv;    /* (nlv,nkn) layer thickness at nodes  mod_layer_thickness*/
  float *hdenv;    /* (nlv,nel) layer thickness at elements                  */
  float *wlnv;     /* (0:nlv,nkn) vertical velocity             mod_hydro_vel*/
  float *tempv;    /* (nlv,nkn) temperature                     mod_ts       */
  float *saltv;    /* (nlv,nkn) salinity                        mod_ts       */
  float *rhov;     /* (nlv,nkn) density anomaly rho'            mod_ts       */
  float *conzv;    /* (nlv,nkn,nconz) passive tracers                        */
} shy_state;

/* Per-step diagnostics of one basin (last completed step).               */
typedef struct shy_step_info {
  int32_t status;        /* SHY_OK or the first error of the step          */
  int32_t krylov_iters;  /* inner Krylov iterations of the zeta solve      */
  int32_t refinements;   /* FP64 residual refinement sweeps                */
  int32_t istot;         /* transport sub-steps of the last scalar pass    */
  double resid0;         /* ||b - A z_guess|| (FP64)                       */
  double resid;          /* final ||b - A z|| (FP64)                       */
  double volume;         /* total water volume, FP64 sum (vol_mass)        */
  double dtime;          /* model time of the state [s]                    */
  double volume_budget;  /* FP64 volume budget: the initial volume plus    */
                         /*   every step's dt times the flows into the     */
                         /*   node columns (element fluxes of the zeta     */
                         /*   equation, discharges), summed in FP64, so a  */
                         /*   closed basin keeps it to FP64 round-off      */
} shy_step_info;

typedef struct shygpu_model shygpu_model;   /* opaque, device-resident    */

/* ------------------------------------------------------------------ */
/* Geometry (init only)                                                */
/* ------------------------------------------------------------------ */

/* set_ev (src/utils/shyutil/evgeom.f90:167-320): shape-function gradients
 * b = ev(4:6), c = ev(7:9), aj = area/24 = ev(10), angles, heights and side
 * lengths for each element, cartesian coordinates.  ev is (SHY_EVDIM,nel). */
int shygpu_set_ev(int32_t nkn, int32_t nel, const int32_t *nen3v,
                  const float *xgv, const float *ygv, float *ev);

/* ------------------------------------------------------------------ */
/* Whole-phase, device-resident entries                                */
/* ------------------------------------------------------------------ */

/* shyfem_initialize's part for the step (shyfem_subs.f90:358-506): geometry,
 * areas (set_area), diffusion weights (diffweight), element neighbours, the
 * zeta-system sparsity (coo_init_new) and its gather maps, for `nbasin`
 * independent basins advanced together.  params has one entry per basin.  */
int shygpu_create(int32_t nbasin, const shy_basin *basins,
                  const shy_params *params, shygpu_model **model);
int shygpu_destroy(shygpu_model *model);

/* Upload a basin's state (znv, utlnv, vtlnv, tempv, saltv, conzv are read;
 * zenv, layer thicknesses and rhov are derived as sp111(1)/barocl(0) do).  */
int shygpu_set_state(shygpu_model *model, int32_t ibasin, const shy_state *st);
/* Download any subset of a basin's state.                                 */
int shygpu_get_state(shygpu_model *model, int32_t ibasin, shy_state *st);

/* `nsteps` iterations of shyfem_run's loop body for every basin:
 * copy_uvz/copy_depth, sp111(2) level boundaries, hydro
 * (hydrodynamic.f90:284-485) and run_scalar (shyfem_subs.f90:975-1028).
 * Returns the first non-zero status of any basin.                         */
int shygpu_run(shygpu_model *model, int32_t nsteps);
/* shygpu_run split in two: queue the steps on the model's stream and return
 * at once; then wait for them and report the first error of any basin.   */
int shygpu_enqueue(shygpu_model *model, int32_t nsteps);
int shygpu_sync(shygpu_model *model);

/* The same step split at the reference's phase boundaries:
 * new_step = copy_uvz + copy_depth + sp111(2); hydro = hydrodynamic.f90:284;
 * scalar = run_scalar (barocl T/S + rhoset + tracers).                    */
int shygpu_new_step(shygpu_model *model);
int shygpu_hydro(shygpu_model *model);
int shygpu_scalar(shygpu_model *model);

/* Wetting and drying state of basin ib (mod_geom_dynamic): per element the
 * number of its vertices that took it out of the system (0: in it) and its
 * wet/dry step counter (iwetv), per node 0 internal, > 0 open boundary, -1
 * boundary of the wet domain, -2 out of the system (inodv, as of the last
 * solve).  Zeros for a model without wetting and drying.                 */
int shygpu_get_wetdry(shygpu_model *model, int32_t ibasin, int32_t *iwegv,
                      int32_t *iwetv, int32_t *inodv);
int shygpu_step_info(shygpu_model *model, int32_t ibasin, shy_step_info *info);

/* Non-hydrostatic pressure of a basin made with inohyd = 1 (nohydro.f90).
 * Each step, after the hydrostatic transports, solves the 3D pressure
 * system (nonhydro_prepare_matrix, :589-753, from the w of sp256wnh,
 * :205-524) and corrects levels and transports (nonhydro_correct_uveta,
 * :761-829).  set_nh_distance replaces the per-node weight of the pressure
 * (qdistv, made by qhdist :962-1040 from the open boundaries' nad; 1 by
 * default), values in [0, 1].  get_nh_pressure copies the pressure the
 * next step starts from, (nlv,nkn), first layer zero (qpnv after
 * nonhydro_adjust).  nh_info gives the last solve's Krylov iterations,
 * FP64 refinements and residuals (initial, final).                        */
int shygpu_set_nh_distance(shygpu_model *model, int32_t ibasin, const float *qdistv);
int shygpu_get_nh_pressure(shygpu_model *model, int32_t ibasin, float *qpnv);
int shygpu_nh_info(shygpu_model *model, int32_t ibasin, int32_t *iters, int32_t *refinements,
                   double *resid0, double *resid);

/* Per-step forcing of a basin from host memory (pinned for overlap):
 * tauxnv, tauynv, ppv, rqv (nkn each); NULL members are left unchanged.
 * The copies are queued on the model's stream ahead of the next step,
 * like the meteo/boundary reads that precede hydro in shyfem_run.        */
int shygpu_set_forcing(shygpu_model *model, int32_t ibasin, const float *tauxnv,
                       const float *tauynv, const float *ppv, const float *rqv);

/* Whole-model transfers for pipelined serving (no reference counterpart:
 * the reference runs one basin per process).  set_forcing_all copies the
 * forcing of every basin, concatenated in basin order (NKN values per
 * array, NULL skips one); get_levels copies the water level of every basin
 * of the latest enqueued step the same way.  Both return at once and act
 * in order with the steps enqueued around them; they are complete after
 * shygpu_sync (or shygpu_run).  The copies run on two transfer streams of
 * the model, so with pinned host buffers they overlap the steps as well as
 * the host's work: the forcing of the next step goes up while the current
 * one runs (through one of two device staging copies, allocated on first
 * use and counted by shygpu_model_bytes), and a step's level comes down
 * while the following step runs.  The host buffers must stay untouched
 * until shygpu_sync.                                                        */
int shygpu_set_forcing_all(shygpu_model *model, const float *tauxnv, const float *tauynv,
                           const float *ppv, const float *rqv);
int shygpu_get_levels(shygpu_model *model, float *znv);

/* Hydro output of basin ib in the reference's .shy format (io_shy.f90,
 * shy_util.f90:450-480, 1210-1250: the header of shyfem_init_hydro_file,
 * then per shygpu_shy_write the water level at nodes and element vertices
 * and the transports U, V of the current state).  basin is the
 * description the model was made from (mesh arrays for the header).  Each
 * write enqueues its device-to-host copies on the model's stream into one
 * of two pinned buffers and returns; a writer thread writes the records
 * once the copies are done, so output overlaps the next steps.  close
 * waits for the writes and reports any error.                              */
typedef struct shygpu_shyfile shygpu_shyfile;
int shygpu_shy_open(shygpu_model *model, int32_t ibasin, const shy_basin *basin, const char *path,
                    int32_t date, int32_t time, const char *title, shygpu_shyfile **file);
int shygpu_shy_write(shygpu_shyfile *file);
int shygpu_shy_close(shygpu_shyfile *file);
/* Scalar output of basin ib in the same way: what 1, temperature and
 * salinity (the ts.shy file of bcl_write_output, baroclinic.f90:1163-1190:
 * records 11 salinity, 12 temperature, and 13 density when with_rho);
 * what 2, the passive tracers (the conz.shy file of tracer_write,
 * conz_admin.f90:535-575: record 10 for one tracer, 300 + i for several).
 * Scalar files are ftype 2 with npr 1 (shyfem_init_scalar_file,
 * shy_util.f90:484-518); each record holds the active layers of each node.
 * shygpu_shy_write and shygpu_shy_close serve both kinds of file.          */
int shygpu_shy_open_scalar(shygpu_model *model, int32_t ibasin, const shy_basin *basin,
                           const char *path, int32_t date, int32_t time, const char *title,
                           int32_t what, int32_t with_rho, shygpu_shyfile **file);

/* Time series at chosen nodes of basin ib in the reference's .ext format
 * (wrexta, extra.f90:254-575; records of io_ext.f90:468-575).  nodes are
 * n basin node numbers (1-based, the knaus of the $extra section); names
 * (optional) n blank-padded 80-character station names; atime0 the
 * absolute time of the model's time origin, added to the model time of
 * each record.  Per shygpu_ext_write one record per variable: 1 the nodal
 * barotropic velocities and the water level, 2 the nodal velocities of each
 * layer (uvtop0, uvtopr, transforms.f90:160-270: area-weighted means over
 * the node's elements in the system), 12 temperature, 11 salinity, 13
 * density (with_rho and T/S transported), 10 the tracer of a one-tracer
 * basin.  A write waits for the model's stream.                           */
typedef struct shygpu_extfile shygpu_extfile;
int shygpu_ext_open(shygpu_model *model, int32_t ibasin, const shy_basin *basin, const char *path,
                    int32_t n, const int32_t *nodes, const char *names, const char *title,
                    double atime0, int32_t with_rho, shygpu_extfile **file);
int shygpu_ext_write(shygpu_extfile *file);
int shygpu_ext_close(shygpu_extfile *file);

/* Checkpoints (restart.f90:445-660, made exact): every device array of the
 * model and its time-level indices, copied to or from a host buffer of
 * shygpu_checkpoint_bytes(model) bytes.  A checkpoint loads into the model
 * that saved it or into one made from the same basins and parameters (and
 * the same calls that add arrays: shygpu_set_nudging, shygpu_conz3d, and
 * shygpu_conz3d with a source term); the run
 * then continues bit for bit.
 * Loading into a model with other arrays fails with SHY_EARG.  Both calls
 * wait for the model's stream.                                             */
int64_t shygpu_checkpoint_bytes(const shygpu_model *model);
int shygpu_checkpoint_save(shygpu_model *model, void *buf, int64_t nbytes);
int shygpu_checkpoint_load(shygpu_model *model, const void *buf, int64_t nbytes);

/* conz3d_omp (concentration_omp.f90:65-76) with its argument list, by value
 * and with the model and basin in front: one transport sub-step (isact of
 * istot) of one scalar of basin ib on the model's current hydrodynamic
 * state, for a host that keeps its own scal3sh loop and calls this where
 * it called conz3d_omp (concentration.f90:748) after shygpu_hydro.  cn1
 * (nlvddi, nkn) is read and overwritten with the new concentration; the
 * open-boundary values stay to the caller (bndo_setbc), gradxv/gradyv are
 * the caller's tvd_grad_3d result for itvd = 1.  Scalar nudging relaxes
 * toward cobs (nlvddi, nkn) at robs*rtauv, explicitly (an = 0,
 * concentration_omp.f90:694-709); settling lowers the vertical velocity by
 * wsink*wsinkv (0:nlvddi, nkn) (:496); loading adds rload*load (nlvddi, nkn)
 * in mass per second and, for a sink, takes at most an exponential decay
 * of the layer's mass over the sub-step, writing the load it took back
 * into load (conz3d_nodes :816-833).  An array whose factor is 0 is not
 * read.  cbound (nlvddi, nkn) is the concentration that inflows bring at
 * nodes with a discharge (the basin's rqv, spread over the layers as
 * mfluxv; :805-813); NULL lets them bring the node's own concentration.
 * co1 is not read (the reference's scratch).  nlvddi and nlev must be the
 * basin's nlv, azpar the model's.  The
 * first call (and the first with a source term) allocates the call's
 * device arrays.                                                          */
int shygpu_conz3d(shygpu_model *model, int32_t ibasin, float *cn1, float *co1, double ddt,
                  float rkpar, const float *difhv, const float *difv, float difmol,
                  const float *cbound, int32_t itvd, int32_t itvdv, const float *gradxv,
                  const float *gradyv, const float *cobs, float robs, const float *rtauv,
                  float wsink, const float *wsinkv, float rload, float *load,
                  float azpar, float adpar, float aapar, int32_t istot, int32_t isact,
                  int32_t nlvddi, int32_t nlev);

/* Water-level nudging of basin ib (hydro_zeta, hydrodynamic.f90:612,
 * 677-679): andgzv(nkn), the per-node contribution that the reference's
 * nudge_zeta (nudge.f90:300-338) makes from its observation stations,
 * enters each element's right-hand side as 4 aj dt andgzv.  The caller
 * computes it from its observations; it stays in force until set again.
 * The first call for a model allocates the array and rebuilds its step
 * graph.                                                                   */
int shygpu_set_nudging(shygpu_model *model, int32_t ibasin, const float *andgzv);

/* Boundary values of one scalar of basin ib, (nlv, nkn), as the reference's
 * boundary input of that scalar (r3v of make_scal_flux, bnd_routines.f90:
 * 1215-1300): imposed on the level-boundary nodes after every transport
 * sub-step (bndo_impbc) and brought in by the inflows at nodes with a
 * discharge (conz3d_nodes, concentration_omp.f90:805-813).  what: 0
 * temperature, 1 salinity, 2 passive tracer itr.  shygpu_set_state sets
 * them to the scalar's initial columns; call this after it.              */
int shygpu_set_bound_scalar(shygpu_model *model, int32_t ibasin, int32_t what,
                            int32_t itr, const float *values);

/* Tuning options by name: "use_graph" (CUDA-graph replay of whole steps,
 * the transport sub-step loop as a device-driven conditional node; default
 * 1), "cluster_size" and "zeta_threads" (shape of the per-basin cluster of
 * the zeta solve), "zeta_variant" (0 cluster solver with vectors in global
 * memory, 1 shared-memory clusters where every basin fits, 2 one
 * device-wide cooperative solve), "zeta_stage" (device-wide solve with
 * TMA-staged tiles), "inner_rtol" (residual reduction of each FP32 Krylov
 * sweep, default 1e-4), "inner_tol_frac" (an FP32 sweep also stops at this
 * fraction of the outer target, default 0.75), "max_outer" (FP64
 * refinement sweeps), "symmetric" (CG instead of BiCGStab; refused when
 * Coriolis makes the system non-symmetric), "column_threads" (1 one thread
 * per element column for up to 16 layers, 0 one warp segment),
 * "zeta_tile_rows" (rows per tile of the device-wide solver, default 1024),
 * "zeta_barrier_timeout_test" (failure detection: the device-wide solve's
 * barrier waits for an arrival that never comes and reports SHY_ECUDA).
 * Every change rebuilds the step graphs at the next step.                  */
int shygpu_set_option(shygpu_model *model, const char *name, double value);
double shygpu_get_option(shygpu_model *model, const char *name);

/* Autotuning of the launch shapes on the model's own basins (no counterpart
 * in the reference, which runs on CPU cores).  Candidates are sets of the
 * options above: the zeta solver's plan (zeta_variant, zeta_tile_rows,
 * zeta_stage; symmetric systems without wetting and drying), the column
 * kernels' form (column_threads; at most 16 layers) and the FP32 sweep's
 * tolerance (inner_tol_frac).  Each trial starts from the model's current
 * state (a host checkpoint), runs one untimed step and times `steps`
 * steps; the search takes one group at a time over the best of the groups
 * before it.  The model keeps the fastest candidate's options and the state
 * it had.  The winner is cached per model shape (basins, rows to two
 * digits, layers, solver, scalars, device) for the process, and appended to
 * the file named by the environment variable SHYGPU_TUNE_FILE, if set, which
 * later processes read; a cached shape is applied without trials.  choice
 * (optional) receives the options as "name=value ...", ms_per_step
 * (optional) the winner's time per step (-1 when it came from the cache).
 * get_option(model, "tuned") is 1 afterwards.                             */
int shygpu_autotune(shygpu_model *model, int32_t steps, char *choice, int32_t choice_len,
                    double *ms_per_step);

/* The CUDA stream every launch of the model goes to (cudaStream_t).      */
void *shygpu_model_stream(shygpu_model *model);

/* Run `nsteps` steps with CUDA events between the kernels of each step and
 * return the summed device time per kernel kind in ms_out[SHY_NKERNEL] and
 * the launches per kind in count_out (kinds: column, zeta, final, node,
 * stab, reduce, conz, rho).                                               */
#define SHY_NKERNEL 8
int shygpu_profile_steps(shygpu_model *model, int32_t nsteps, double *ms_out, int32_t *count_out);
/* Device bytes held by the model (admission by HBM footprint).            */
int64_t shygpu_model_bytes(const shygpu_model *model);
/* Bytes a model of these basins would hold, without allocating.           */
int64_t shygpu_footprint(int32_t nbasin, const shy_basin *basins,
                         const shy_params *params);

/* Kernel launches issued by this process so far (for accounting).         */
int64_t shygpu_launch_count(void);
const char *shygpu_last_error(void);

/* ------------------------------------------------------------------ */
/* The reference's simsys interface (src/shyfem/simsys_spkaux.f90)     */
/* gfortran by-reference convention; element data in shy_zeta_system.  */
/* ------------------------------------------------------------------ */

/* mod_zeta_system :: kn(3), hia(3,3), hik(3)  (simsys_spkaux.f90:75-83).
 * hia is column-major like the Fortran array: hia[(m-1)*3 + (n-1)].      */
typedef struct shy_zeta_system_t {
  int32_t kn[3];
  float hia[9];
  float hik[3];
} shy_zeta_system_t;
extern shy_zeta_system_t shy_zeta_system;

/* Registration that replaces the module state system_initialize reads
 * (basin :: nkn, nel, nen3v).  Must precede system_initialize_.           */
int shygpu_simsys_register(int32_t nkn, int32_t nel, const int32_t *nen3v);
/* Solver controls (defaults 1e-8, 1e-8, 1000 as sparskit_admin.f90).      */
int shygpu_simsys_set_tolerance(double rtol, double atol, int32_t maxit);
/* Assembled matrix of the last solve, CSR rows = nodes (FP64 values, as
 * the reference's c2coo) and its right-hand side, for inspection.         */
int shygpu_simsys_get_matrix(int32_t *n, int32_t *nnz, int32_t *rowptr,
                             int32_t *col, double *val, double *rhs);
int shygpu_simsys_iterations(void);
/* The 3D system of the non-hydrostatic pressure and of poisson_3d
 * (coo_init_new's 3D part, coo_matrix.f90:180-247): nlv layers (levels ::
 * nlv, read by system_initialize from its module) are declared here before
 * system_initialize_; 0 (the default) leaves the 3D system out, as the
 * reference does without bsys3d.  Its unknowns are (nlv+2) per node, layer
 * 0 and nlv+1 padding rows with a unit diagonal.                          */
int shygpu_simsys_set_layers(int32_t nlv);
/* The assembled 3D matrix of the last solve, CSR over (nlv+2)*nkn rows in
 * the order of the reference's c3coo (FP64), and its right-hand side.     */
int shygpu_simsys_get_matrix_3d(int32_t *n, int32_t *nnz, int32_t *rowptr,
                                int32_t *col, double *val, double *rhs);

/* Solve A x = rhs for one sparse system whose CSR arrays (0-based, rows with
 * their diagonal stored), right-hand side, start x0 and result x are all in
 * device memory, without allocating any device memory.  This entry point
 * has no counterpart in the reference: it serves callers that cannot let a
 * solver take device memory (a model embedded in a framework whose memory
 * pool owns the GPU, a server that admits work by an exact memory budget, a
 * time loop that must not stall other streams on cudaMalloc/cudaFree).  The
 * solver is the one of system_solve_ (Jacobi-preconditioned CG when
 * symmetric != 0, else BiCGStab, FP32 inside FP64 refinement, stop when
 * ||r|| <= rtol*||r0|| + atol); its work vectors live in a fixed 5 MiB
 * array inside the library.  At most 65536 rows and 524288 stored entries:
 * larger systems return SHY_ECAPACITY.  The kernel checks the CSR arrays
 * before it writes anything (rowptr[0] = 0, rowptr[n] = nnz, no row of
 * negative length, columns in [0, n)) and returns SHY_EARG otherwise.
 * maxit bounds the Krylov iterations of the whole call, summed over its
 * refinement rounds (at most 12), and the returned status always describes
 * the returned x.  The first call on a device, with
 * that device current, looks the array up and must come before any stream
 * capture begins.  There is one such array per device, so calls that
 * overlap on one device race: serialise them.  x may equal x0.  The call
 * waits for the solve on `stream` (a cudaStream_t, NULL = default stream);
 * *iterations (optional) receives the Krylov iteration count.            */
int shygpu_csr_solve_static(int32_t n, int32_t nnz, const int32_t *rowptr,
                            const int32_t *col, const double *val,
                            const double *rhs, const float *x0, float *x,
                            double rtol, double atol, int32_t maxit,
                            int32_t symmetric, void *stream,
                            int32_t *iterations);

/* ------------------------------------------------------------------ */
/* Serving: a continuous-batching request loop (no counterpart in the   */
/* reference, which runs one simulation per process).  A request is a   */
/* basin, its parameters, its initial state and a step count; it is     */
/* admitted in arrival order once a slot is free and its footprint      */
/* (shygpu_footprint) fits the rest of the HBM budget, then runs with   */
/* its state resident on the device, concurrently with the other runs,  */
/* in quanta of `quantum_steps` CUDA-graph steps.  Inputs are copied at */
/* submit; results (znv, utlnv, vtlnv and the transported scalars) are  */
/* copied to host memory when the run finishes.  One host thread at a  */
/* time drives a server.                                                */
/* ------------------------------------------------------------------ */
typedef struct shygpu_server shygpu_server;
enum { SHY_REQ_QUEUED = 0, SHY_REQ_ACTIVE = 1, SHY_REQ_DONE = 2, SHY_REQ_FAILED = 3 };
int shygpu_serve_create(int64_t hbm_budget_bytes, int32_t max_active,
                        int32_t quantum_steps, shygpu_server **server);
int shygpu_serve_submit(shygpu_server *server, const shy_basin *basin,
                        const shy_params *params, const shy_state *initial,
                        int32_t nsteps, int64_t *request_id);
/* Retire finished runs, launch the next quantum of every run whose last
 * one has finished, admit queued requests.  block != 0 first waits for
 * the oldest quantum in flight.  Counts of active, queued and newly
 * finished requests are returned through the (optional) pointers.       */
int shygpu_serve_progress(shygpu_server *server, int32_t block,
                          int32_t *n_active, int32_t *n_queued,
                          int32_t *n_finished);
/* state SHY_REQ_*; times in seconds since the server was created        */
int shygpu_serve_status(shygpu_server *server, int64_t request_id,
                        int32_t *state, int32_t *steps_enqueued,
                        double *t_submit, double *t_admit, double *t_done);
int shygpu_serve_result(shygpu_server *server, int64_t request_id,
                        shy_state *out, shy_step_info *info);
int shygpu_serve_release(shygpu_server *server, int64_t request_id);
/* Preempt a running request: it stops after its quantum in flight, its
 * device arrays are saved to host memory (shygpu_checkpoint_save), its
 * device memory is freed, and it queues behind the requests already
 * waiting (an urgent request submitted before the call is admitted first);
 * when admitted again it continues bit for bit.                            */
int shygpu_serve_preempt(shygpu_server *server, int64_t request_id);
int64_t shygpu_serve_used(shygpu_server *server);   /* admitted footprint */
int shygpu_serve_destroy(shygpu_server *server);

void system_initialize_(void);                      /* :85   */
void system_init_(void);                            /* :137  */
void system_set_explicit_(void);                    /* :160  */
void system_assemble_(const int32_t *ie);           /* :533  */
void system_add_rhs_(const float *dt, const int32_t *n, const float *array); /* :687 */
void system_solve_(const int32_t *n, const float *z);                        /* :454 */
void system_get_(const int32_t *n, float *z);                                /* :638 */
void system_finalize_(void);                        /* :722  */
/* The 3D interface (simsys_spkaux.f90:495-716), used by nonhydro_prepare_
 * matrix (nohydro.f90:589-753) and poisson_3d (poisson.f90:272-445):
 * mass(-1:1,3,3) and rhs(3) of element ie, layer l, nodes kn (Fortran
 * order, mass[(d+1) + 3*(i-1) + 9*(j-1)]) are added to the rows of layer l
 * and their couplings to layers l-1 and l+1; adjust_matrix sets a unit
 * diagonal where no element layer reached it; solve_3d takes z(nlvdi,n)
 * as the guess and solves on the GPU (BiCGStab in FP32 inside FP64
 * refinement, the stop test of system_solve_); get_3d copies the solution
 * into z(nlvdi,n).                                                        */
void system_assemble_3d_(const int32_t *ie, const int32_t *l, const int32_t *nlv, const int32_t *kn,
                         const float *mass, const float *rhs);                          /* :597 */
void system_adjust_matrix_3d_(void);                                                  /* :709 */
void system_solve_3d_(const int32_t *n, const int32_t *nlvdi, const int32_t *nlv, const float *z); /* :495 */
void system_get_3d_(const int32_t *n, const int32_t *nlvdi, const int32_t *nlv, float *z);        /* :657 */

#ifdef __cplusplus
}
#endif

#endif /* SHYGPU_H */
