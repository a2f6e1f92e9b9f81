/*
 * sem_b200.h - C ABI of the B200 elastic spectral-element time loop.
 *
 * Drop-in replacement for the hot path that SpecFWAT's xfwat_fwd_measure_adj
 * drives through its SPECFEM interface layer:
 *
 *   reference call                                   replaced by
 *   -----------------------------------------------  -------------------------
 *   read_mesh_databases_fwat + prepare_GPU (mesh)     sem_prepare_mesh
 *     src/specfem_interface/read_mesh_databases.f90:91-1396
 *     src/specfem_interface/prepare_timerun_fwat.f90:120
 *   prepare_timerun_fwat(ievt)                        sem_prepare_timerun
 *     src/specfem_interface/prepare_timerun_fwat.f90:29-168
 *   setup_sources_receivers_fwat(ievt)                sem_set_sources,
 *     src/specfem_interface/setup_sources_receivers_fwat.f90:29-88
 *                                                     sem_set_receivers
 *   iterate_time() (SIMULATION_TYPE 1 / 3)            sem_iterate_time
 *     called at src/preproc/prepare_fwd.f90:364
 *   seismograms_d read by read_syn_data               sem_get_seismograms
 *     src/preproc/syn_data.f90:64-66
 *   SEM/<sta>.adj written by write_adj, read back as      sem_set_adjoint_sources
 *   source_adjoint                                    (or sem_measure_l2)
 *     src/preproc/syn_data.f90:232-251,
 *     src/specfem_interface/setup_sources_receivers_fwat.f90:487-490
 *   WaveformMisfit%calc_adjoint_source                sem_measure_l2
 *     src/preproc/adjoint_sources/waveform_misfit.f90:15-64
 *   compute_kernels + save_adjoint_kernels            sem_save_adjoint_kernels
 *     called at src/preproc/prepare_fwd.f90:381
 *   PostFlow%sum_kernel (cross-event sum)             sem_sum_kernels
 *     src/postproc/post_processing.f90:108-149
 *   FinalizeSpecfem / prepare_cleanup_device          sem_release_run,
 *     src/specfem_interface/specfem_api.f90:298-369    sem_release_mesh
 *   Veloc_FK / Tract_FK (FK injection)                sem_set_injection
 *     src/shared/fk_coupling.f90:71-439
 *   hess_kernel (APPROXIMATE_HESS_KL) and its sum      sem_set_approximate_hessian,
 *     src/postproc/post_processing.f90:171-218         sem_save_hessian_kernel,
 *                                                     sem_sum_hessian
 *   invert_hess / zprecond_gll                        sem_hessian_precond,
 *     post_processing.f90:333-372, zprecond.f90:34-71  sem_depth_precond
 *   smooth_sem_pde                                    sem_smooth_pde
 *     src/postproc/smooth.f90:7-437
 *   gll2grid (Project_model_SEM2FD_grid)              sem_grid_project
 *     src/grid/model_grid_data.f90:183-198,
 *     src/shared/projection_on_FD_grid_mod_fwat.f90:186-596,935-1125
 *   PostFlow%taper_kernel_grid (taper_cls)            sem_grid_taper
 *     src/postproc/post_processing.f90:283-325, taper_3D_mod.f90
 *   zprecond_grid                                     sem_grid_zprecond
 *     src/postproc/zprecond.f90:73-100
 *
 * Conventions
 *  - Every function returns SEM_OK (0) or a negative sem_status; the reason
 *    is kept per thread and returned by sem_last_error().  No call aborts
 *    the process (the reference aborts through exit_MPI).
 *  - All arrays are caller-owned HOST arrays; the library copies them.
 *  - Index arrays may be 0- or 1-based (sem_mesh_desc.index_base), so the
 *    Fortran database arrays can be passed unchanged.
 *  - Array layouts are the reference's Fortran column-major layouts read as
 *    C row-major with the indices reversed: ibool(5,5,5,nspec) is
 *    ibool[nspec][5][5][5] with i fastest; abs_boundary_ijk(3,25,nf) is
 *    ijk[nf][25][3]; seismograms are [nrec][3][nstep] with components
 *    (x=East, y=North, z=Up).
 *  - One run handle per host thread; calls on one handle must not overlap.
 *    All device work of a run is queued on the run's own CUDA stream.
 */
#ifndef SEM_B200_H
#define SEM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SEM_ABI_VERSION 2

typedef enum {
  SEM_OK = 0,
  SEM_ERR_ARG = -1,          /* invalid argument or inconsistent sizes      */
  SEM_ERR_CUDA = -2,         /* CUDA runtime error                          */
  SEM_ERR_NOMEM = -3,        /* device memory budget or allocation failed   */
  SEM_ERR_STATE = -4,        /* call out of order (e.g. adjoint w/o forward)*/
  SEM_ERR_UNSUPPORTED = -5,  /* input outside what this build implements    */
  SEM_ERR_NUMERIC = -6,      /* non-finite wavefield detected               */
  SEM_ERR_NODEVICE = -7      /* no usable sm_100 device                      */
} sem_status;

/* Mesh database of one slice (read_mesh_databases.f90:158-193,455-486,
 * 766-804).  Regular elements (cubes) share xix_regular and
 * jacobian_regular.  irregular_element_number[e] (read_mesh_databases.f90:
 * 168) is 0 for a regular element and k >= 1 for an irregular one, whose
 * mapping derivatives and Jacobian are row k-1 of xixstore .. jacobianstore
 * (read_mesh_databases.f90:172-181), each [nspec_irregular][5][5][5].  A
 * mesh with irregular elements runs the thread-per-point element kernel. */
typedef struct {
  int nspec;
  int nglob;
  int index_base;                   /* 0 (C) or 1 (Fortran) for ibool/ijk  */
  const int *ibool;                 /* [nspec][5][5][5]                    */
  const float *xstore, *ystore, *zstore;   /* [nglob] metres               */
  float xix_regular;                /* d xi / d x of the regular elements  */
  float jacobian_regular;           /* (h/2)^3                             */
  const int *irregular_element_number;     /* [nspec] or NULL              */
  const float *kappastore, *mustore, *rhostore;   /* [nspec][125]          */
  const float *rmass;               /* [nglob] assembled mass (no Stacey)  */
  const float *rho_vp, *rho_vs;     /* [nspec][125]                        */
  int num_abs_boundary_faces;
  const int *abs_boundary_ispec;    /* [nf]                                */
  const int *abs_boundary_ijk;      /* [nf][25][3]                         */
  const float *abs_boundary_jacobian2Dw;   /* [nf][25]                     */
  const float *abs_boundary_normal; /* [nf][25][3]                         */
  int nspec_irregular;              /* rows of the irregular arrays (>= 0) */
  const float *xixstore, *xiystore, *xizstore;         /* [nirr][125]      */
  const float *etaxstore, *etaystore, *etazstore;      /* [nirr][125]      */
  const float *gammaxstore, *gammaystore, *gammazstore;/* [nirr][125]      */
  const float *jacobianstore;                          /* [nirr][125]      */
} sem_mesh_desc;

/* Run options (prepare_timerun_fwat.f90:29-168 + Par_file switches). */
typedef enum { SEM_STORE_FP32 = 0, SEM_STORE_FP16 = 1 } sem_store_kind;

typedef struct {
  int nev;            /* events in this run (1 = plain path)               */
  int nstep;          /* NSTEP                                             */
  double dt;          /* DT (s)                                            */
  int store_kind;     /* sem_store_kind for the Stacey boundary store      */
  int use_graph;      /* 1: replay the step loop as CUDA graphs            */
  int graph_steps;    /* steps per captured graph (0 = default 50)         */
  int max_receivers;  /* receivers per event upper bound (>= 1)            */
  int check_every;    /* steps between non-finite checks (0 = off): the
                         wavefields (adjoint and backward in sim_type 3)
                         are scanned per event inside the loop, at the
                         first graph boundary after every check_every
                         steps; an event found non-finite stops there
                         and sem_iterate_time returns SEM_ERR_NUMERIC
                         with the event and step.  Lane-driven runs check
                         their lanes the same way (sem_lane_status /
                         sem_lane_finish report SEM_ERR_NUMERIC for the
                         stopped lane only).  The solver's equivalent is
                         the check every NTSTEP_BETWEEN_OUTPUT_INFO steps */
  int kernel_variant; /* element kernel: 0 autotuned per phase,
                         1 thread-per-point, 2 pencil decomposition,
                         3 pencil, persistent and cp.async-pipelined,
                         4 as 3 with 2 events per block, 5 as 3 with 2
                         events per thread, 6 as 5 with 4 events per
                         thread (forward) / 8 per block (adjoint),
                         7 / 8 as 5 forward and, in the adjoint phase,
                         the adjoint and backward fields of an event as
                         one float2 (4 / 8 events per block), 9 / 10 as
                         7 / 8 with the gather prefetched in registers,
                         11 forward with 2 events per thread and the
                         gather in registers, adjoint as 10, 12 as 11
                         with the forward scatter as plain read-modify-
                         writes in one launch per element colour, 13
                         thread per point with xi contractions by warp
                         shuffles (one event per block), 14 forward as 11
                         and an adjoint kernel sized for three blocks per
                         SM (divergence summed in shared memory), 15 a
                         forward kernel sized for five blocks per SM the
                         same way and the adjoint kernel of 11           */
} sem_run_cfg;

/* CMTSOLUTION-style moment-tensor source.  Moment tensor in the Harvard
 * CMT frame (r up, theta south, phi east), mapped to x=E, y=N, z=Up as
 * locate_source_fwat.f90:215-228 does; Ricker wavelet with dominant
 * frequency f0 centred at 1.2/f0 + tshift (locate_source_fwat.f90:499-506). */
typedef struct {
  double x, y, z;             /* metres, z <= 0 is depth                  */
  double Mrr, Mtt, Mpp, Mrt, Mrp, Mtp;   /* N m                            */
  double f0;                  /* Hz                                       */
  double tshift;              /* s                                        */
} sem_source;

typedef struct sem_mesh_s sem_mesh;
typedef struct sem_run_s sem_run;

/* Library / device information. */
int sem_abi_version(void);
const char *sem_last_error(void);
int sem_device_info(int *sm_count, long long *hbm_bytes, int *cc_major,
                    int *cc_minor);

/* Mesh residency: upload a database once; many runs may share it. */
int sem_prepare_mesh(const sem_mesh_desc *desc, sem_mesh **out);
int sem_release_mesh(sem_mesh *mesh);
int sem_mesh_info(const sem_mesh *mesh, int *nspec, int *nglob, int *nfaces,
                  long long *device_bytes);

/* Per-run device state: mass matrix with the Stacey term for this dt,
 * wavefields, boundary store, seismogram and kernel buffers. */
int sem_prepare_timerun(sem_mesh *mesh, const sem_run_cfg *cfg,
                        sem_run **out);
int sem_release_run(sem_run *run);
/* Bytes sem_prepare_timerun would allocate for this cfg with sim types
 * 1 and 3 (HBM-budget admission). */
long long sem_run_bytes(const sem_mesh *mesh, const sem_run_cfg *cfg);

/* Sources and receivers (located on the host, nearest element centre). */
int sem_set_sources(sem_run *run, int nev, const sem_source *src);
int sem_set_receivers(sem_run *run, int ev, int nrec, const double *xyz);

/* Time loop.  sim_type 1: forward (save_forward=1 keeps the boundary store
 * and the final state in HBM for a later sim_type 3).  sim_type 3: adjoint
 * field driven by the adjoint sources plus backward reconstruction with
 * kernel accumulation.  Asynchronous: returns after queueing. */
int sem_iterate_time(sem_run *run, int sim_type, int save_forward);
int sem_synchronize(sem_run *run);

/* Seismograms of event ev: out[nrec][3][nstep] (displacement, m). */
int sem_get_seismograms(sem_run *run, int ev, float *out);
/* Adjoint sources of event ev in forward time order, [nrec][3][nstep]. */
int sem_set_adjoint_sources(sem_run *run, int ev, const double *adj);
/* L2 waveform misfit on the device in FP64 between the last forward
 * seismograms of ev and obs[nrec][3][nstep]; sets the adjoint sources of ev
 * and writes the misfit (sum over receivers and components). */
int sem_measure_l2(sem_run *run, int ev, const double *obs,
                   double taper_pct, int taper_type, double *misfit);

/* Kernels of event ev after sim_type 3: out[6][nspec][125] in the order
 * rho, mu, kappa, rhop, beta, alpha (names of post_processing.f90:417-422). */
int sem_save_adjoint_kernels(sem_run *run, int ev, double *out);
/* FP64 sum of the six kernels over all events of the run, same layout. */
int sem_sum_kernels(sem_run *run, double *out);

/* Observed data of event ev kept in device memory, [nrec][3][nstep]; a
 * later sem_measure_l2 with obs == NULL uses it (no host transfer). */
int sem_set_observed(sem_run *run, int ev, const double *obs);

/* Queue all work of the run on the caller's CUDA stream (a cudaStream_t
 * passed as void*; NULL restores the run's own stream). */
int sem_set_stream(sem_run *run, void *stream);

/* FP64 sum of the six kernels over all events into DEVICE memory
 * dev_out[6][nspec][125] (e.g. a buffer handed to a collective). */
int sem_sum_kernels_device(sem_run *run, double *dev_out);

/* Spatial share of the GPU for runs of different meshes working at once:
 * the run's persistent element kernels fill at most sm_limit SMs (0: all),
 * leaving room for the other runs' kernels, and high_priority = 1 puts the
 * run's own stream at the device's highest stream priority (0: lowest), so
 * that the blocks of a small mesh's short kernels go ahead of a large
 * mesh's queued ones.  A stream set with sem_set_stream keeps its own
 * priority.  No counterpart in the reference. */
int sem_set_sm_share(sem_run *run, int sm_limit, int high_priority);

/* Boundary store held partly in host memory (the reference keeps the
 * whole store on disk: absorb_field.bin, src/specfem_interface/
 * specfem_api.f90:359-361, deleted at src/preproc/prepare_fwd.f90:376-377).
 * device_store_bytes = 0 (default): the whole store is in HBM.  > 0: at
 * most that many device bytes hold the store; < 0: the device memory free
 * when the store is first allocated, less the kernel-output and
 * measurement buffers and 1 GiB.  When the store does not fit, it is cut
 * into chunks of graph_steps steps (all events) and the device keeps D >= 2
 * chunk slots; during the forward run each chunk that a later chunk will
 * overwrite is copied to pinned host memory on a copy stream, and during
 * the adjoint run it comes back into its slot right after the slot's
 * occupant is replayed, at least one launch ahead of its use.  One
 * cudaMemcpyAsync per chunk (plus one for the FP16 scales).  Fails with
 * SEM_ERR_NOMEM when fewer than 2 slots fit or the pinned host memory
 * cannot be had.  Batched runs (sem_iterate_time) only; changing it drops a
 * saved forward state.  No counterpart for the call itself. */
int sem_set_store_spill(sem_run *run, long long device_store_bytes);
/* Store layout after the first saved forward run: chunk_steps and
 * device_slots are 0 when the whole store is resident; chunks = chunk
 * count; device and pinned host bytes of the store. */
int sem_store_info(sem_run *run, int *chunk_steps, int *device_slots, int *chunks,
                   long long *device_bytes, long long *host_bytes);

/* Average device time in ms of each kernel of one step - forces, stacey,
 * points, update - measured with CUDA events over nsteps further steps of
 * the current state (sim_type 1 or 3 kernels).  Advances the wavefields. */
int sem_time_kernels(sem_run *run, int sim_type, int nsteps, double *ms4);

/* Serving: each event lane of a run is driven on its own.  A lane takes a
 * request (sem_lane_start_forward), advances with every other active lane
 * in the same launches (sem_advance), switches to its adjoint run once its
 * forward is complete (sem_lane_start_adjoint, FP64 L2 measurement on the
 * device) and hands back its results (sem_lane_finish), after which it
 * takes the next request while the others keep running.  Lanes have their
 * own NSTEP (<= the run's nstep) and their own boundary store, allocated
 * stream-ordered when the forward starts and freed when the lane
 * finishes.  No counterpart in the reference, whose driver runs one event
 * per process at a time (src/preproc/fwat_fwd_measure_adj.f90:43-51). */
long long sem_lane_store_bytes(const sem_run *run, int nstep);
int sem_lane_start_forward(sem_run *run, int lane, const sem_source *src,
                           int nrec, const double *xyz, int nstep,
                           int save_forward);
int sem_lane_start_adjoint(sem_run *run, int lane, const double *obs,
                           double taper_pct, int taper_type, double *misfit);
/* Queue nsteps steps for every active lane (lanes that reach their NSTEP
 * stop inside the launches).  Asynchronous. */
int sem_advance(sem_run *run, int nsteps);
/* Completion marks on the run's stream, for a scheduler that keeps work
 * queued on several runs and services whichever finishes first.
 * sem_mark records a mark after everything queued so far and returns its
 * token; sem_mark_done returns 1 once the work before it has finished, 0
 * if not yet (wait = 1 blocks until it has); sem_mark_elapsed gives the
 * device time in ms between two marks still among the last 16.  No
 * counterpart in the reference. */
int sem_mark(sem_run *run, long long *token);
int sem_mark_done(sem_run *run, long long token, int wait);
int sem_mark_elapsed(sem_run *run, long long t0, long long t1, double *ms);
/* phase: 0 idle, 1 forward, 3 adjoint; step: steps done in that phase. */
int sem_lane_status(sem_run *run, int lane, int *phase, int *step,
                    int *nstep);
/* Results of a lane whose phase is complete: forward seismograms
 * [nrec][3][nstep] (forward lanes), kernels [6][nspec][125] to the host
 * and/or added in FP64 into the device array ksum_dev (adjoint lanes).  A
 * forward lane that saved its store stays reserved for its adjoint run;
 * any other lane becomes idle.  Blocks until the copies are done. */
int sem_lane_finish(sem_run *run, int lane, float *seis, double *kernels6,
                    double *ksum_dev);

/* Non-blocking forms for a scheduler that keeps work queued on the run.
 * sem_lane_finish_async queues what sem_lane_finish does (results to the
 * host and/or the FP64 device sum, the lane's store freed stream-ordered)
 * and returns at once; seis / kernels6 should be page-locked host memory
 * (pageable memory makes the copy wait for the queued work), and must not
 * be read before sem_lane_ready(run, lane, 0) returns 1 (wait = 1 blocks
 * until it does).  With check_every > 0 it blocks as sem_lane_finish does.
 * sem_lane_start_adjoint with misfit = NULL does not wait either;
 * sem_lane_misfit then queues the copy of the lane's FP64 misfit to
 * *misfit, readable after sem_lane_ready (at once for pageable memory).
 * No counterpart in the reference. */
int sem_lane_finish_async(sem_run *run, int lane, float *seis, double *kernels6,
                          double *ksum_dev);
/* Lane compaction: move the request on lane `from` (forward or adjoint, any
 * step) to the free lane `to`, so that a scheduler can keep requests packed
 * into few 8-lane groups (each active group costs a share of every step).
 * Its wavefields, kernel accumulators, source, receivers, seismograms,
 * adjoint sources and boundary store go with it; the copies queue behind
 * the work on the run's stream.  Results queued by an earlier async finish
 * of `from` are not affected.  No counterpart in the reference. */
int sem_lane_move(sem_run *run, int from, int to);
int sem_lane_ready(sem_run *run, int lane, int wait);
int sem_lane_misfit(sem_run *run, int lane, double *misfit);

/* Element-kernel variants in use for the forward and adjoint phases
 * (1 thread-per-point, 2 pencil, 3 pencil pipelined, 4 pencil pipelined
 * with 2 events per block, 5 and 6 pencil pipelined with 2 or 4 events
 * per thread, 7 to 10 with the adjoint-phase field pair as a float2,
 * 11 forward with register prefetch, 12 as 11 with colour-ordered
 * non-atomic forward assembly, 13 thread per point with warp-shuffle
 * contractions, 14 as 11 with the three-blocks-per-SM adjoint kernel, 15
 * the five-blocks-per-SM forward kernel with the adjoint kernel of 11).
 * With kernel_variant = 0 the first
 * sem_iterate_time times the candidates on this run and keeps the fastest
 * per phase; -1 until then. */
int sem_kernel_variants(sem_run *run, int *fwd, int *adj);

/* L2 waveform misfit and adjoint sources on caller-owned DEVICE buffers,
 * allocating nothing.  No counterpart in the reference: it is for callers
 * that cannot call cudaMalloc (code inside another framework's memory pool
 * or a fixed device-memory budget, or a Fortran host that only passes
 * buffers it already owns).  Same arithmetic as sem_measure_l2: seis_dev
 * [nrec][3][nstep] float, obs_dev [nrec][3][nstep] double; writes adj_dev
 * [nrec][3][nstep] float and the summed misfit to misfit_dev (one double).
 * Working memory is one static device array per GPU (about 608 KiB, kept
 * until exit) sized for SEM_L2_NOALLOC_MAX_RECEIVERS receivers and
 * SEM_L2_NOALLOC_MAX_STEPS samples; larger requests return SEM_ERR_ARG.
 * Work is queued on `stream` (a cudaStream_t, NULL = legacy default).  The
 * first call on a device (and the first after its context was reset) looks
 * up that array's device address; CUDA loads device code lazily, so that
 * call is also when the array is placed on the GPU, and on a full device
 * it returns SEM_ERR_CUDA.  Make one small call at start-up, before a
 * fixed budget applies and before capturing the stream into a CUDA graph.
 * All calls share the array: calls that overlap on the GPU race and must
 * not be issued. */
#define SEM_L2_NOALLOC_MAX_RECEIVERS 4096
#define SEM_L2_NOALLOC_MAX_STEPS 32768
int sem_measure_l2_noalloc(const float *seis_dev, const double *obs_dev,
                           int nrec, int nstep, double dt, double taper_pct,
                           int taper_type, float *adj_dev, double *misfit_dev,
                           void *stream);

/* ------------------------------------------------------------------------
 * Waveform measurement with the reference's pre-processing, on the device.
 *
 * Replaces LEQData%measure_adj for the waveform (L2) misfit
 * (src/preproc/leq_data.f90:48-188) with one window per trace and band,
 * the window types whose windows are given by formula (group velocity,
 * arrival time; leq_data.f90:132-146): observed traces are interpolated
 * onto the synthetic axis, detrended, demeaned, Hann-tapered (pre_taper)
 * and band-passed; synthetics are rotated to Z,R,T (rotate = 1), tapered
 * and band-passed; the window's L2 misfit and adjoint source follow
 * waveform_misfit.f90:15-64 and filter_adj (adjoint_source.f90:92-114);
 * bands are summed (or normalised, ADJ_SRC_NORM) and rotated back to
 * E,N,Z (noise_data.f90:213-252).  The Butterworth band-pass is xapiir's
 * design (order, passes as IORD, PASSES) computed and applied in FP64; the
 * reference runs it in FP32.
 *
 * Arrays: obs [nrec][3][obs_npts] FP64 (components Z,R,T when rotate,
 * else x=E,y=N,z=Z); windows [max(nband,1)][nrec][3][2] start/end in
 * origin time (s); baz [nrec] back-azimuth in degrees (rotate only).
 * ------------------------------------------------------------------------ */
#define SEM_MEAS_MAX_BANDS 4

typedef struct {
  double t0;               /* the synthetic record starts at -t0 (s)           */
  double obs_tbeg;         /* time of the first observed sample (s)            */
  double obs_dt;           /* observed sampling interval (s)                   */
  int obs_npts;            /* observed samples per trace                       */
  int nband;               /* band-pass filters, 0 (none) .. SEM_MEAS_MAX_BANDS */
  double short_p[SEM_MEAS_MAX_BANDS]; /* SHORT_P per band (s)                  */
  double long_p[SEM_MEAS_MAX_BANDS];  /* LONG_P per band (s)                   */
  int order;               /* Butterworth order IORD (reference: 2)            */
  int passes;              /* 1 or 2 (reference PASSES: 2, zero phase)         */
  double pre_taper;        /* taper_per of whole traces (reference: 0.1)       */
  double win_taper;        /* taper_percentage of the windows                  */
  int win_taper_type;      /* itaper_type, 1..4                                */
  double weight;           /* src_weight of the event                          */
  int rotate;              /* 1: obs and windows are Z,R,T; needs baz          */
  int adj_norm;            /* ADJ_SRC_NORM across bands                        */
} sem_meas_cfg;

/* Run form: measures event ev's resident seismograms (after
 * sem_iterate_time(run, 1, 1)) and leaves the adjoint source on the device
 * for sem_iterate_time(run, 3, 0).  misfit_band [max(nband,1)] and
 * misfit_trace [max(nband,1)][nrec][3] (host, either may be NULL).
 * No reference counterpart for the exact signature: it bundles
 * measure_adj's per-trace loop for one event. */
int sem_measure_waveform(sem_run *run, int ev, const sem_meas_cfg *cfg,
                         const double *obs, const double *windows,
                         const double *baz, double *misfit_band,
                         double *misfit_trace);

/* Device-buffer form on caller-owned device memory: seis [nrec][3][nstep]
 * FP32 (x,y,z), adj out [nrec][3][nstep] FP32, misfit_trace out
 * [max(nband,1)][nrec][3] FP64 (NaN for a window outside the record).
 * Asynchronous on `stream`; allocates its scratch stream-ordered. */
int sem_measure_waveform_dev(const float *seis_dev, int nrec, int nstep, double dt,
                             const sem_meas_cfg *cfg, const double *obs_dev,
                             const double *windows_dev, const double *baz_dev,
                             float *adj_dev, double *misfit_trace_dev, void *stream);

/* ------------------------------------------------------------------------
 * Kernel post-processing: PDE smoothing of element fields.
 *
 * Replaces smooth_sem_pde (src/postproc/smooth.f90:7-437), called from
 * PostFlow%pde_smooth and %sum_precond (src/postproc/post_processing.f90:
 * 222,270), and its GPU form smooth_pde_cuda_ (src/postproc/
 * smooth_sem_pde.cu:298-478).  Each field (a kernel or Hessian,
 * dat(NGLLX,NGLLY,NGLLZ,NSPEC)) is projected onto the global points, then
 * diffused for nstep explicit steps with horizontal/vertical coefficients
 * ch/cv, and gathered back.  cmax = distance_min^2/9; the larger of
 * sigma_h, sigma_v gets cmax and the other cmax*(sigma_small/sigma_large)^2;
 * nstep = ceiling(max(sigma)^2 / (2 cmax)) (smooth.f90:99-109).  Points of
 * CPML elements are held at 0 (ZERO_PML).
 *
 * mapping: SEM_SMOOTH_MAP_CUBE uses the regular element's diagonal mapping
 * (xix = etay = gammaz = xix_regular).  SEM_SMOOTH_MAP_REFERENCE reproduces
 * the reference's regular-element branch as written, which sets all nine
 * mapping terms to xix_regular (smooth.f90:269-279): a diffusion along
 * (1,1,1) that exceeds the step-size bound and grows without limit within
 * tens of steps.  It exists for parity checks.
 * ------------------------------------------------------------------------ */
#define SEM_SMOOTH_MAP_CUBE 0
#define SEM_SMOOTH_MAP_REFERENCE 1

typedef struct {
  double sigma_h, sigma_v; /* smoothing lengths (mesh units)                 */
  double distance_min;     /* minimum GLL point distance (distance_min_glob);
                              <= 0: (xi_1 - xi_0)/xix_regular of the mesh  */
  int is_sph;              /* 1: vertical = radial r = x/|x| (spherical)     */
  int mapping;             /* SEM_SMOOTH_MAP_CUBE or SEM_SMOOTH_MAP_REFERENCE */
  int nstep;               /* > 0 replaces the computed step count           */
} sem_smooth_cfg;

typedef struct {
  int nstep;               /* steps taken                                    */
  int fields_per_pass;     /* fields smoothed together on the device (1/2/4) */
  double cv, ch;           /* diffusion coefficients (FP32 values)           */
  double distance_min;     /* the distance used                              */
  double step_ms;          /* device time of the diffusion steps (all passes)*/
} sem_smooth_stats;

/* dat_in, dat_out: host [nfield][nspec][125] FP32 (Fortran dat order);
 * is_cpml: [nspec] or NULL; stats may be NULL.  Blocking. */
int sem_smooth_pde(sem_mesh *mesh, const sem_smooth_cfg *cfg, int nfield,
                   const float *dat_in, const int *is_cpml, float *dat_out,
                   sem_smooth_stats *stats);

/* Incident wavefield injected on the absorbing faces of event ev's
 * forward run: FK injection (COUPLE_WITH_INJECTION_TECHNIQUE with
 * INJECTION_TECHNIQUE_TYPE 3, prepare_timerun_fwat.f90:104-117), fed with
 * the arrays read_fk_coupling_file loads (src/shared/fk_coupling.f90:396-439).
 * veloc, tract: [nt][nf*25][3] FP32, the reference's Veloc_FK and
 * Tract_FK(NDIM, npt, k0 : k0+nt-1) with npt ordered face by face as
 * ipt_table (fk_coupling.f90:299-327); sample k is at time
 * k * np_resamp * DT (the reference uses k0 = -NP_RESAMP).  Step it takes
 * the 4-point Lagrange interpolant at it / np_resamp (the sample itself
 * when np_resamp divides it).  The absorbing term becomes
 *     accel -= (Stacey(v - veloc) - tract) * jacobian2Dw
 * with tract = sigma . n for the outward normal; the boundary store saves
 * that term, so the backward reconstruction replays it.  An event with an
 * injection needs no point source.  veloc = NULL removes it.  Batched runs
 * (sem_iterate_time) only.  Setting the first injection or removing the last
 * one drops the run's captured step graphs, so that the next run of each
 * phase captures the matching kernels. */
int sem_set_injection(sem_run *run, int ev, const float *veloc, const float *tract, int nt,
                      int np_resamp, int k0);

/* Approximate Hessian kernel (SPECFEM's APPROXIMATE_HESS_KL, read by
 * PostFlow%sum_precond / apply_precond as hess_kernel,
 * src/postproc/post_processing.f90:164-230).  Enabled before a
 * sim_type 3 run, the adjoint run also accumulates per GLL point
 *     hess = 2 * sum_it DT * (adjoint accel . backward accel).
 * Batched runs (sem_iterate_time) only; lanes driven by sem_lane_* do not
 * hand it back.  Costs 8 bytes per point and event and step.  Changing the
 * switch drops the run's captured step graphs (recaptured at the next run). */
int sem_set_approximate_hessian(sem_run *run, int enable);
/* hess_kernel of event ev: out[nspec][125]. */
int sem_save_hessian_kernel(sem_run *run, int ev, double *out);
/* FP64 sum over the run's events of hess (abs_each = 0) or |hess| (1):
 * out[nspec][125]. */
int sem_sum_hessian(sem_run *run, int abs_each, double *out);

/* Preconditioner of PostFlow%apply_precond (post_processing.f90:164-197)
 * from the event-summed Hessian (n values; sem_sum_hessian over all
 * batches): precond_type 1 takes hess_sum = sum |hess|, 0 takes
 * |sum hess|; then invert_hess (post_processing.f90:333-372): normalise by
 * the maximum (all ones when it is below 1e-18), invert with
 * THRESHOLD_HESS = 1e-3, normalise by the maximum.  The kernels are
 * multiplied by precond.  Computed on the device in FP64; precond FP32. */
int sem_hessian_precond(const double *hess_sum, long long n, int precond_type,
                        float *precond);
/* Depth preconditioner zprecond_gll (src/postproc/zprecond.f90:11-71),
 * precond_type 2 (1/|z|) or 3 (1/sqrt|z|): the profile on the model
 * grid's depth levels zlev[nz] (strictly ascending; z = 1e-8 above the
 * surface, z + 1e-8 below), linearly interpolated to the GLL points'
 * z, times nevents, normalised, inverted, normalised.  Points outside
 * [zlev[0], zlev[nz-1]] take the end values.  precond[nspec][125]. */
int sem_depth_precond(sem_mesh *mesh, const double *zlev, int nz, int precond_type,
                      int nevents, float *precond);

/* Regular model grid of the kernels: points x0[d] + i h[d], i < n[d],
 * grid arrays [nx][ny][nz] (z fastest, the C view of the reference's
 * Fortran (nz, ny, nx) arrays).  ngnod: anchor nodes of the mesher's
 * elements (8 or 27), used to locate grid points in irregular elements. */
typedef struct {
  double x0[3];
  double h[3];
  int n[3];
  int ngnod;
} sem_grid_desc;

/* Projection of element fields onto the grid (gll2grid), on the device in
 * FP64: a grid point belongs to the first element (lowest index) whose
 * candidate index range, from its GLL points' bounding box with the
 * reference's truncation, holds it; its value is that element's 5x5x5
 * Lagrange interpolant at the point's reference coordinates, clamped to
 * [-1, 1] (affine elements: linear in the box; irregular elements: the
 * reference locator's start at the nearest interior GLL node and four
 * Newton steps on the anchor nodes).  Points no element takes are 0.
 * fields[nfield][nspec][125] FP32, out[nfield][nx][ny][nz] FP32. */
int sem_grid_project(sem_mesh *mesh, const sem_grid_desc *grid, int nfield,
                     const float *fields, float *out);

/* Taper widths of taper_kernel_grid (m): zero for *_suppress from the
 * sides (h) and the bottom (v), a half cosine over the next *_buffer,
 * one inside; no taper at the surface. */
typedef struct {
  double h_suppress, h_buffer, v_suppress, v_buffer;
} sem_grid_taper_cfg;

/* taper_kernel_grid on the device: the mask lives on a grid of spacing
 * (smallest + largest GLL point distance) / 2 over the mesh's extent and is
 * interpolated trilinearly at the grid points (0 outside its box);
 * grid_fields[nfield][nx][ny][nz] are multiplied by it in place, and mask
 * (may be null) receives it [nx][ny][nz] in FP64.  nfield may be 0 when
 * mask is given.  Widths beyond half the mesh are refused (SEM_ERR_ARG). */
int sem_grid_taper(sem_mesh *mesh, const sem_grid_desc *grid, const sem_grid_taper_cfg *taper,
                   int nfield, float *grid_fields, double *mask);

/* zprecond_grid on the device: the depth preconditioner, precond_type 2
 * (1/|z|) or 3 (1/sqrt|z|), of the levels zlev[nz] (NULL: the grid's
 * x0[2] + k h[2]) for nevents events, normalised, inverted, normalised,
 * repeated over x and y: out[nx][ny][nz] FP32. */
int sem_grid_zprecond(const sem_grid_desc *grid, const double *zlev, int precond_type,
                      int nevents, float *out);

/* FP32 FMA throughput of the current device in TFLOP/s (an FMA counts
 * as 2 flops), the best of 5 timed launches of independent fmaf chains on
 * every SM; *ms (may be null) is that launch's time.  No reference
 * counterpart: it is the denominator of the element kernels' FP32
 * roofline fraction. */
int sem_fp32_fma_peak(double *tflops, double *ms);

/* Device-time of the last sem_iterate_time in milliseconds. */
int sem_last_loop_ms(sem_run *run, double *ms);
/* Number of kernel launches queued by the last sem_iterate_time. */
int sem_last_launch_count(sem_run *run, long long *count);

#ifdef __cplusplus
}
#endif
#endif /* SEM_B200_H */
