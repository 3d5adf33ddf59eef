/*
 * surfatt_gpu.h -- C ABI of the B200 engine for SurfATTPP's forward + adjoint
 * misfit-gradient hot path (libsurfatt_gpu.so).
 *
 * Plain pointers and sizes only.  Every entry point returns an sa_status code
 * (0 = success); the reference's exceptions and Fortran `stop` become codes,
 * and the adapter layer turns them back into the reference's behaviour.
 * Per-call diagnostics are available from sa_ctx_error().
 *
 * Array layout (same as the reference):
 *   2-D surface fields: Eigen column-major nx x ny, index ix + nx*iy.
 *   Per-period media:   [iper][iy][ix] planes (one nx*ny plane per period).
 *   3-D model fields:   (nx, ny, nz) row-major, as ModelGrid::vs3d_loc.
 *   Depth kernels:      (nx, ny, nz, nper) row-major, nper fastest, as
 *                       SurfGrid::sen_vs_loc (src/surf_grid.cpp:3-8).
 *   Events:             one per (source, period) as SrcRec::events_local;
 *                       receivers in CSR form rec_ptr[ne+1] / rec_idx[].
 *
 * Precision: SA_FP64 reproduces the reference's FP64 arithmetic (parity
 * path); SA_FP32 sweeps in FP32 with FP64 T0, travel times, residuals,
 * adjoint coefficients and accumulation.
 */
#ifndef SURFATT_GPU_H
#define SURFATT_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sa_ctx sa_ctx;
typedef struct sa_plan sa_plan;

enum sa_status {
    SA_OK = 0,
    SA_ERR_ARG = 1,        /* invalid argument (reference: std::invalid_argument / runtime_error) */
    SA_ERR_CUDA = 2,       /* CUDA runtime failure */
    SA_ERR_NOCONV = 3,     /* a sweep hit its iteration cap (reference: stderr warning) */
    SA_ERR_NOROOT = 4,     /* dispersion root not found (reference: stop 'Dispersion calculation failed') */
    SA_ERR_NONFINITE = 5,  /* NaN/Inf in an output field */
    SA_ERR_NOMEM = 6,      /* device allocation failed */
    SA_ERR_TEAM = 7        /* a cooperative sweep's wait gave up (FP32 tail teams; no reference counterpart) */
};

enum sa_precision { SA_FP64 = 0, SA_FP32 = 1 };

/* ---- context -------------------------------------------------------------- */
/* Binds a CUDA device, a stream and a grow-only pool of device scratch. */
int sa_ctx_create(int device, sa_ctx** out);
void sa_ctx_destroy(sa_ctx* ctx);
const char* sa_ctx_error(const sa_ctx* ctx);
int sa_version(void);

/* ---- eikonal:: drop-ins (host arrays, one solve) --------------------------- */

/* Replaces eikonal::FSM_UW_PS_lonlat_2d (reference include/eikonal_solver.h:32-40,
 * src/eikonal_solver.cpp:22-318).  spha/sphb/sphc/fun/T_out: nx*ny.
 * niter (may be NULL) receives the number of sweep iterations. */
int sa_eik_fwd_field(sa_ctx* ctx, int precision, int nx, int ny, const double* xx_deg,
                     const double* yy_deg, const double* spha, const double* sphb,
                     const double* sphc, const double* fun, double x0_deg, double y0_deg,
                     double* T_out, int* niter);

/* Replaces eikonal::FSM_O1_JSE_lonlat_2d (reference include/eikonal_solver.h:74-83,
 * src/eikonal_solver.cpp:323-511).  Ta_out is unmasked, zero on the boundary. */
int sa_eik_adj_field(sa_ctx* ctx, int precision, int nx, int ny, const double* xx_deg,
                     const double* yy_deg, const double* spha, const double* sphb,
                     const double* sphc, const double* T, int nr, const double* xrec_deg,
                     const double* yrec_deg, const double* source_adj, double* Ta_out,
                     int* niter);

/* Replaces eikonal::mask_uniform_grid (reference include/eikonal_solver.h:85-89,
 * src/eikonal_solver.cpp:514-536) on a host field. */
int sa_mask_uniform_grid(int nx, int ny, const double* xx, const double* yy, double* table,
                         double x0, double y0);

/* ---- preproc::forward_for_event (batched) ---------------------------------- */

/* A plan fixes the surface grid, the periods count and the event set
 * (reference SrcRec::events_local, src/src_rec.cpp:138-228): unique sources,
 * great-circle geometry per source and the scratch pool are built once and
 * reused by every sa_plan_forward_adjoint() call (one per misfit evaluation).
 * All arrays are host arrays; evlo/evla/stlo/stla in degrees. */
int sa_plan_create(sa_ctx* ctx, int precision, int nx, int ny, int nper, const double* xx_deg,
                   const double* yy_deg, int ne, const double* evlo, const double* evla,
                   const int* iper, const int* rec_ptr, const int* rec_idx, int nsta,
                   const double* stlo, const double* stla, sa_plan** out);
void sa_plan_destroy(sa_plan* plan);

/* Replay the whole misfit evaluation as one CUDA graph when the argument
 * pointers repeat (default on). */
int sa_plan_set_graph(sa_plan* plan, int enable);

/* Deterministic accumulation of adj_s and the misfit (default off): the
 * reference adds every event's masked Ta * svel^-3 plane to adj_s and its
 * misfit to chi in event order (src/preproc.cpp:28-31, :142, one MPI rank).
 * Enabled, each event writes its plane to a buffer and an ordered reduction
 * adds the planes in event order, so adj_s and chi are reproducible bit for
 * bit (FP64 plans: equal to the reference's single-rank sums) instead of
 * being summed with atomics in completion order.  Events then run in chunks
 * whose planes fit max_bytes of device memory (0 = a quarter of the free
 * memory). */
int sa_plan_set_deterministic(sa_plan* plan, int enable, size_t max_bytes);

/* The adjoint a plan computes.  kind 0 (default): the reference's
 * (eikonal::FSM_O1_JSE_lonlat_2d, src/eikonal_solver.cpp:323-511) with the
 * reference's forward stopping rule.  kind 1 (FP64 plans; no reference
 * counterpart): forward solves run to a fixed point (an iteration that
 * changes no cell) and the adjoint is the exact discrete adjoint of the
 * forward solve -- the derivative of the receiver times the plan computes,
 * including the source's slowness -- so adj_s receives dchi/dsvel (per
 * period plane) instead of the accumulated Ta svel^-3; is_kden is not
 * computed.  sa_grad_run then chains adj_s with the derivatives of
 * surfdisp96's phase-velocity roots (Rayleigh phase data), and
 * sa_grad_vjp takes convention 2.  SA_ERR_ARG for an FP32 plan. */
int sa_plan_set_adjoint(sa_plan* plan, int kind);

/* is_kden on a plan: while kden_s (device, [nper][ny][nx]) is set, every
 * evaluation with the adjoint also solves the kernel-density adjoint
 * (src/preproc.cpp:128-137) and overwrites kden_s with its accumulation
 * (accumulate_kernels, :32-34).  NULL turns it off. */
int sa_plan_kden_output(sa_plan* plan, double* kden_s);

/* One forward (+ adjoint) evaluation of every event of the plan: replaces
 * preproc::forward_for_event (reference include/preproc.h:14,
 * src/preproc.cpp:71-148) with accumulate_kernels (:19-34), isotropic
 * branch, is_kden = false.
 *   svel           [nper][ny][nx] phase/group velocity (device)
 *   m11, m12, m22  [nper][ny][nx] media (device) or all NULL for the flat
 *                  isotropic surface (m11 = m22 = 1, m12 = -0, reference
 *                  src/surf_grid.cpp:178-190)
 *   tt_obs, weight [npair] observed times and weights (device)
 * Outputs (device, any may be NULL unless required):
 *   syn [npair]; adj_s [nper][ny][nx] (overwritten, FP64); chi (1 double,
 *   0.5*sum w r^2 over all events); fwd_iters/adj_iters/status [ne].
 *   stream: a cudaStream_t, or NULL for the context's stream.
 * Returns SA_ERR_NOCONV / SA_ERR_NONFINITE when any event reports it. */
int sa_plan_forward_adjoint(sa_plan* plan, const double* svel, const double* m11,
                            const double* m12, const double* m22, const double* tt_obs,
                            const double* weight, int calc_adj, double* syn, double* adj_s,
                            double* chi, int* fwd_iters, int* adj_iters, int* status,
                            void* stream);

/* preproc::forward_for_event (reference src/preproc.cpp:71-148) with the
 * adjoint source given by the caller instead of the residuals w*(Tsyn - Tobs)
 * (:111-127): per receiver source_adj [npair] (device).  Every forward field
 * is recomputed, the adjoint solved with that source, masked and accumulated
 * into adj_s [nper][ny][nx] (overwritten), i.e. the reference's adjoint
 * applied to an arbitrary vector on the receiver times -- the
 * vector-Jacobian product used by an autograd backward.  syn [npair] and
 * status [ne] may be NULL; no misfit is formed. */
int sa_plan_adjoint_source(sa_plan* plan, const double* svel, const double* m11,
                           const double* m12, const double* m22, const double* source_adj,
                           double* syn, double* adj_s, int* status, void* stream);

/* Host-array convenience over a transient plan (uploads, runs, downloads):
 * the drop-in for one call of preproc::forward_for_event. */
int sa_forward_for_events(sa_ctx* ctx, int precision, int nx, int ny, int nper,
                          const double* xx_deg, const double* yy_deg, const double* svel,
                          const double* m11, const double* m12, const double* m22, int ne,
                          const double* evlo, const double* evla, const int* iper,
                          const int* rec_ptr, const int* rec_idx, int nsta, const double* stlo,
                          const double* stla, const double* tt_obs, const double* weight,
                          int calc_adj, double* syn, double* adj_s, double* chi, int* fwd_iters,
                          int* adj_iters);

/* No counterpart in the reference, which has no GPU launch to configure.
 * Autotunes this plan's batch-kernel launch on its own workload: every
 * candidate configuration -- for FP32 plans the forward sweep step rolled or
 * unrolled times the adjoint sweep loading 2 or 3 steps ahead times tail
 * teams on or off, for either precision all or three quarters of the resident
 * event slots, with tail teams also a quarter (one solve per block) -- runs
 * the plan's evaluation (arguments as sa_plan_forward_adjoint; adj_s may be
 * NULL) twice and its second batch launch is timed.  The fastest is kept by
 * the plan and by plans of the same grid size (nx, ny, precision) created
 * later on this context.  ms_out (may be NULL) receives up to
 * SA_TUNE_MAX_CANDIDATES timings, n_out the number of candidates, choice the
 * index of the one kept.  Outputs do not depend on the configuration (FP32:
 * every variant rounds the same explicit operations; adj_s up to the order
 * of its FP64 atomic sums).  Synchronises `stream`. */
#define SA_TUNE_MAX_CANDIDATES 32
int sa_plan_autotune(sa_plan* plan, const double* svel, const double* m11, const double* m12,
                     const double* m22, const double* tt_obs, const double* weight,
                     int calc_adj, double* adj_s, float* ms_out, int* n_out, int* choice,
                     void* stream);

/* The plan's launch configuration: variant (0-7 for FP32, bit 0 = unrolled
 * forward step, bit 1 = adjoint lead 3, bit 2 = tail teams: warps whose
 * queue pull finds no event left join the solves still running in their
 * block; 0 for FP64), event slots in use (set: 0 = all; more than allocated =
 * all; with tail teams the other resident warps start as team members), and
 * slots allocated.  Setting it (e.g. a configuration tuned in an earlier run)
 * affects this plan only. */
int sa_plan_set_tune(sa_plan* plan, int variant, int active_slots);
int sa_plan_get_tune(sa_plan* plan, int* variant, int* active_slots, int* nslots);

/* Timing of the batch kernel (no counterpart in the reference).  While
 * enabled, sa_plan_forward_adjoint launches without the graph and records CUDA
 * events on its stream around the batched forward/adjoint kernel;
 * sa_plan_kernel_ms waits for the last of them and returns its duration. */
int sa_plan_kernel_timing(sa_plan* plan, int enable);
int sa_plan_kernel_ms(sa_plan* plan, float* ms);

/* Full-field outputs for testing (device arrays [ne][ny][nx], may be NULL):
 * forward T and the masked adjoint field of the next sa_plan_forward_adjoint. */
int sa_plan_debug_fields(sa_plan* plan, double* T_out, double* Ta_out);


/* ---- one launch over several grids ---------------------------------------- */

/* No counterpart in the reference, which solves each grid's events in its
 * own loop.  Binds plans of one context and precision -- e.g. the levels of
 * a multi-grid topography batch, 101^2, 201^2 and 401^2 -- so that one
 * persistent launch solves every plan's events: each queue entry names its
 * plan (grid, media, geometry, outputs), scratch slots are sized for the
 * largest grid, and the queue is ordered by the previous evaluation's work
 * (sweeps x cells) across plans, longest first.  Results equal each plan's
 * own sa_plan_forward_adjoint (adj_s to the order of its FP64 atomics). */
typedef struct sa_multi sa_multi;
int sa_multi_create(sa_plan* const* plans, int nplans, sa_multi** out);
void sa_multi_destroy(sa_multi* multi);

/* One evaluation of every plan's events in one launch: the arguments of
 * sa_plan_forward_adjoint, one pointer per plan (m11/m12/m22 NULL or set for
 * every plan; syn, adj_s, chi, status may be NULL or hold NULL entries).
 * The first plan's FP32 launch variant applies to all.  Enqueued on
 * `stream` (NULL = the context's stream). */
int sa_multi_forward_adjoint(sa_multi* multi, const double* const* svel, const double* const* m11,
                             const double* const* m12, const double* const* m22,
                             const double* const* tt_obs, const double* const* weight,
                             int calc_adj, double* const* syn, double* const* adj_s,
                             double* const* chi, int* const* status, void* stream);
/* Device time of the last evaluation's batch launch (waits for it). */
int sa_multi_kernel_ms(sa_multi* multi, float* ms);
/* The worst event status of the last evaluation over all plans (synchronous). */
int sa_multi_status(sa_multi* multi, int* worst);

/* ---- surfker:: and preproc::combine_kernels (device arrays) --------------- */

/* Replaces the column loop of SurfGrid::fwdsurf (reference
 * src/surf_grid.cpp:194-245), i.e. build_disp_req (src/surfdisp.cpp:60-108)
 * with the Brocher Vp/rho relations and surfker::surfdisp -> surfdisp96_c
 * (src/surfdisp.cpp:428-462, src/surfker/surfdisp96.f:57-373), spherical
 * earth (IFLSPH = 1), fundamental mode.  One thread per column.
 *   zgrid [nz] (host), periods [nper] (host, nper <= 64), nz + 1 <= 64
 *   vs3d  (nx, ny, nz) row-major (device)
 *   svel  [nper][ny][nx] (device out); status [ny][nx] (device, may be NULL):
 *         1 where the root search failed (the Fortran's `stop`). */
int sa_surfdisp_columns(sa_ctx* ctx, int nx, int ny, int nz, const double* zgrid,
                        const double* vs3d, int nper, const double* periods, int iwave, int igr,
                        double* svel, int* status, void* stream);

/* Replaces the column loop of SurfGrid::compute_dispersion_kernel for phase
 * velocity (src/surf_grid.cpp:247-305) through surfker::depthkernelHTI1d
 * (src/surfdisp.cpp:481-547) and sregn96_hti_c (src/surfker/sregn96.f90:1745-1849).
 * One thread per (column, period).
 *   cp [nper][ny][nx] Rayleigh phase velocities from sa_surfdisp_columns(igr = 0)
 *   sen_vs, sen_vp, sen_rho (nx, ny, nz, nper) row-major (device out). */
int sa_depthkernel_columns(sa_ctx* ctx, int nx, int ny, int nz, const double* zgrid,
                           const double* vs3d, int nper, const double* periods,
                           const double* cp, double* sen_vs, double* sen_vp, double* sen_rho,
                           void* stream);

/* Replaces the column loop of SurfGrid::compute_dispersion_kernel for group
 * velocity (src/surf_grid.cpp:247-305, itype 1) through
 * surfker::depthkernel_rayleigh_group (src/surfdisp.cpp:203-285) and sregnpu
 * (src/surfker/sregn96.f90:1851-1992): phase velocities at t and t(1 +- 0.005)
 * (three surfdisp96 runs per column), then per (column, period) the group
 * kernels dU/dvs, dU/dvp, dU/drho.  sen_* (device) (nx, ny, nz, nper);
 * status (HOST, ny*nx ints, may be NULL): nonzero where a root search failed;
 * the call then returns SA_ERR_NOROOT.  Synchronous on `stream`. */
int sa_depthkernel_columns_group(sa_ctx* ctx, int nx, int ny, int nz, const double* zgrid,
                                 const double* vs3d, int nper, const double* periods,
                                 double* sen_vs, double* sen_vp, double* sen_rho, int* status,
                                 void* stream);

/* Replaces the column loop of SurfGrid::compute_dispersion_kernel for Love
 * waves: surfker::depthkernel_love_phase (igr 0, src/surfdisp.cpp:295-349,
 * slegn96 src/surfker/slegn96.f90:672-783) and depthkernel_love_group
 * (igr 1, src/surfdisp.cpp:351-426, slegnpu :785-919): Love phase velocities
 * (surfdisp96, iwave 1) at t (and t(1 +- 0.005)) per column, then per
 * (column, period) sen_vs = dc/db (du/db) and sen_rho = dc/drho (du/drho)
 * (device, (nx, ny, nz, nper)); Love waves have no vp kernel.  status (HOST,
 * ny*nx, may be NULL) as sa_depthkernel_columns_group.  Synchronous. */
int sa_depthkernel_columns_love(sa_ctx* ctx, int nx, int ny, int nz, const double* zgrid,
                                const double* vs3d, int nper, const double* periods, int igr,
                                double* sen_vs, double* sen_rho, int* status, void* stream);

/* Replaces preproc::combine_kernels, vs-only parametrisation
 * (src/preproc.cpp:276-304): ker_vs(ix,iy,k) = -sum_iper adj_s(iper,ix,iy) *
 * (sen_vs + sen_vp*dVp/dVs + sen_rho*drho/dVp*dVp/dVs), periods in order.
 *   adj_s [nper][ny][nx]; vs3d, vp3d, ker_vs (nx, ny, nz); sen_* (nx, ny, nz, nper).
 *   vp3d may be NULL: vp = vs2vp(vs3d) (Brocher, include/utils.h:237-245). */
int sa_combine_kernels_vs(sa_ctx* ctx, int nx, int ny, int nz, int nper, const double* adj_s,
                          const double* vs3d, const double* vp3d, const double* sen_vs,
                          const double* sen_vp, const double* sen_rho, double* ker_vs,
                          void* stream);

/* ---- PostProc::pde_smooth ------------------------------------------------- */

/* Step count and per-step diffusion coefficients of PostProc::pde_smooth
 * (reference src/postproc.cpp:394-434): nstep, ch (deg^2), cv (km^2).
 * ygrid[ny] latitudes in degrees (only the first and last are used).
 * Host arithmetic only.  SA_ERR_ARG for non-positive sigma or too fine a grid
 * (the reference logs an error and aborts). */
int sa_pde_smooth_nstep(int ny, double dx_deg, double dy_deg, double dz_km, const double* ygrid,
                        double sigma_h, double sigma_v, int* nstep, double* ch, double* cv);

/* Replaces PostProc::pde_smooth (src/postproc.cpp:388-463) on one rank:
 * nstep explicit Euler steps of the spherical Laplacian (:35-128) with the
 * Neumann boundary copies (:130-158).  field (device, in/out): (nx, ny, nz)
 * row-major, depth fastest (Tensor3r); work: device scratch of nx*ny*nz
 * doubles, or NULL to allocate one for the call.  ygrid[ny] (degrees) and
 * zgrid[nz] (km) are host arrays; dx_deg, dy_deg, dz_km the grid intervals.
 * nstep_out (host, may be NULL) receives the step count.  Returns after the
 * smoothing has completed on `stream` (NULL = the context's stream). */
int sa_pde_smooth(sa_ctx* ctx, int nx, int ny, int nz, double dx_deg, double dy_deg,
                  double dz_km, const double* ygrid, const double* zgrid, double sigma_h,
                  double sigma_v, double* field, double* work, int* nstep_out, void* stream);

/* Multigrid smoothing, the reference's smooth_method 1
 * (PostProc::InvGrid::init / fwd2inv / inv2fwd, src/postproc.cpp:160-386;
 * PostProc::smooth, :465-480): nset staggered coarse grids of n_inv[0..2] +
 * 2 nodes over the model grid x[nx] (deg), y[ny] (deg), z[nz] (km) (host
 * arrays); sa_multigrid_smooth projects a (nx, ny, nz) row-major device field
 * onto them and interpolates back, averaged over the sets, into out (device,
 * not aliasing field).  As the reference computes it: the projection adds
 * each fine node to a single corner, and the coarse index uses the inner
 * counts as strides.  Equal bit for bit to a CPU evaluation.  SA_ERR_ARG when
 * a node lies outside a coarse grid (the reference aborts). */
typedef struct sa_multigrid sa_multigrid;
int sa_multigrid_create(int device, int nx, int ny, int nz, const double* x, const double* y,
                        const double* z, const int* n_inv, int nset, sa_multigrid** out);
void sa_multigrid_destroy(sa_multigrid* mg);
int sa_multigrid_smooth(sa_multigrid* mg, const double* field, double* out, void* stream);

/* ---- observation table and event builder (host only) ----------------------- */

/* SrcRec::load with get_periods and get_events (reference src/src_rec.cpp:20-228,
 * :232-264): reads the CSV (columns tt, staname, stla, stlo, evtname, evla,
 * evlo, period, optional weight / dist / vel, which default to 1, the
 * great-circle distance (include/utils.h:287-299) and dist / tt), builds the
 * sorted unique periods with their mean velocities and one event per
 * (evtname, period) holding its observation rows, ordered as the reference's
 * events map ("{evtname}_{iper}" keys).  The event arrays feed
 * sa_plan_create with the per-observation station coordinates as stations
 * (rec_idx = observation rows).  SA_ERR_ARG for a missing file or column. */
typedef struct sa_srcrec sa_srcrec;
int sa_srcrec_load(const char* csv_path, sa_srcrec** out);
void sa_srcrec_destroy(sa_srcrec* sr);
int sa_srcrec_sizes(const sa_srcrec* sr, int* n_obs, int* nperiod, int* n_events);
int sa_srcrec_periods(const sa_srcrec* sr, double* periods, double* meanvel,
                      int* n_obs_per_period);
int sa_srcrec_observations(const sa_srcrec* sr, double* stlo, double* stla, double* tt,
                           double* weight, double* dist, double* vel, double* period);
/* evlo, evla, iper [n_events]; rec_ptr [n_events + 1]; rec_idx [rec_ptr[n_events]]. */
int sa_srcrec_events(const sa_srcrec* sr, double* evlo, double* evla, int* iper, int* rec_ptr,
                     int* rec_idx);
const char* sa_srcrec_event_name(const sa_srcrec* sr, int event);
/* SrcRec::write (src/src_rec.cpp:407-457): the observed table, or with
 * tt_fwd[n_obs] the forward times and dist / tt_fwd velocities
 * (gather_syn_tt, :326-371). */
int sa_srcrec_write(const sa_srcrec* sr, const char* csv_path, const double* tt_fwd);

/* ---- topography media (config with topography) ----------------------------- */

/* Topography::grid (reference src/topo.cpp:46-95): interp2d of a raw
 * topography z_raw (column-major nx_raw x ny_raw, km; host) onto the model
 * grid x[nx], y[ny] (host) -> z_out (device, column-major nx x ny).
 * SA_ERR_ARG when the model grid extends beyond the topography (the
 * reference aborts). */
int sa_grid_topography(sa_ctx* ctx, int nx_raw, int ny_raw, const double* lon_raw,
                       const double* lat_raw, const double* z_raw, int nx, int ny,
                       const double* x, const double* y, double* z_out);

/* The per-period loop of SurfGrid::build_media_matrix_with_topo
 * (src/surf_grid.cpp:80-166): for each period, gaussian_smooth_geo_2 of the
 * gridded topography with sigma_deg[iper] (include/utils.h:505-571), its
 * geographic gradient (gradient_2_geo, :593-649), the dip angle
 * (src/topo.cpp:97-114) and the media m11 = a, m12 = -c, m22 = b
 * (src/surf_grid.cpp:185-190).  z_gridded (device, column-major nx x ny);
 * lon[nx], lat[ny], sigma_deg[nper] host; outputs (device) [nper][ny][nx],
 * angle in degrees.  The caller forms sigma_deg = c_avg * T * wavelen_factor
 * / (2 pi) / (R_EARTH * DEG2RAD) (:116-119). */
int sa_topo_media(sa_ctx* ctx, int nx, int ny, const double* lon, const double* lat,
                  const double* z_gridded, int nper, const double* sigma_deg, double* m11,
                  double* m12, double* m22, double* angle, void* stream);

/* SurfGrid::correct_depth_with_topo (src/surf_grid.cpp:307-354): each depth
 * kernel column (ix, iy, iper) resampled at zgrid / cos(dip), clamped to the
 * depth range (interp1d, include/utils.h:451-485).  sen_* (device, may be
 * NULL) are (nx, ny, nz, nper) row-major, in place; angle [nper][ny][nx]
 * (device, degrees); zgrid[nz] host, nz <= 64. */
int sa_correct_depth_with_topo(sa_ctx* ctx, int nx, int ny, int nz, int nper, const double* zgrid,
                               const double* angle, double* sen_vs, double* sen_vp,
                               double* sen_rho, void* stream);

/* ---- optimizer: L-BFGS, strong Wolfe, model update (vs-only) --------------- */

/* History of the last 6 iterates (model vs and gradient, n values each, kept
 * on the device) for optimize::lbfgs_direction (reference
 * src/optimize.cpp:150-255), replacing the model_vs_NNN / grad_vs_NNN
 * datasets that Inversion::store_model / store_gradient write to HDF5
 * (src/inversion.cpp:326-373).  sa_lbfgs_store copies device arrays into the
 * slot of `iter`; sa_lbfgs_direction(iter) returns H_k g_k of the two-loop
 * recursion (5 pairs at most, log-space model differences) in dir (device). */
typedef struct sa_lbfgs sa_lbfgs;
int sa_lbfgs_create(sa_ctx* ctx, size_t n, sa_lbfgs** out);
void sa_lbfgs_destroy(sa_lbfgs* lbfgs);
int sa_lbfgs_store(sa_lbfgs* lbfgs, int iter, const double* model, const double* grad);
int sa_lbfgs_direction(sa_lbfgs* lbfgs, int iter, double* dir);

/* Inner product of two device arrays (FP64, fixed reduction order), result on
 * the host (optimize::field_dot + MPI sum, src/optimize.cpp:18-27, :62-68). */
int sa_dot(sa_ctx* ctx, size_t n, const double* a, const double* b, double* out);
/* Inversion::grad_normalization (src/inversion.cpp:302-323): g /= max|g|
 * unless max|g| < DBL_EPSILON; max_out (host, may be NULL) receives max|g|. */
int sa_grad_normalization(sa_ctx* ctx, size_t n, double* g, double* max_out);
/* optimize::calc_descent_angle (src/optimize.cpp:33-57), degrees, on the host. */
int sa_descent_angle(sa_ctx* ctx, size_t n, const double* dir, const double* grad, double* deg);
/* optimize::wolfe_condition (src/optimize.cpp:74-145) from gd = grad.dir and
 * kd = ker_next.dir (host arithmetic).  Returns 0 ACCEPT, 1 TRY, 2 FAIL (-1
 * for NULL pointers); updates the bracket and next_alpha as the reference. */
int sa_wolfe_condition(double gd, double kd, double alpha, double* alpha_L, double* alpha_R,
                       double f0, double f1, int subiter, double c1, double c2,
                       int max_sub_niter, double alpha_init, double* next_alpha);
/* Inversion::model_update, vs-only (src/inversion.cpp:465-490):
 * vs_out = vs*(1 - alpha*dir), vp_out = vs2vp(vs_out), rho_out = vp2rho(vp_out)
 * (vp_out, rho_out may be NULL; vs_out may alias vs).  Device arrays. */
int sa_model_update_vs(sa_ctx* ctx, size_t n, const double* vs, const double* dir, double alpha,
                       double* vs_out, double* vp_out, double* rho_out, void* stream);

/* ---- one misfit-gradient evaluation ---------------------------------------- */

/* Replaces one data type's pass of Inversion::run_forward_adjoint(true)
 * (reference src/inversion.cpp:245-276) up to and including combine_kernels,
 * for Rayleigh phase-velocity data and the vs-only parametrisation:
 * SurfGrid::fwdsurf (src/surf_grid.cpp:194-245), compute_dispersion_kernel
 * (:247-305), preproc::forward_for_event (src/preproc.cpp:71-148) over the
 * plan's events, combine_kernels (:276-304).  Kernel preconditioning and
 * smoothing (src/postproc.cpp) are not part of it.
 * sa_grad_create binds an existing plan (its grid, events and precision) to a
 * depth grid zgrid[nz] and the plan's nper periods[] (host arrays) and keeps
 * the depth-kernel arrays (3 x nx*ny*nz*nper doubles) on the device. */
typedef struct sa_grad sa_grad;
int sa_grad_create(sa_plan* plan, int nz, const double* zgrid, const double* periods,
                   sa_grad** out);
void sa_grad_destroy(sa_grad* grad);

/* The data type the handle evaluates (the reference's surfType loop,
 * src/inversion.cpp:250-296): 0 Rayleigh phase velocities (default), 1
 * Rayleigh group velocities -- fwdsurf with igr = 1 for the travel times and
 * the group depth kernels of SurfGrid::compute_dispersion_kernel, itype 1
 * (depthkernel_rayleigh_group, src/surfdisp.cpp:203-285: phase velocities at
 * t and t(1 +- 0.005), sregnpu).  The joint misfit and gradient are the
 * weighted sums over one handle per data type (weights of the reference's
 * data section). */
int sa_grad_set_data_type(sa_grad* grad, int igr);
/* The wave type (the reference's data iwave): 2 Rayleigh (default), 1 Love.
 * Love data: fwdsurf with iwave 1 for the travel times; as in the reference,
 * depth kernels exist for Love group data only (depthkernel_love_group via
 * depthkernel1d, src/surf_grid.cpp:282-286), so a Love phase-data run returns
 * SA_ERR_ARG where the reference's depthkernelHTI1d throws. */
int sa_grad_set_wave_type(sa_grad* grad, int iwave);

/* Kernel-density preconditioning (the reference's is_kden, postproc
 * kdensity_coe != 0).  Enabled, every sa_grad_run also solves, per event, the
 * kernel-density adjoint (src/preproc.cpp:128-137: source -w at every
 * receiver; the reference masks adj_field a second time rather than this
 * field, so it is accumulated unmasked) into kden_s; sa_grad_ker_den
 * combines it with the run's depth kernels into ker_den (nx, ny, nz)
 * (src/preproc.cpp:294-300), and sa_kernel_precondition applies
 * postproc::kernel_precondition (src/postproc.cpp:487-517) to a kernel.
 * The plan accumulates into this handle's buffer while enabled
 * (sa_plan_kden_output); one handle per plan may enable it. */
int sa_grad_set_kden(sa_grad* grad, int enable);
int sa_grad_ker_den(sa_grad* grad, const double* vs3d, const double* vp3d, double* ker_den,
                    void* stream);
/* ker[n] *= 1 / (ker_den / max|ker_den|) where that ratio exceeds 1e-12
 * (VERYTINY), unchanged elsewhere; nothing if max|ker_den| < 1e-12.  Device
 * arrays, enqueued on `stream` (NULL = the context's stream). */
int sa_kernel_precondition(sa_ctx* ctx, size_t n, const double* ker_den, double* ker,
                           void* stream);

/* Device arrays: vs3d, vp3d (NULL = Brocher vs2vp(vs3d), as the model keeps it
 * for vs-only inversions), ker_vs: (nx, ny, nz) row-major; tt_obs, weight:
 * [npair]; chi: 1 double.  svel_out and adj_s_out ([nper][ny][nx], may be
 * NULL) receive the phase velocities and the accumulated adjoint kernels;
 * status (1 device int, may be NULL) receives SA_ERR_NOROOT when a column's
 * root search failed, else the worst event status.  Enqueued on `stream`
 * (NULL = the context's stream); the depth kernels run on an internal stream
 * concurrently with the event batch. */
int sa_grad_run(sa_grad* grad, const double* vs3d, const double* vp3d, const double* tt_obs,
                const double* weight, double* ker_vs, double* chi, double* svel_out,
                double* adj_s_out, int* status, void* stream);

/* Receiver travel times of a vs model: SurfGrid::fwdsurf
 * (src/surf_grid.cpp:194-245) and the forward solve of every event
 * (src/preproc.cpp:88-111), no adjoint.  syn [npair] (device out); svel_out
 * (may be NULL) receives the phase velocities; status as sa_grad_run. */
int sa_grad_forward(sa_grad* grad, const double* vs3d, double* syn, double* svel_out,
                    int* status, void* stream);

/* Vector-Jacobian product of sa_grad_forward: for a vector source_adj [npair]
 * on the receiver times, fwdsurf and every forward field are recomputed, the
 * adjoint is driven by source_adj (sa_plan_adjoint_source), and the depth
 * kernels are combined into grad (nx, ny, nz):
 *   convention 0: the reference's combine_kernels (src/preproc.cpp:276-304),
 *     i.e. sa_grad_run's ker_vs when source_adj = w*(Tsyn - Tobs): a kernel
 *     per unit area from dimensionless depth kernels;
 *   convention 1: a derivative with respect to the vs nodes: times the cell
 *     area dx R cos(lat) dy R (the adjoint source is divided by it,
 *     src/eikonal_solver.cpp:366-367), with dc/dvs = K_b/b + K_a/a da/db +
 *     (rho dc/drho)/rho drho/da da/db formed from the dimensionless sregn96
 *     kernels, the density kernel corrected for the flattened velocities its
 *     elastic terms carry once more (src/surfker/sregn96.f90:1132, :1176), and
 *     the half-space layer added to the deepest node.  The eikonal part stays
 *     the reference's continuous adjoint;
 *   convention 2 (the plan's adjoint kind 1, sa_plan_set_adjoint): the exact
 *     gradient of the discrete forward model -- forward fields at a fixed
 *     point, the discrete adjoint (dchi/dsvel per cell and period), chained
 *     with dc/dvs from implicit differentiation of surfdisp96's Rayleigh
 *     secular function (dltar4) at each phase velocity; matches central
 *     differences of the receiver times' misfit.
 * vp3d NULL = vs2vp(vs3d).  svel_out, adj_s_out, status may be NULL. */
int sa_grad_vjp(sa_grad* grad, const double* vs3d, const double* vp3d, const double* source_adj,
                int convention, double* grad_out, double* svel_out, double* adj_s_out,
                int* status, void* stream);

/* dc/dvs of every node (nx, ny, nz, nper) row-major, device) from the
 * Rayleigh phase velocities of vs3d (no reference counterpart): implicit
 * differentiation of surfdisp96's secular function (dltar4) at each root,
 * chained through the earth flattening and the Brocher vp, rho; the
 * half-space layer adds to the deepest node.  Rayleigh phase data only. */
int sa_grad_root_derivatives(sa_grad* grad, const double* vs3d, double* dcdvs, void* stream);

/* Copies the last run's depth kernels into device arrays sen_vs, sen_vp,
 * sen_rho ((nx, ny, nz, nper) row-major; any may be NULL), on `stream`. */
int sa_grad_sen(sa_grad* grad, double* sen_vs, double* sen_vp, double* sen_rho, void* stream);

/* Multi-rank gradient: preproc::combine_kernels after the rank sum of adj_s
 * (src/preproc.cpp:225-304, mpi.sum_all_all of adj_s_local per period, then
 * the combination).  Combines the depth kernels of this handle's last
 * sa_grad_run with a caller-supplied adj_s (nper, ny, nx) -- the sum over
 * ranks of every rank's adj_s_out -- into ker_vs (nx, ny, nz).  vp3d NULL =
 * vs2vp(vs3d); vs3d must be the model of the last run.  Device pointers. */
int sa_grad_combine(sa_grad* grad, const double* vs3d, const double* vp3d, const double* adj_s,
                    double* ker_vs, void* stream);

/* ---- device math test hook ------------------------------------------------- */

/* No counterpart in the reference.  Evaluates the correctly rounded FP64
 * functions the dispersion and depth-kernel routines use in place of CUDA's
 * (and which agree with the C library the reference calls except where the C
 * library misrounds): f = 0 exp, 1 log, 2 sin, 3 cos, 4 sin and cos (y holds
 * n (sin, cos) pairs), 5 pow(x, -3) (the kernel accumulation's svel^-3).  x [n], y [n or 2n]: device arrays; enqueued on
 * `stream` (a cudaStream_t, NULL = legacy stream). */
int sa_math_eval(int f, size_t n, const double* x, double* y, void* stream);

/* ---- allocation-free entry point ------------------------------------------ */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory when they call in (inside another framework's allocator or memory
 * pool, hosts that forbid cudaMalloc after start-up, fully reserved device
 * memory): one eikonal::FSM_UW_PS_lonlat_2d solve in FP64 with every
 * intermediate in a fixed 64 MiB device array that each GPU loading this
 * library keeps until exit (145 bytes per cell: grids up to 462,400 cells,
 * e.g. 680 x 680; larger ones return SA_ERR_ARG with a message on stderr).
 * All array arguments are DEVICE pointers: xx_deg [nx], yy_deg [ny],
 * spha/sphb/sphc/fun/T_out [nx*ny]; niter and status (may be NULL) are single
 * device ints.  All work is enqueued on `stream` (a cudaStream_t, NULL =
 * legacy stream); the call does not wait for the GPU.  Calls share the array:
 * calls that overlap on the GPU race and must be serialised.  The first call
 * in each context (after start-up or a device reset) looks up the array's
 * address; make it before any stream capture. */
int sa_eik_fwd_field_noalloc(int nx, int ny, const double* xx_deg, const double* yy_deg,
                             const double* spha, const double* sphb, const double* sphc,
                             const double* fun, double x0_deg, double y0_deg, double* T_out,
                             int* niter, int* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif
