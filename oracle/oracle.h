/*
 * CPU oracle for the SurfATTPP forward + adjoint misfit-gradient path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain C++ restatement, operation
 * for operation, of the reference's CPU arithmetic.  It is the parity checker for
 * the CUDA engine in surfattpp_b200/ and the timed CPU baseline; nothing in the
 * product links or calls it.
 *
 * Build rule: -O2 -ffp-contract=off, no -march, no -ffast-math, so every
 * expression rounds in source order exactly as written (the reference's own
 * release build uses -O3 -march=native, whose FMA contraction is machine
 * dependent; the oracle fixes the uncontracted IEEE semantics).
 *
 * Storage conventions follow the reference:
 *   2-D fields are Eigen column-major (nx x ny): index ix + nx*iy.
 *   Per-period media are [iper][iy][ix] planes here (one plane per period).
 *   Depth kernels sen_* are row-major (nx, ny, nz, nper), nper fastest
 *   (reference src/surf_grid.cpp:5-8).
 */
#ifndef SURFATT_ORACLE_H
#define SURFATT_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* eikonal::FSM_UW_PS_lonlat_2d (src/eikonal_solver.cpp:22-318).
 * Returns 0, or -1 for a grid smaller than 3x3.  *niter = sweep iterations run. */
int orc_eik_fwd(int nx, int ny, const double* xx_deg, const double* yy_deg,
                const double* spha, const double* sphb, const double* sphc,
                const double* fun, double x0_deg, double y0_deg,
                double* T_out, int* niter);
/* The forward solve with the stopping rule as a parameter: tol > 0 as the
 * reference (1e-4), tol == 0 to a fixed point (no cell changes). */
/* Derivatives of surfdisp96's Rayleigh phase velocities c[kmax] with
 * respect to each layer's vs, vp, rho ([k * nlayer + layer]). */
int orc_dispersion_dcdm(const float* thkm, const float* vpm, const float* vsm, const float* rhom,
                        int nlayer, int kmax, const double* t, const double* c, double* dcdb,
                        double* dcda, double* dcdr);
int orc_eik_fwd_tol(int nx, int ny, const double* xx_deg, const double* yy_deg,
                    const double* spha, const double* sphb, const double* sphc, const double* fun,
                    double x0_deg, double y0_deg, double tol, int maxiter, double* T_out,
                    int* niter);
/* Exact discrete adjoint of the forward solve (eikonal_discrete.cpp):
 * receiver times syn[nr] and, with dchi_dT[nr], grad_fun = dchi/dfun. */
int orc_eik_discrete_grad(int nx, int ny, const double* xx_deg, const double* yy_deg,
                          const double* spha, const double* sphb, const double* sphc,
                          const double* fun, double x0_deg, double y0_deg, double tol,
                          int maxiter, int nr, const double* xrec_deg, const double* yrec_deg,
                          const double* dchi_dT, double* syn, double* grad_fun, int* niter);
/* All events with the discrete gradient: grad_svel [nper][ny][nx] +=
 * dchi/dsvel, chi, syn (sadj: a vector-Jacobian product instead). */
int orc_discrete_for_events(int nx, int ny, int nper, const double* xx_deg, const double* yy_deg,
                            const double* svel, const double* m11, const double* m12,
                            const double* m22, int ne, const double* evlo, const double* evla,
                            const int* iper, const int* rec_ptr, const int* rec_idx,
                            const double* stlo, const double* stla, const double* tt_obs,
                            const double* weight, const double* sadj, double tol, int maxiter,
                            double* syn, double* grad_svel, double* chi, int* fwd_iters,
                            int nthreads);

/* eikonal::FSM_O1_JSE_lonlat_2d (src/eikonal_solver.cpp:323-511). */
int orc_eik_adj(int nx, int ny, const double* xx_deg, const double* yy_deg,
                const double* spha, const double* sphb, const double* sphc,
                const double* T, int nr, const double* xrec_deg,
                const double* yrec_deg, const double* source_adj,
                double* Ta_out, int* niter);

/* eikonal::mask_uniform_grid (src/eikonal_solver.cpp:514-536). */
void orc_mask_uniform_grid(int nx, int ny, const double* xx, const double* yy,
                           double* table, double x0, double y0);

/* interp2d (include/utils.h:358-409). */
void orc_interp2d(int nx, int ny, const double* xgrid, const double* ygrid,
                  const double* z, int nq, const double* xq, const double* yq,
                  double* zq);

/* preproc::forward_for_event over a flat event list (src/preproc.cpp:71-148),
 * isotropic branch, is_kden = false.
 *   svel, m11, m12, m22 : [nper][ny][nx] planes (column-major per period)
 *   events              : evlo[ne], evla[ne], iper[ne], rec_ptr[ne+1] (CSR),
 *                         rec_idx[rec_ptr[ne]] station indices
 *   stations            : stlo[nsta], stla[nsta]
 *   obs per pair        : tt_obs[rec_ptr[ne]], weight[rec_ptr[ne]]
 * Outputs: syn[rec_ptr[ne]] synthetic times; if calc_adj, adj_s [nper][ny][nx]
 * is ACCUMULATED (caller zeroes it) and the misfit is returned in *chi.
 * fwd_iters/adj_iters (may be NULL) receive per-event iteration counts.
 * nthreads > 1 deals events round-robin over threads (reference
 * include/parallel.h:39-41) and sums per-thread accumulators in thread order.
 * kden_s (may be NULL; is_kden) [nper][ny][nx] ACCUMULATES the
 * kernel-density adjoint (src/preproc.cpp:128-137). */
int orc_forward_for_events(int nx, int ny, int nper, const double* xx_deg,
                           const double* yy_deg, const double* svel,
                           const double* m11, const double* m12, const double* m22,
                           int ne, const double* evlo, const double* evla,
                           const int* iper, const int* rec_ptr, const int* rec_idx,
                           const double* stlo, const double* stla,
                           const double* tt_obs, const double* weight,
                           int calc_adj, double* syn, double* adj_s, double* chi,
                           int* fwd_iters, int* adj_iters, int nthreads, double* kden_s);

/* postproc::kernel_precondition (src/postproc.cpp:487-517), in place on ker[n]. */
void orc_kernel_precondition(size_t n, const double* ker_den, double* ker);

/* preproc::combine_kernels, vs-only branch (src/preproc.cpp:276-304).
 *   adj_s [nper][ny][nx]; vs3d, vp3d (nx, ny, nz) row-major;
 *   sen_vs/vp/rho (nx, ny, nz, nper) row-major; ker_vs (nx, ny, nz) out. */
void orc_combine_kernels_vs(int nx, int ny, int nz, int nper, const double* adj_s,
                            const double* vs3d, const double* vp3d,
                            const double* sen_vs, const double* sen_vp,
                            const double* sen_rho, double* ker_vs);

/* Brocher (2005) relations (include/utils.h:185-234). */
double orc_vs2vp(double vs);
double orc_vp2rho(double vp);
double orc_dalpha_dbeta(double vs);
double orc_drho_dalpha(double vp);

/* surfdisp96 (src/surfker/surfdisp96.f:57-373) via the C ABI surfdisp96_c.
 * Returns 0 on success, 1 when the root search failed for the fundamental mode
 * (where the Fortran executes `stop 'Dispersion calculation failed'`). */
int orc_surfdisp96(const float* thkm, const float* vpm, const float* vsm,
                   const float* rhom, int nlayer, int iflsph, int iwave, int mode,
                   int igr, int kmax, const double* t, double* cg);

/* sregn96_hti (src/surfker/sregn96.f90:1745-1849). All arrays length nlayer. */
void orc_sregn96_hti(const float* thk, const float* vp, const float* vs,
                     const float* rhom, int nlayer, double* t, double* cp,
                     double* cg, double* dispu, double* dispw, double* stressu,
                     double* stressw, double* dc2da, double* dc2db, double* dc2dh,
                     double* dc2dr, double* dc2dgc, double* dc2dgs, int iflsph);

/* sregn96 (src/surfker/sregn96.f90:1640-1743). */
void orc_sregn96(const float* thk, const float* vp, const float* vs,
                 const float* rhom, int nlayer, double* t, double* cp, double* cg,
                 double* dispu, double* dispw, double* stressu, double* stressw,
                 double* dc2da, double* dc2db, double* dc2dh, double* dc2dr,
                 int iflsph);

/* SurfGrid::fwdsurf over columns (src/surf_grid.cpp:194-245) with the
 * Brocher branch (use_alpha_beta_rho = false).
 *   zgrid[nz]; vs3d (nx, ny, nz) row-major; periods[nper]
 *   svel out: [nper][ny][nx] planes.  status[nx*ny] (0 ok, 1 no root). */
int orc_fwdsurf(int nx, int ny, int nz, const double* zgrid, const double* vs3d,
                int nper, const double* periods, int iwave, int igr,
                double* svel, int* status, int nthreads);

/* SurfGrid::compute_dispersion_kernel for phase velocity (PH) columns, which
 * always runs depthkernelHTI1d (src/surf_grid.cpp:247-305,
 * src/surfdisp.cpp:481-547).  sen_vs/vp/rho out (nx, ny, nz, nper) row-major. */
int orc_depthkernel_hti(int nx, int ny, int nz, const double* zgrid,
                        const double* vs3d, int nper, const double* periods,
                        double* sen_vs, double* sen_vp, double* sen_rho,
                        int* status, int nthreads);

/* PostProc::pde_smooth (src/postproc.cpp:388-463), one rank.  field (nx, ny, nz)
 * row-major, depth fastest, smoothed in place.  dx, dy in degrees, dz in km;
 * ygrid[ny] latitudes (degrees), zgrid[nz] depths (km).  Returns 0, or < 0 for
 * invalid sigma (-1), too fine a grid (-2) or a grid below 3x3x3 (-3).
 * orc_pde_smooth_nstep returns the step count and the per-step diffusion
 * coefficients ch (deg^2) and cv (km^2) (:407-434). */
int orc_pde_smooth_nstep(int ny, double dx, double dy, double dz, double y_first,
                         double y_last, double sigma_h, double sigma_v, double* ch, double* cv);
int orc_pde_smooth(int nx, int ny, int nz, double dx, double dy, double dz, const double* ygrid,
                   const double* zgrid, double sigma_h, double sigma_v, double* field,
                   int* nstep_out);

/* Optimizer (vs-only parametrisation, src/optimize.cpp, src/inversion.cpp).
 * orc_lbfgs_direction: models/grads are nhist + 1 consecutive iterates (oldest
 * first, the current one last), n values each; dir receives H g. */
void orc_lbfgs_direction(size_t n, int nhist, const double* const* models,
                         const double* const* grads, double* dir);
double orc_grad_normalization(size_t n, double* g);
double orc_descent_angle(size_t n, const double* dir, const double* grad);
int orc_wolfe_condition(double gd, double kd, double alpha, double* alpha_L, double* alpha_R,
                        double f0, double f1, int subiter, double c1, double c2,
                        int max_sub_niter, double alpha_init, double* next_alpha);
void orc_model_update_vs(size_t n, const double* vs, const double* dir, double alpha,
                         double* vs_out, double* vp_out, double* rho_out);
double orc_vs2vp(double vs);
double orc_vp2rho(double vp);

/* Topography (src/surf_grid.cpp:80-166, :307-354; include/utils.h:505-649;
 * src/topo.cpp:97-114).  2-D fields column-major nx x ny; per-period outputs
 * [nper][ny][nx]; ker (nx, ny, nz, nper) row-major, corrected in place. */
void orc_gaussian_smooth_geo_2(int nx, int ny, const double* data, const double* lons,
                               const double* lats, double sigma, double* out);
void orc_gradient_2_geo(int nx, int ny, const double* f, const double* lon, const double* lat,
                        double* tx, double* ty);
void orc_topo_media(int nx, int ny, const double* lon, const double* lat,
                    const double* z_gridded, int nper, const double* sigma_deg, double* m11,
                    double* m12, double* m22, double* angle);
void orc_correct_depth_with_topo(int nx, int ny, int nz, int nper, const double* zgrid,
                                 const double* angle, double* ker);

/* sregnpu (src/surfker/sregn96.f90:1851-1992) and the per-column Rayleigh
 * group-velocity depth kernels (surfker::depthkernel_rayleigh_group,
 * src/surfdisp.cpp:203-285); outputs as orc_depthkernel_hti. */
void orc_sregnpu(const float* thk, const float* vp, const float* vs, const float* rhom,
                 int nlayer, double t, double cp, double t1, double cp1, double t2, double cp2,
                 double* cg, double* du2da, double* du2db, double* du2dh, double* du2dr,
                 double* dc2da, double* dc2db, double* dc2dh, double* dc2dr, int iflsph);
int orc_depthkernel_group(int nx, int ny, int nz, const double* zgrid, const double* vs3d,
                          int nper, const double* periods, double* sen_vs, double* sen_vp,
                          double* sen_rho, int* status, int nthreads);

/* slegn96 / slegnpu (src/surfker/slegn96.f90:672-919): Love phase kernels
 * dc2db = b dc/db, dc2dr at cp; group kernels du2db, du2dr from the phase
 * velocities at t, t1, t2.  Arrays of length nlayer; cg (may be NULL). */
void orc_slegn96(const float* thk, const float* vs, const float* rhom, int nlayer, double t,
                 double cp, double* cg, double* dc2db, double* dc2dr, int iflsph);
void orc_slegnpu(const float* thk, const float* vs, const float* rhom, int nlayer, double t,
                 double cp, double t1, double cp1, double t2, double cp2, double* cg,
                 double* du2db, double* du2dr, int iflsph);
/* Per-column Love depth kernels (surfker::depthkernel_love_phase / _group,
 * src/surfdisp.cpp:295-426): sen_vs, sen_rho (nx, ny, nz, nper). */
int orc_depthkernel_love(int nx, int ny, int nz, const double* zgrid, const double* vs3d,
                         int nper, const double* periods, int igr, double* sen_vs,
                         double* sen_rho, int* status, int nthreads);

/* PostProc::smooth, smooth_method 1 (src/postproc.cpp:160-386, :465-480):
 * buf, out (nx, ny, nz) row-major; -1 when a node lies outside. */
int orc_multigrid_smooth(int nx, int ny, int nz, const double* x, const double* y,
                         const double* z, const int* n_inv, int nset, const double* buf,
                         double* out);

#ifdef __cplusplus
}
#endif
#endif
