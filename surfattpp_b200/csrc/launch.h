// Host-side launch descriptors shared by the C ABI (capi.cu) and the kernel
// translation units (eik64.cu, eik32.cu, surfker.cu).
#pragma once
#include <algorithm>
#include <cstddef>
#include <cuda_runtime.h>

#include "common.cuh"

namespace sa {

struct BatchDesc {
    Grid g;
    int nper;
    int iso;
    // FP64 media / geometry
    const double* fun64;
    const double* inv3;
    const double* a_f_row64;
    const double* a_a_row64;
    double b_iso;
    const double* mt64;     // packed {a, b, c, 0} forward metric per period (general)
    const double* b_p64;
    const double* a_a64;
    const double* c_a64;
    const double* G64;
    const double* Gx64;
    const double* Gy64;
    // FP32 media / geometry
    const float* fun32;
    const float* a_f_row32;
    float b_iso32;
    const float* mt32;
    const float* G32;
    const float* Gx32;
    const float* Gy32;
    Events ev;
    Outputs out;
    Scratch sc;
    int maxr;
    int mode;
    int variant;   // FP32 launch variant (batch.cuh), 0 = default
    // 0: the reference's adjoint and forward stopping rule; 1 (FP64 plans):
    // forward solves run to a fixed point and the adjoint is the exact
    // discrete adjoint (batch.cuh, discrete_adjoint); adj_s then receives
    // dchi/dsvel
    int discrete;
};

// Number of FP32 batch-kernel launch variants (batch.cuh).
constexpr int kBatchVariants = 8;

size_t batch64_slot_bytes(int nx, int ny, int maxr);
int batch64_max_slots(int device);
size_t batch32_slot_bytes(int nx, int ny, int maxr);
int batch32_max_slots(int device);

cudaError_t launch_media64(int nx, int ny, int nper, const double* svel, const double* m11,
                           const double* m12, const double* m22, const double* cosy,
                           double* fun, double* inv3, double* mt, double* b_p, double* a_a,
                           double* c_a, cudaStream_t st);
cudaError_t launch_media32(int nx, int ny, int nper, const double* fun64, const double* mt64,
                           float* fun32, float* mt32, cudaStream_t st);
template <class T>
cudaError_t launch_geometry(int nx, int ny, int nsrc, const double* siny, const double* cosy,
                            const double* sy0, const double* cy0, const double* cdl,
                            const double* sdl, T* G, T* Gx, T* Gy, double* G64,
                            cudaStream_t st);
cudaError_t launch_batch64(const BatchDesc& d, cudaStream_t st);
// one launch over nlev plans' events (code[qi] = level << 24 | event); the
// levels' arguments are copied to dev_args (nlev x batch{32,64}_args_bytes())
cudaError_t launch_batch32_multi(const BatchDesc* d, int nlev, void* dev_args, unsigned ntotal,
                                 const unsigned* code, const Scratch& sc, cudaStream_t st);
cudaError_t launch_batch64_multi(const BatchDesc* d, int nlev, void* dev_args, unsigned ntotal,
                                 const unsigned* code, const Scratch& sc, cudaStream_t st);
size_t batch32_args_bytes();
size_t batch64_args_bytes();
// launch_batch64 with the grid spacing read on the device from dxdy[0..1]
cudaError_t launch_batch64_dev_spacing(const BatchDesc& d, const double* dxdy, cudaStream_t st);
cudaError_t launch_batch32(const BatchDesc& d, cudaStream_t st);

}  // namespace sa

namespace sa {
// deterministic accumulation of one chunk of per-event contributions, and
// the misfit summed in event order
cudaError_t launch_ordered_accumulate(size_t n, int nper, int e0, const int* per_ptr,
                                      const int* per_ev, const double* contrib, double* adj_s,
                                      cudaStream_t st);
cudaError_t launch_sum_events_ordered(int ne, const double* chi_ev, double* chi,
                                      cudaStream_t st);
cudaError_t launch_sum_events(int ne, const double* chi_ev, double* chi, cudaStream_t st);
cudaError_t launch_fold_status(int ne, const int* status, int* worst, cudaStream_t st);
}  // namespace sa

namespace sa {
// surfker.cu
size_t layer_const_bytes();
int build_layer_const(int nz, const double* zgrid, void* out);
cudaError_t launch_surfdisp_columns(int nx, int ny, int nz, const double* vs3d, int nper,
                                    const double* periods, int iflsph, int iwave, int igr,
                                    const void* layer_const, double* svel, int* status,
                                    cudaStream_t st);
cudaError_t launch_depthkernel(int nx, int ny, int nz, const double* vs3d, int nper,
                               const double* periods, const double* cp, const void* layer_const,
                               double* sen_vs, double* sen_vp, double* sen_rho, cudaStream_t st,
                               double* sen_hs = nullptr);
cudaError_t launch_event_cost(int ne, const int* fwd_it, const int* adj_it, unsigned int* key,
                              int* idx, cudaStream_t st);
// multi-grid queue keys of one level (work = sweeps x cells) and codes
cudaError_t launch_multi_cost(int ne, const int* fwd_it, const int* adj_it, unsigned int scale,
                              int lev, unsigned int* key, int* code, cudaStream_t st);
size_t sort_events_temp_bytes(int ne);
cudaError_t launch_sort_events(int ne, const unsigned int* key_in, unsigned int* key_out,
                               const int* idx_in, int* order, void* temp, size_t temp_bytes,
                               cudaStream_t st);
cudaError_t launch_grad_status(int ncol, const int* colst, const int* ev_worst, int* out,
                               cudaStream_t st);
// optimize.cu (scratch of reduce_scratch_doubles(); the result lands in its last entry)
size_t reduce_scratch_doubles();
cudaError_t launch_dot(size_t n, const double* a, const double* b, double* scratch,
                       cudaStream_t st);
cudaError_t launch_absmax(size_t n, const double* a, double* scratch, cudaStream_t st);
// postproc::kernel_precondition of ker by ker_den (scratch: reduction scratch)
cudaError_t launch_kernel_precondition(size_t n, const double* ker_den, double* scratch,
                                       double* ker, cudaStream_t st);
cudaError_t launch_lbfgs_pair(size_t n, const double* m0, const double* m1, const double* g0,
                              const double* g1, double* s, double* y, cudaStream_t st);
cudaError_t launch_axpy(size_t n, int kind, double c, const double* x, double* y,
                        cudaStream_t st);
cudaError_t launch_model_update_vs(size_t n, const double* vs, const double* dir, double alpha,
                                   double* vs_out, double* vp_out, double* rho_out,
                                   cudaStream_t st);
// topo.cu
cudaError_t launch_gauss_geo(int nx, int ny, const double* data, const double* lons,
                             const double* lats, double sigma, double* out, cudaStream_t st);
cudaError_t launch_topo_media(int nx, int ny, const double* z, const double* lon,
                              const double* lat, double* m11, double* m12, double* m22,
                              double* angle, cudaStream_t st);
cudaError_t launch_depth_topo(int nx, int ny, int nz, int nper, const double* zg,
                              const double* angle, double* k0, double* k1, double* k2,
                              cudaStream_t st);
cudaError_t launch_grid_topo(int nxr, int nyr, const double* xr, const double* yr,
                             const double* zr, int nx, int ny, const double* x, const double* y,
                             double* out, cudaStream_t st);
// postproc.cu
cudaError_t launch_pde_smooth(int nx, int ny, int nz, double B, double D, const double* rowX,
                              const double* rowY, const double* depE, int nstep, double* field,
                              double* work, cudaStream_t st);
// Love depth kernels (igr 0 phase at cp; 1 group from cp, cp1, cp2)
cudaError_t launch_depthkernel_love(int nx, int ny, int nz, const double* vs3d, int nper,
                                    const double* periods, const double* p1, const double* p2,
                                    const double* cp, const double* cp1, const double* cp2,
                                    int igr, const void* layer_const, double* sen_vs,
                                    double* sen_rho, cudaStream_t st);
cudaError_t launch_depthkernel_group(int nx, int ny, int nz, const double* vs3d, int nper,
                                     const double* periods, const double* p1, const double* p2,
                                     const double* cp, const double* cp1, const double* cp2,
                                     const void* layer_const, double* sen_vs, double* sen_vp,
                                     double* sen_rho, cudaStream_t st);
// exact dc/dvs per node from the phase-velocity roots (surfker.cu)
cudaError_t launch_dispersion_dcdvs(int nx, int ny, int nz, const double* vs3d, int nper,
                                    const double* periods, const double* svel,
                                    const void* layer_const, double* dcdvs, cudaStream_t st);
cudaError_t launch_combine_exact(int nx, int ny, int nz, int nper, const double* dchi_dsvel,
                                 const double* dcdvs, double* grad, cudaStream_t st);
cudaError_t launch_combine_vs(int nx, int ny, int nz, int nper, const double* adj_s,
                              const double* vs3d, const double* vp3d, const double* sen_vs,
                              const double* sen_vp, const double* sen_rho, double* ker_vs,
                              cudaStream_t st);
// the vs gradient as a derivative (area Jacobian, plain dc/dvs, corrected
// density term, half-space at the deepest node); sen_hs may be NULL
cudaError_t launch_combine_vs_derivative(int nx, int ny, int nz, int nper, const double* adj_s,
                                         const double* vs3d, const double* vp3d,
                                         const double* sen_vs, const double* sen_vp,
                                         const double* sen_rho, const double* sen_hs,
                                         const double* area_row, const void* layer_const,
                                         double* grad, cudaStream_t st);
}  // namespace sa
