// Optimizer primitives on device (vs-only parametrisation): deterministic FP64
// inner products and max-abs, the L-BFGS history vectors, axpy-type updates
// and the multiplicative model update with the Brocher relations.
// Reference: src/optimize.cpp:14-255, src/inversion.cpp:302-323, :465-490.
// Compiled with -fmad=false: elementwise results round as the reference's.
// All kernels are HBM-bound streams over n values.
#include "launch.h"

namespace sa {

namespace {
constexpr int RED_BLOCKS = 1184;   // 148 SMs x 8: fixed, so sums are reproducible
constexpr int RED_THREADS = 256;

__device__ __forceinline__ double brocher_vs2vp(double vs) {   // include/utils.h:237-245
    return 0.9409 + 2.0947 * vs - 0.8206 * vs * vs + 0.2683 * vs * vs * vs
         - 0.0251 * vs * vs * vs * vs;
}
__device__ __forceinline__ double brocher_vp2rho(double vp) {  // include/utils.h:247-254
    return 1.6612 * vp - 0.4721 * vp * vp + 0.0671 * vp * vp * vp - 0.0043 * vp * vp * vp * vp
         + 0.000106 * vp * vp * vp * vp * vp;
}

template <int OP>   // 0: sum a*b, 1: max |a|
__global__ void __launch_bounds__(RED_THREADS) reduce_partial(size_t n, const double* __restrict__ a,
                                                              const double* __restrict__ b,
                                                              double* partial) {
    __shared__ double sh[RED_THREADS];
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)RED_THREADS + threadIdx.x; i < n;
         i += (size_t)gridDim.x * RED_THREADS) {
        if (OP == 0) acc += a[i] * b[i];
        else acc = fmax(acc, fabs(a[i]));
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            sh[threadIdx.x] = OP == 0 ? sh[threadIdx.x] + sh[threadIdx.x + w]
                                      : fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

template <int OP>
__global__ void __launch_bounds__(1024) reduce_final(int np, const double* partial, double* out) {
    __shared__ double sh[1024];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += 1024)
        acc = OP == 0 ? acc + partial[i] : fmax(acc, partial[i]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            sh[threadIdx.x] = OP == 0 ? sh[threadIdx.x] + sh[threadIdx.x + w]
                                      : fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

__global__ void pair_kernel(size_t n, const double* __restrict__ m0, const double* __restrict__ m1,
                            const double* __restrict__ g0, const double* __restrict__ g1,
                            double* s, double* y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        s[i] = log(m1[i]) - log(m0[i]);   // src/optimize.cpp:190-191 (log space)
        y[i] = g1[i] - g0[i];             // :197
    }
}

// y = a*x + b*y  (kind 0: y - c*x; 1: c*y; 2: y + c*x; 3: y / c)
__global__ void axpy_kernel(size_t n, int kind, double c, const double* __restrict__ x, double* y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double v = y[i];
        if (kind == 0) y[i] = v - c * x[i];
        else if (kind == 1) y[i] = c * v;
        else if (kind == 2) y[i] = v + c * x[i];
        else y[i] = v / c;
    }
}

__global__ void model_update_kernel(size_t n, const double* __restrict__ vs,
                                    const double* __restrict__ dir, double alpha, double* vs_out,
                                    double* vp_out, double* rho_out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double v = vs[i] * (1 - alpha * dir[i]);   // src/inversion.cpp:471
        vs_out[i] = v;
        if (vp_out || rho_out) {
            const double vp = brocher_vs2vp(v);             // :478-479
            if (vp_out) vp_out[i] = vp;
            if (rho_out) rho_out[i] = brocher_vp2rho(vp);
        }
    }
}

// postproc::kernel_precondition (src/postproc.cpp:487-517): with L = max
// |ker_den| (linf[0], from launch_absmax), ker *= 1 / (ker_den / L) where
// ker_den / L > VERYTINY (include/config.h:71), and nothing when L < VERYTINY.
__global__ void precondition_kernel(size_t n, const double* __restrict__ ker_den,
                                    const double* __restrict__ linf, double* ker) {
    const double L = *linf;
    if (L < 1e-12) return;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double norm = ker_den[i] / L;
        const double h = norm > 1e-12 ? 1.0 / norm : 1.0;
        ker[i] = ker[i] * h;
    }
}

unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }
}  // namespace

cudaError_t launch_kernel_precondition(size_t n, const double* ker_den, double* scratch,
                                       double* ker, cudaStream_t st) {
    cudaError_t e = launch_absmax(n, ker_den, scratch, st);
    if (e != cudaSuccess) return e;
    precondition_kernel<<<grid_for(n), 256, 0, st>>>(n, ker_den,
                                                    scratch + reduce_scratch_doubles() - 1, ker);
    return cudaGetLastError();
}

size_t reduce_scratch_doubles() { return RED_BLOCKS + 1; }

cudaError_t launch_dot(size_t n, const double* a, const double* b, double* scratch,
                       cudaStream_t st) {
    reduce_partial<0><<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, a, b, scratch);
    reduce_final<0><<<1, 1024, 0, st>>>(RED_BLOCKS, scratch, scratch + RED_BLOCKS);
    return cudaGetLastError();
}

cudaError_t launch_absmax(size_t n, const double* a, double* scratch, cudaStream_t st) {
    reduce_partial<1><<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, a, a, scratch);
    reduce_final<1><<<1, 1024, 0, st>>>(RED_BLOCKS, scratch, scratch + RED_BLOCKS);
    return cudaGetLastError();
}

cudaError_t launch_lbfgs_pair(size_t n, const double* m0, const double* m1, const double* g0,
                              const double* g1, double* s, double* y, cudaStream_t st) {
    pair_kernel<<<grid_for(n), 256, 0, st>>>(n, m0, m1, g0, g1, s, y);
    return cudaGetLastError();
}

cudaError_t launch_axpy(size_t n, int kind, double c, const double* x, double* y,
                        cudaStream_t st) {
    axpy_kernel<<<grid_for(n), 256, 0, st>>>(n, kind, c, x, y);
    return cudaGetLastError();
}

cudaError_t launch_model_update_vs(size_t n, const double* vs, const double* dir, double alpha,
                                   double* vs_out, double* vp_out, double* rho_out,
                                   cudaStream_t st) {
    model_update_kernel<<<grid_for(n), 256, 0, st>>>(n, vs, dir, alpha, vs_out, vp_out, rho_out);
    return cudaGetLastError();
}

}  // namespace sa
