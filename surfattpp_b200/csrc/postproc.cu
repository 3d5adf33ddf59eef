// PDE kernel smoothing (PostProc::pde_smooth, reference src/postproc.cpp:388-463):
// explicit Euler steps of the spherical 7-point Laplacian with Neumann boundary
// copies, one launch per step over a row-major (nx, ny, nz) field, depth
// fastest.  Compiled with -fmad=false: every product and sum rounds as the
// reference's FP64 expression reads (row and depth factors are formed on the
// host in the reference's left-to-right order).
//
// The boundary copies of :130-158 (x faces, then y faces, then z faces) leave
// every boundary cell equal to the updated cell at the clamped index
// (ix, iy, k) -> (clamp(ix, 1, nx-2), clamp(iy, 1, ny-2), clamp(k, 1, nz-2)),
// so one pass writes the whole step: a boundary thread recomputes the update
// of its clamped interior cell.  One read and one write of the field per
// step, neighbours from L1/L2.
#include "launch.h"

namespace sa {

struct PdeConst {
    int nx, ny, nz;
    double B;     // ch * dy2_inv
    double D;     // cv * dz2_inv
};

__global__ void __launch_bounds__(256) pde_step_kernel(PdeConst P, const double* __restrict__ u,
                                                       double* __restrict__ out,
                                                       const double* __restrict__ rowX,
                                                       const double* __restrict__ rowY,
                                                       const double* __restrict__ depE) {
    const size_t n = (size_t)P.nx * P.ny * P.nz;
    const size_t sy = (size_t)P.nz, sx = (size_t)P.ny * P.nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(i % P.nz);
        const size_t col = i / P.nz;
        const int iy = (int)(col % P.ny);
        const int ix = (int)(col / P.ny);
        const int cx = min(max(ix, 1), P.nx - 2);
        const int cy = min(max(iy, 1), P.ny - 2);
        const int ck = min(max(k, 1), P.nz - 2);
        const size_t c = ((size_t)cx * P.ny + cy) * P.nz + ck;
        const double center = u[c];
        // src/postproc.cpp:91-124
        const double d2u_dx2 = rowX[cy] * (u[c + sx] + u[c - sx] - 2.0 * center);
        const double u_jp1 = u[c + sy];
        const double u_jm1 = u[c - sy];
        const double d2u_dy2 = P.B * (u_jp1 + u_jm1 - 2.0 * center);
        const double du_dy = rowY[cy] * (u_jp1 - u_jm1);
        const double lat_term = d2u_dy2 - du_dy;
        const double u_kp1 = u[c + 1];
        const double u_km1 = u[c - 1];
        const double d2u_dz2 = P.D * (u_kp1 + u_km1 - 2.0 * center);
        const double du_dz = depE[ck] * (u_kp1 - u_km1);
        const double depth_term = d2u_dz2 - du_dz;
        // :453, dt = 1
        out[i] = center + 1.0 * (d2u_dx2 + lat_term + depth_term);
    }
}

// Division by an invariant divisor d as a multiply-high and a shift
// (Granlund and Montgomery, PLDI 1994, section 4): s = ceil(log2 d),
// m = floor(2^32 (2^s - d) / d) + 1, q = (umulhi(n, m) + n) >> s, exact for
// every n < 2^31 (the sum then fits 32 bits).
struct FastDiv {
    unsigned d, m, s;
};
static FastDiv make_fastdiv(unsigned d) {
    unsigned s = 0;
    while ((1ull << s) < d) s++;
    const unsigned long long m = ((1ull << 32) * ((1ull << s) - d)) / d + 1;
    return {d, (unsigned)m, s};
}
__device__ __forceinline__ unsigned fdiv_q(unsigned n, const FastDiv& f) {
    return (__umulhi(n, f.m) + n) >> f.s;
}

// The same step with 32-bit cell indices (fields below 2^31 cells): the
// row, column and depth of a cell from two multiply-high divisions instead
// of 64-bit divisions, which made the index arithmetic the bulk of the
// instructions.
__global__ void __launch_bounds__(256) pde_step_kernel32(PdeConst P, FastDiv fz, FastDiv fy,
                                                         const double* __restrict__ u,
                                                         double* __restrict__ out,
                                                         const double* __restrict__ rowX,
                                                         const double* __restrict__ rowY,
                                                         const double* __restrict__ depE) {
    const unsigned n = (unsigned)P.nx * P.ny * P.nz;
    const unsigned sy = (unsigned)P.nz, sx = (unsigned)P.ny * P.nz;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned col = fdiv_q(i, fz);
        const int k = (int)(i - col * fz.d);
        const unsigned ixu = fdiv_q(col, fy);
        const int iy = (int)(col - ixu * fy.d);
        const int ix = (int)ixu;
        const int cx = min(max(ix, 1), P.nx - 2);
        const int cy = min(max(iy, 1), P.ny - 2);
        const int ck = min(max(k, 1), P.nz - 2);
        const unsigned c = ((unsigned)cx * P.ny + cy) * P.nz + ck;
        const double center = u[c];
        // src/postproc.cpp:91-124
        const double d2u_dx2 = rowX[cy] * (u[c + sx] + u[c - sx] - 2.0 * center);
        const double u_jp1 = u[c + sy];
        const double u_jm1 = u[c - sy];
        const double d2u_dy2 = P.B * (u_jp1 + u_jm1 - 2.0 * center);
        const double du_dy = rowY[cy] * (u_jp1 - u_jm1);
        const double lat_term = d2u_dy2 - du_dy;
        const double u_kp1 = u[c + 1];
        const double u_km1 = u[c - 1];
        const double d2u_dz2 = P.D * (u_kp1 + u_km1 - 2.0 * center);
        const double du_dz = depE[ck] * (u_kp1 - u_km1);
        const double depth_term = d2u_dz2 - du_dz;
        // :453, dt = 1
        out[i] = center + 1.0 * (d2u_dx2 + lat_term + depth_term);
    }
}

cudaError_t launch_pde_smooth(int nx, int ny, int nz, double B, double D, const double* rowX,
                              const double* rowY, const double* depE, int nstep, double* field,
                              double* work, cudaStream_t st) {
    PdeConst P{nx, ny, nz, B, D};
    const size_t n = (size_t)nx * ny * nz;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)nsm * 8);
    double* a = field;
    double* b = work;
    const bool idx32 = n < (1ull << 31);
    const FastDiv fz = make_fastdiv((unsigned)nz), fy = make_fastdiv((unsigned)ny);
    for (int s = 0; s < nstep; s++) {
        if (idx32) pde_step_kernel32<<<blocks, 256, 0, st>>>(P, fz, fy, a, b, rowX, rowY, depE);
        else pde_step_kernel<<<blocks, 256, 0, st>>>(P, a, b, rowX, rowY, depE);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        double* t = a;
        a = b;
        b = t;
    }
    if (a != field) return cudaMemcpyAsync(field, a, n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    return cudaSuccess;
}

}  // namespace sa
