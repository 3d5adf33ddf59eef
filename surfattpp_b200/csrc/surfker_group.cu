// Group-velocity depth kernels (sregnpu), in a translation unit of their
// own where every shared routine stays inline.  With layer_integrals out of
// line (as the other column kernels have it), the kernels of the first
// evaluation, held in local arrays while the two later evaluations run, come
// back overwritten on the device (dU/dvp wrong by 1e-8 of the column
// maximum, by 1e4 with all eigenfunction routines out of line; dU/dvs and
// dU/drho exact).  The same source built for the host, inline or out of
// line, is exact, and neither the stack limit, the callee's spills nor FMA
// contraction change it.  The inline form matches the oracle bit for bit.
// Compiled with -fmad=false.
#define SK_MATH_NOINLINE 0
#include "surfker_dev.cuh"


namespace sa {
using sk::LayerConst;

// surfker::depthkernel_rayleigh_group (src/surfdisp.cpp:203-285) through
// sregnpu (src/surfker/sregn96.f90:1851-1992): one thread per (column,
// period); phase kernels at t, t1 = t(1 + 0.005) and t2 = t(1 - 0.005) from
// the three phase-velocity planes, the finite-difference group kernels and
// their earth-flattening conversion.  As in the reference, the first term of
// du/dm reads the kernels left by the last (t2) evaluation.
__global__ void SK_DEPTH_BOUNDS
depthkernel_group_kernel(int nx, int ny, int nz, const double* __restrict__ vs3d, int nper,
                         const double* __restrict__ periods, const double* __restrict__ p1,
                         const double* __restrict__ p2, const double* __restrict__ cp_plane,
                         const double* __restrict__ cp1_plane,
                         const double* __restrict__ cp2_plane, const LayerConst* __restrict__ Lp,
                         double* sen_vs, double* sen_vp, double* sen_rho) {
    long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool live = gid < (long long)nx * ny * nper;
    if (!live) {
        if (SK_DEPTH_PHASED == 0) return;
        gid = (long long)nx * ny * nper - 1;   // meets the barriers, stores nothing
    }
    // period-major: a warp takes 32 neighbouring columns at one period, whose
    // phase velocities stand alike against the layer velocities, so its lanes
    // take the same evanescent / oscillatory branches layer by layer
    const long long ncol = (long long)nx * ny;
    const int ip = (int)(gid / ncol);
    const int col = (int)(gid % ncol);
    const int ix = col / ny, iy = col % ny;
    const LayerConst& L = *Lp;
    float vp[sk::MMAX], vs[sk::MMAX], rho[sk::MMAX];
    sk::column_model(vs3d + (size_t)col * nz, nz, L, vp, vs, rho);
    sk::RW W;
    const int mmax = L.mmax;
    W.mmax = mmax;
    W.allfluid = true;
    for (int i = 0; i < mmax; i++) {
        W.zb[i] = vs[i];
        W.za[i] = vp[i];
        W.zrho[i] = rho[i];
        W.zd[i] = L.thk[i];
        W.iwat[i] = (W.zb[i] > 0.0) ? 0 : 1;
        if (W.zb[i] > 0.0) W.allfluid = false;
    }
    for (int i = 0; i < mmax; i++) {   // bldsph
        W.za[i] = W.za[i] * L.rg_vtp[i];
        W.zb[i] = W.zb[i] * L.rg_vtp[i];
        W.zrho[i] = W.zrho[i] * L.rg_rtp[i];
        W.zd[i] = L.rg_zd[i];
    }
    for (int i = 0; i < mmax; i++) {
        W.xmu[i] = W.zrho[i] * (W.zb[i] * W.zb[i]);
        W.xlam[i] = W.zrho[i] * (W.za[i] * W.za[i]) - 2.0 * W.xmu[i];
    }
    const size_t pix = (size_t)ip * nx * ny + ix + (size_t)nx * iy;
    const double pi = 3.1415926535897932384626433832795;
    const double twopi = 2.0 * pi;
    const double t = periods[ip], t1 = p1[ip], t2 = p2[ip];
    const double cp = cp_plane[pix];
    double ugr, fac;
    // period t (:1908-1918)
    double omega = twopi / t;
    sk::svfunc_phased(W, omega, omega / cp);
    sk::energy(W, omega, omega / cp, ugr, fac);
    const double cg = ugr;
    double a0[sk::MMAX], b0[sk::MMAX], r0[sk::MMAX], a1[sk::MMAX], b1[sk::MMAX], r1[sk::MMAX];
    for (int k = 0; k < nz; k++) {
        a0[k] = W.dcda[k];
        b0[k] = W.dcdb[k];
        r0[k] = W.dcdr[k];
    }
    // period t1 (:1921-1930)
    omega = twopi / t1;
    const double c1 = cp1_plane[pix];
    sk::svfunc_phased(W, omega, omega / c1);
    sk::energy(W, omega, omega / c1, ugr, fac);
    for (int k = 0; k < nz; k++) {
        a1[k] = W.dcda[k];
        b1[k] = W.dcdb[k];
        r1[k] = W.dcdr[k];
    }
    // period t2 (:1933-1942); W.dc* now hold this evaluation
    omega = twopi / t2;
    const double c2 = cp2_plane[pix];
    sk::svfunc_phased(W, omega, omega / c2);
    sk::energy(W, omega, omega / c2, ugr, fac);
    if (!live) return;
    // :1945-1971
    const double uc1 = cg / cp;
    const double ar = 6371.0;
    omega = twopi / t;
    const double r = cp / (2.0 * ar * omega);
    const double tm = sqrt(1.0 + r * r);
    const double q = 0.5 / (ar * omega);
    const double tm1 = (q * q) / tm;
    for (int k = 0; k < nz; k++) {
        const double dua = uc1 * (2.0 - uc1) * W.dcda[k] - uc1 * uc1 * t * (W.dcda[k] - a1[k]) / (t2 - t1);
        const double dub = uc1 * (2.0 - uc1) * W.dcdb[k] - uc1 * uc1 * t * (W.dcdb[k] - b1[k]) / (t2 - t1);
        const double dur = uc1 * (2.0 - uc1) * W.dcdr[k] - uc1 * uc1 * t * (W.dcdr[k] - r1[k]) / (t2 - t1);
        const size_t i4 = ((size_t)col * nz + k) * nper + ip;
        sen_vp[i4] = (tm * dua + cg * cp * a0[k] * tm1) * L.rg_vtp[k];
        sen_vs[i4] = (tm * dub + cg * cp * b0[k] * tm1) * L.rg_vtp[k];
        sen_rho[i4] = (tm * dur + cg * cp * r0[k] * tm1) * L.rg_rtp[k];
    }
}

cudaError_t launch_depthkernel_group(int nx, int ny, int nz, const double* vs3d, int nper,
                                     const double* periods, const double* p1, const double* p2,
                                     const double* cp, const double* cp1, const double* cp2,
                                     const void* layer_const, double* sen_vs, double* sen_vp,
                                     double* sen_rho, cudaStream_t st) {
    const long long n = (long long)nx * ny * nper;
    depthkernel_group_kernel<<<(unsigned)((n + SK_DEPTH_BLOCK - 1) / SK_DEPTH_BLOCK), SK_DEPTH_BLOCK,
                               0, st>>>(
        nx, ny, nz, vs3d, nper, periods, p1, p2, cp, cp1, cp2,
        reinterpret_cast<const LayerConst*>(layer_const), sen_vs, sen_vp, sen_rho);
    return cudaGetLastError();
}

}  // namespace sa
