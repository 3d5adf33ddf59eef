// FP64 engine: per-period media preparation, per-source geometry, and the
// persistent batch kernel (one warp per (source, period) event; forward FSM,
// receiver interpolation, adjoint FSM, source mask, kernel accumulation).
//
// Compiled with -fmad=false: every multiply and add rounds separately, as in
// the reference's FP64 source.  The FP64 path is the parity path.
#include <vector>

#include "common.cuh"
#include "event_common.cuh"
#include "batch.cuh"
#include "crmath.cuh"
#include "launch.h"

namespace sa {

// ---------------------------------------------------------------------------
// Per-period media: fun = (1/svel)*1 (src/preproc.cpp:97-98), svel^-3
// (src/preproc.cpp:28-29), and for a general (topography) metric the forward
// and adjoint a, b, c planes (src/eikonal_solver.cpp:55-65 and :380-389).
// ---------------------------------------------------------------------------
__global__ void media64_kernel(int nx, int ny, int nper, const double* __restrict__ svel,
                               const double* __restrict__ m11, const double* __restrict__ m12,
                               const double* __restrict__ m22, const double* __restrict__ cosy,
                               double* fun, double* inv3, double* mt, double* b_p, double* a_a,
                               double* c_a) {
    const size_t n = (size_t)nx * ny;
    const size_t total = n * nper;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const double s = svel[i];
        fun[i] = (1.0 / s) * 1.0;
        inv3[i] = cr::pow_m3(s);   // pow(svel, -3), correctly rounded
        if (m11) {
            const int iy = (int)((i % n) / nx);
            const double cos_y = cosy[iy];
            const double cos2_y = cos_y * cos_y;
            const double R2 = R_EARTH * R_EARTH;
            const double spha = m11[i], sphb = m22[i], sphc = -m12[i];
            const double bv = sphb / R2;
            mt[4 * i + 0] = spha / (R2 * cos2_y);
            mt[4 * i + 1] = bv;
            mt[4 * i + 2] = sphc / (R_EARTH * R_EARTH * cos_y);
            mt[4 * i + 3] = 0.0;
            b_p[i] = bv;
            a_a[i] = spha / (R2 * cos_y * cos_y);
            c_a[i] = sphc / (R2 * cos_y);
        }
    }
}

// ---------------------------------------------------------------------------
// Great-circle geometry per unique source (src/eikonal_solver.cpp:96-116
// without the fun0 factor): G = acos(.)*R, Gx, Gy with T0 = G*fun0 etc.
// cdl/sdl = cos/sin(xx - x0) per (source, column), siny/cosy per row and
// sy0/cy0 per source come from the host C library.
// ---------------------------------------------------------------------------
template <class T>
__global__ void geometry_kernel(int nx, int ny, int nsrc, const double* __restrict__ siny,
                                const double* __restrict__ cosy, const double* __restrict__ sy0,
                                const double* __restrict__ cy0, const double* __restrict__ cdl,
                                const double* __restrict__ sdl, T* G, T* Gx, T* Gy,
                                double* G64) {
    const size_t n = (size_t)nx * ny;
    const size_t total = n * nsrc;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int s = (int)(i / n);
        const size_t k = i % n;
        const int iy = (int)(k / nx), ix = (int)(k % nx);
        const double sy = siny[iy], cy = cosy[iy];
        const double cdlv = cdl[(size_t)s * nx + ix], sdlv = sdl[(size_t)s * nx + ix];
        const double tmp = sy * sy0[s] + cy * cy0[s] * cdlv;
        const double tmp_c = fmax(-1.0, fmin(1.0, tmp));
        const double g = acos(tmp_c) * R_EARTH;
        const double sin_d = sqrt(fmax(0.0, 1.0 - tmp_c * tmp_c));
        double gx, gy;
        if (sin_d < 1e-14) {
            gx = 0.0;
            gy = 0.0;
        } else {
            gx = cy * cy0[s] * sdlv / sin_d * R_EARTH;
            gy = -(cy * sy0[s] - sy * cy0[s] * cdlv) / sin_d * R_EARTH;
        }
        G[i] = (T)g;
        Gx[i] = (T)gx;
        Gy[i] = (T)gy;
        if (G64) G64[i] = g;
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
size_t batch64_slot_bytes(int nx, int ny, int maxr) {
    return slot_layout<double>(nx, ny, maxr).total;
}

int batch64_max_slots(int device) {
    int nsm = 0, per_sm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<double, true, 0>, 128, 0);
    if (per_sm < 1) per_sm = 1;
    return nsm * per_sm * 4;
}

cudaError_t launch_media64(int nx, int ny, int nper, const double* svel, const double* m11,
                           const double* m12, const double* m22, const double* cosy,
                           double* fun, double* inv3, double* mt, double* b_p, double* a_a,
                           double* c_a, cudaStream_t st) {
    const size_t total = (size_t)nx * ny * nper;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((total + threads - 1) / threads, 148 * 16);
    media64_kernel<<<blocks, threads, 0, st>>>(nx, ny, nper, svel, m11, m12, m22, cosy, fun,
                                                inv3, mt, b_p, a_a, c_a);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_geometry(int nx, int ny, int nsrc, const double* siny, const double* cosy,
                            const double* sy0, const double* cy0, const double* cdl,
                            const double* sdl, T* G, T* Gx, T* Gy, double* G64,
                            cudaStream_t st) {
    const size_t total = (size_t)nx * ny * nsrc;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((total + threads - 1) / threads, 148 * 16);
    geometry_kernel<T><<<blocks, threads, 0, st>>>(nx, ny, nsrc, siny, cosy, sy0, cy0, cdl, sdl,
                                                   G, Gx, Gy, G64);
    return cudaGetLastError();
}
template cudaError_t launch_geometry<double>(int, int, int, const double*, const double*,
                                             const double*, const double*, const double*,
                                             const double*, double*, double*, double*, double*,
                                             cudaStream_t);
template cudaError_t launch_geometry<float>(int, int, int, const double*, const double*,
                                            const double*, const double*, const double*,
                                            const double*, float*, float*, float*, double*,
                                            cudaStream_t);

cudaError_t launch_batch64(const BatchDesc& d, cudaStream_t st) {
    const BatchArgs<double> B = make_batch_args<double>(d);
    const int blocks = (d.sc.nslots + 3) / 4;
    if (d.iso) batch_kernel<double, true, 0><<<blocks, 128, 0, st>>>(B);
    else batch_kernel<double, false, 0><<<blocks, 128, 0, st>>>(B);
    return cudaGetLastError();
}

// The FP64 batch kernel with the grid spacing dx, dy taken from device
// memory (dxdy[0], dxdy[1]) instead of the launch arguments: for callers that
// form the radian grid on the device and must not read it back to the host
// (sa_eik_fwd_field_noalloc).
template <bool ISO>
__global__ void __launch_bounds__(128, SA_MINB64)
batch_kernel_dev_spacing(BatchArgs<double> B, const double* __restrict__ dxdy) {
    BatchArgs<double> Bl = B;
    Bl.g.dx = dxdy[0];
    Bl.g.dy = dxdy[1];
    batch_body<double, ISO, 0>(Bl);
}

cudaError_t launch_batch64_dev_spacing(const BatchDesc& d, const double* dxdy,
                                       cudaStream_t st) {
    const BatchArgs<double> B = make_batch_args<double>(d);
    const int blocks = (d.sc.nslots + 3) / 4;
    if (d.iso) batch_kernel_dev_spacing<true><<<blocks, 128, 0, st>>>(B, dxdy);
    else batch_kernel_dev_spacing<false><<<blocks, 128, 0, st>>>(B, dxdy);
    return cudaGetLastError();
}

// One launch over several plans' events (FP64; see launch_batch32_multi).
cudaError_t launch_batch64_multi(const BatchDesc* d, int nlev, void* dev_args, unsigned ntotal,
                                 const unsigned* code, const Scratch& sc, cudaStream_t st) {
    std::vector<BatchArgs<double>> h(nlev);
    for (int i = 0; i < nlev; i++) h[i] = make_batch_args<double>(d[i]);
    cudaError_t e = cudaMemcpyAsync(dev_args, h.data(), nlev * sizeof(BatchArgs<double>),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    const auto* args = static_cast<const BatchArgs<double>*>(dev_args);
    const int blocks = (sc.nslots + 3) / 4;
    if (d[0].iso) batch_multi_kernel<double, true, 0><<<blocks, 128, 0, st>>>(args, ntotal, code, sc);
    else batch_multi_kernel<double, false, 0><<<blocks, 128, 0, st>>>(args, ntotal, code, sc);
    return cudaGetLastError();
}

size_t batch64_args_bytes() { return sizeof(BatchArgs<double>); }

}  // namespace sa
