// Media matrices from topography (SurfGrid::build_media_matrix_with_topo,
// reference src/surf_grid.cpp:80-166) and the kernel-depth correction
// (SurfGrid::correct_depth_with_topo, :307-354), on device.
//   gauss_geo_kernel   gaussian_smooth_geo_2 (include/utils.h:505-571): one
//                      thread per output cell, haversine-distance Gaussian
//                      weights over the lon/lat window; the window's latitude
//                      terms are shared by the block (one block per row).
//   media_kernel       gradient_2_geo (:593-649), dip angle (src/topo.cpp:97-114)
//                      and m11 = a, m12 = -c, m22 = b per cell.
//   depth_topo_kernel  per (column, period): depth nodes stretched by
//                      1/cos(dip), clamped, linear interpolation (utils.h:451-485).
//   grid_kernel        interp2d onto the model grid (Topography::grid).
// Compiled with -fmad=false; sin/cos/atan/exp are CUDA's (ulp-level
// differences from the C library), so parity is to a stated tolerance.
#include "event_common.cuh"
#include "launch.h"

namespace sa {

namespace {
constexpr double PI_T = 3.14159265358979323846264338327950288;
constexpr double DEG2RAD_T = PI_T / 180.0;
constexpr double RAD2DEG_T = 180.0 / PI_T;
constexpr double R_EARTH_T = 6371.0;

__global__ void gauss_geo_kernel(int nx, int ny, const double* __restrict__ data,
                                 const double* __restrict__ lons, const double* __restrict__ lats,
                                 double sigma, double* __restrict__ out) {
    extern __shared__ double sh[];   // [2][wn]: sin^2(dlat/2), cos(lat1)
    const int j = blockIdx.y;
    const double sigma3 = 3.0 * sigma;
    const double dx = lons[1] - lons[0];
    const double dy = lats[1] - lats[0];
    const int hx = static_cast<int>(sigma3 / dx);
    const double cos_lat0 = cos(lats[j] * DEG2RAD_T);
    const int hy = static_cast<int>(sigma3 / cos_lat0 / dy);
    const int n1 = max(0, j - hy);
    const int n2 = min(ny - 1, j + hy);
    const int wn = n2 - n1 + 1;
    double* s2lat = sh;
    double* clat1 = sh + wn;
    for (int q = threadIdx.x; q < wn; q += blockDim.x) {
        const double s = sin((lats[n1 + q] - lats[j]) * (DEG2RAD_T * 0.5));
        s2lat[q] = s * s;
        clat1[q] = cos(lats[n1 + q] * DEG2RAD_T);
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx) return;
    const double inv_2sig2 = 1.0 / (2.0 * (sigma * sigma));
    const double two_rad2deg = 2.0 * RAD2DEG_T;
    const int m1 = max(0, i - hx);
    const int m2 = min(nx - 1, i + hx);
    double sw = 0.0, swd = 0.0;
    for (int m = m1; m <= m2; m++) {
        const double s = sin((lons[m] - lons[i]) * (DEG2RAD_T * 0.5));
        const double lon_c = cos_lat0 * (s * s);
        const double* col = data + m;
        for (int q = 0; q < wn; q++) {
            double a = s2lat[q] + lon_c * clat1[q];
            a = fmin(a, 1.0);
            const double t = two_rad2deg * atan(sqrt(a / (1.0 - a)));
            const double w = exp(-(t * t) * inv_2sig2);
            sw += w;
            swd += w * col[(size_t)nx * (n1 + q)];
        }
    }
    out[i + (size_t)nx * j] = swd / sw;
}

__global__ void media_kernel(int nx, int ny, const double* __restrict__ z,
                             const double* __restrict__ lon, const double* __restrict__ lat,
                             double* m11, double* m12, double* m22, double* angle) {
    const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= (size_t)nx * ny) return;
    const int i = (int)(k % nx), j = (int)(k / nx);
    const double km = R_EARTH_T * DEG2RAD_T;
    const double clat = cos(lat[j] * DEG2RAD_T);
    auto F = [&](int a, int b) { return z[a + (size_t)nx * b]; };
    auto dxk = [&](int a) { return (lon[a] - lon[a - 1]) * km; };
    auto dyk = [&](int b) { return (lat[b] - lat[b - 1]) * km; };
    double fx, fy;
    if (i == 0) fx = (F(1, j) - F(0, j)) / (dxk(1) * clat);
    else if (i == nx - 1) fx = (F(nx - 1, j) - F(nx - 2, j)) / (dxk(nx - 1) * clat);
    else fx = (F(i + 1, j) - F(i - 1, j)) / (2.0 * (dxk(i) * clat));
    if (j == 0) fy = (F(i, 1) - F(i, 0)) / (1.0 * dyk(1));
    else if (j == ny - 1) fy = (F(i, ny - 1) - F(i, ny - 2)) / (1.0 * dyk(ny - 1));
    else fy = (F(i, j + 1) - F(i, j - 1)) / (2.0 * (1.0 * dyk(j)));
    const double fx2 = fx * fx, fy2 = fy * fy;
    angle[k] = atan(sqrt(fx2 + fy2)) * RAD2DEG_T;
    const double denom = 1.0 + fx2 + fy2;
    m11[k] = (1.0 + fy2) / denom;
    m22[k] = (1.0 + fx2) / denom;
    m12[k] = -(fx * fy / denom);
}

__global__ void depth_topo_kernel(int nx, int ny, int nz, int nper, const double* __restrict__ zg,
                                  const double* __restrict__ angle, double* k0, double* k1,
                                  double* k2) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= (size_t)nx * ny * nper) return;
    const int ip = (int)(t % nper);
    const size_t col = t / nper;
    const int iy = (int)(col % ny), ix = (int)(col / ny);
    double cosang = cos(angle[(size_t)ip * nx * ny + ix + (size_t)nx * iy] * DEG2RAD_T);
    if (!isfinite(cosang) || fabs(cosang) < 1e-6) cosang = 1e-6;
    const double zmin = zg[0], zmax = zg[nz - 1];
    const size_t base = col * nz * nper + ip;
    double* ks[3] = {k0, k1, k2};
    double c[64];
    for (int a = 0; a < 3; a++) {
        double* K = ks[a];
        if (!K) continue;
        for (int q = 0; q < nz; q++) c[q] = K[base + (size_t)q * nper];
        for (int q = 0; q < nz; q++) {
            const double qx = fmin(fmax(zg[q] / cosang, zmin), zmax);
            double v;
            if (qx < zg[0]) v = c[0];
            else if (qx > zg[nz - 1]) v = c[nz - 1];
            else {
                int lo = 0, hi = nz;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (zg[mid] < qx) lo = mid + 1;
                    else hi = mid;
                }
                int i = lo;
                if (i == nz) --i;
                if (i > 0 && zg[i] > qx) --i;
                i = max(0, min(i, nz - 2));
                const double x1 = zg[i], x2 = zg[i + 1];
                const double tt = (qx - x1) / (x2 - x1);
                v = (1 - tt) * c[i] + tt * c[i + 1];
            }
            K[base + (size_t)q * nper] = v;
        }
    }
}

__global__ void grid_kernel(int nxr, int nyr, const double* __restrict__ xr,
                            const double* __restrict__ yr, const double* __restrict__ zr, int nx,
                            int ny, const double* __restrict__ x, const double* __restrict__ y,
                            double* out) {
    const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= (size_t)nx * ny) return;
    const int i = (int)(k % nx), j = (int)(k / nx);
    out[k] = interp2d_pt(xr, nxr, yr, nyr, zr, x[i], y[j]);
}
}  // namespace

cudaError_t launch_gauss_geo(int nx, int ny, const double* data, const double* lons,
                             const double* lats, double sigma, double* out, cudaStream_t st) {
    dim3 grid((nx + 127) / 128, ny);
    gauss_geo_kernel<<<grid, 128, 2 * ny * sizeof(double), st>>>(nx, ny, data, lons, lats, sigma,
                                                                 out);
    return cudaGetLastError();
}

cudaError_t launch_topo_media(int nx, int ny, const double* z, const double* lon,
                              const double* lat, double* m11, double* m12, double* m22,
                              double* angle, cudaStream_t st) {
    const size_t n = (size_t)nx * ny;
    media_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nx, ny, z, lon, lat, m11, m12, m22,
                                                              angle);
    return cudaGetLastError();
}

cudaError_t launch_depth_topo(int nx, int ny, int nz, int nper, const double* zg,
                              const double* angle, double* k0, double* k1, double* k2,
                              cudaStream_t st) {
    const size_t n = (size_t)nx * ny * nper;
    depth_topo_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(nx, ny, nz, nper, zg, angle, k0,
                                                                   k1, k2);
    return cudaGetLastError();
}

cudaError_t launch_grid_topo(int nxr, int nyr, const double* xr, const double* yr,
                             const double* zr, int nx, int ny, const double* x, const double* y,
                             double* out, cudaStream_t st) {
    const size_t n = (size_t)nx * ny;
    grid_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nxr, nyr, xr, yr, zr, nx, ny, x, y,
                                                             out);
    return cudaGetLastError();
}

}  // namespace sa
