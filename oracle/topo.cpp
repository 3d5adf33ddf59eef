// CPU oracle: media matrices from topography and the kernel-depth correction.
// TEST INFRASTRUCTURE ONLY (see oracle.h).
//   gaussian_smooth_geo_2   include/utils.h:505-571
//   gradient_2_geo          include/utils.h:593-649
//   Topography::calc_dip_angle  src/topo.cpp:97-114
//   SurfGrid::build_media_matrix_with_topo, per period  src/surf_grid.cpp:80-166
//   SurfGrid::correct_depth_with_topo  src/surf_grid.cpp:307-354 (interp1d utils.h:451-485)
// 2-D fields are column-major (nx x ny); per-period outputs are [iper][iy][ix].
// Window sums run in column-major order over the window (lon fastest).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {
constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double R_EARTH = 6371.0;
constexpr double DEG2RAD = PI / 180.0;
constexpr double RAD2DEG = 180.0 / PI;
}  // namespace

extern "C" void orc_gaussian_smooth_geo_2(int nx, int ny, const double* data, const double* lons,
                                          const double* lats, double sigma, double* out) {
    const double sigma3 = 3.0 * sigma;
    const double sigma_sq = sigma * sigma;
    const double dx = lons[1] - lons[0];
    const double dy = lats[1] - lats[0];
    const int hx = static_cast<int>(sigma3 / dx);
    const double inv_2sig2 = 1.0 / (2.0 * sigma_sq);
    const double two_rad2deg = 2.0 * RAD2DEG;
    std::vector<double> sin2_dlat, cos_lat1, sin2_dlon;
    for (int j = 0; j < ny; ++j) {
        const double lat0_rad = lats[j] * DEG2RAD;
        const double cos_lat0 = std::cos(lat0_rad);
        const int hy = static_cast<int>(sigma3 / cos_lat0 / dy);
        const int n1 = std::max(0, j - hy);
        const int n2 = std::min(ny - 1, j + hy);
        const int wn = n2 - n1 + 1;
        sin2_dlat.assign(wn, 0.0);
        cos_lat1.assign(wn, 0.0);
        for (int q = 0; q < wn; ++q) {
            const double s = std::sin((lats[n1 + q] - lats[j]) * (DEG2RAD * 0.5));
            sin2_dlat[q] = s * s;
            cos_lat1[q] = std::cos(lats[n1 + q] * DEG2RAD);
        }
        for (int i = 0; i < nx; ++i) {
            const int m1 = std::max(0, i - hx);
            const int m2 = std::min(nx - 1, i + hx);
            const int wm = m2 - m1 + 1;
            sin2_dlon.assign(wm, 0.0);
            for (int p = 0; p < wm; ++p) {
                const double s = std::sin((lons[m1 + p] - lons[i]) * (DEG2RAD * 0.5));
                sin2_dlon[p] = cos_lat0 * (s * s);   // lon_contrib
            }
            double sw = 0.0, swd = 0.0;
            for (int q = 0; q < wn; ++q)
                for (int p = 0; p < wm; ++p) {
                    double a = sin2_dlat[q] + sin2_dlon[p] * cos_lat1[q];
                    a = std::min(a, 1.0);
                    const double t = two_rad2deg * std::atan(std::sqrt(a / (1.0 - a)));
                    const double w = std::exp(-(t * t) * inv_2sig2);
                    sw += w;
                    swd += w * data[(m1 + p) + (size_t)nx * (n1 + q)];
                }
            out[i + (size_t)nx * j] = swd / sw;
        }
    }
}

extern "C" void orc_gradient_2_geo(int nx, int ny, const double* f, const double* lon,
                                   const double* lat, double* tx, double* ty) {
    std::vector<double> dx1(nx, 0.0), dy1(ny, 0.0), cos_lat(ny);
    for (int i = 1; i < nx; i++) dx1[i] = lon[i] - lon[i - 1];
    for (int j = 1; j < ny; j++) dy1[j] = lat[j] - lat[j - 1];
    for (int j = 0; j < ny; j++) cos_lat[j] = std::cos(lat[j] * DEG2RAD);
    const double km = R_EARTH * DEG2RAD;
    for (int i = 0; i < nx; i++) dx1[i] *= km;
    for (int j = 0; j < ny; j++) dy1[j] *= km;
    auto F = [&](int i, int j) { return f[i + (size_t)nx * j]; };
    for (int j = 0; j < ny; j++) {
        for (int i = 1; i < nx - 1; i++)
            tx[i + (size_t)nx * j] = (F(i + 1, j) - F(i - 1, j)) / (2.0 * (dx1[i] * cos_lat[j]));
        tx[0 + (size_t)nx * j] = (F(1, j) - F(0, j)) / (dx1[1] * cos_lat[j]);
        tx[(nx - 1) + (size_t)nx * j] = (F(nx - 1, j) - F(nx - 2, j)) / (dx1[nx - 1] * cos_lat[j]);
    }
    for (int i = 0; i < nx; i++) {
        for (int j = 1; j < ny - 1; j++)
            ty[i + (size_t)nx * j] = (F(i, j + 1) - F(i, j - 1)) / (2.0 * (1.0 * dy1[j]));
        ty[i] = (F(i, 1) - F(i, 0)) / (1.0 * dy1[1]);
        ty[i + (size_t)nx * (ny - 1)] = (F(i, ny - 1) - F(i, ny - 2)) / (1.0 * dy1[ny - 1]);
    }
}

extern "C" void orc_topo_media(int nx, int ny, const double* lon, const double* lat,
                               const double* z_gridded, int nper, const double* sigma_deg,
                               double* m11, double* m12, double* m22, double* angle) {
    const size_t n = (size_t)nx * ny;
    std::vector<double> z(n), fx(n), fy(n);
    for (int ip = 0; ip < nper; ip++) {
        orc_gaussian_smooth_geo_2(nx, ny, z_gridded, lon, lat, sigma_deg[ip], z.data());
        orc_gradient_2_geo(nx, ny, z.data(), lon, lat, fx.data(), fy.data());
        for (size_t k = 0; k < n; k++) {
            const double ang = std::atan(std::sqrt(fx[k] * fx[k] + fy[k] * fy[k]));
            angle[ip * n + k] = ang * RAD2DEG;
            const double fx2 = fx[k] * fx[k], fy2 = fy[k] * fy[k];
            const double denom = 1.0 + fx2 + fy2;
            m11[ip * n + k] = (1.0 + fy2) / denom;
            m22[ip * n + k] = (1.0 + fx2) / denom;
            m12[ip * n + k] = -(fx[k] * fy[k] / denom);
        }
    }
}

extern "C" void orc_correct_depth_with_topo(int nx, int ny, int nz, int nper, const double* zgrid,
                                            const double* angle, double* ker) {
    const double zmin = zgrid[0], zmax = zgrid[nz - 1];
    std::vector<double> col(nz), newz(nz);
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy)
            for (int ip = 0; ip < nper; ++ip) {
                const double a = angle[(size_t)ip * nx * ny + ix + (size_t)nx * iy];
                double cosang = std::cos(a * DEG2RAD);
                if (!std::isfinite(cosang) || std::abs(cosang) < 1e-6) cosang = 1e-6;
                for (int k = 0; k < nz; k++) newz[k] = std::min(std::max(zgrid[k] / cosang, zmin), zmax);
                const size_t base = (((size_t)ix * ny + iy) * nz) * nper + ip;
                for (int k = 0; k < nz; k++) col[k] = ker[base + (size_t)k * nper];
                for (int k = 0; k < nz; k++) {
                    const double qx = newz[k];
                    double v;
                    if (qx < zgrid[0]) v = col[0];
                    else if (qx > zgrid[nz - 1]) v = col[nz - 1];
                    else {
                        int i = (int)(std::lower_bound(zgrid, zgrid + nz, qx) - zgrid);
                        if (i == nz) --i;
                        if (i > 0 && zgrid[i] > qx) --i;
                        i = std::clamp(i, 0, nz - 2);
                        const double x1 = zgrid[i], x2 = zgrid[i + 1];
                        const double t = (qx - x1) / (x2 - x1);
                        v = (1 - t) * col[i] + t * col[i + 1];
                    }
                    ker[base + (size_t)k * nper] = v;
                }
            }
}
