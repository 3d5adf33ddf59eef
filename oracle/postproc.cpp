// CPU oracle: PDE kernel smoothing.  TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// PostProc::pde_smooth (src/postproc.cpp:388-463) on one rank (no domain
// decomposition): explicit Euler steps of the spherical Laplacian
// (compute_laplacian_3d_standard, :35-128) followed by the Neumann boundary
// copies (apply_boundary_conditions, :130-158).  Fields are row-major
// (nx, ny, nz), depth fastest, as Tensor3r.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {
constexpr double PI = 3.14159265358979323846264338327950288;   // include/config.h:54
constexpr double R_EARTH = 6371.0;                             // include/config.h:55
constexpr double DEG2RAD = PI / 180.0;                         // include/config.h:68
}  // namespace

extern "C" int orc_pde_smooth_nstep(int ny, double dx, double dy, double dz, double y_first,
                                    double y_last, double sigma_h, double sigma_v, double* ch,
                                    double* cv) {
    (void)ny;
    if (sigma_h <= 0.0 || sigma_v <= 0.0) return -1;   // :397-400
    // :407-413
    double lat_max = std::max(std::abs(y_first), std::abs(y_last));
    lat_max = std::min(lat_max, 89.0);
    const double cos2_lat_max = std::pow(std::cos(lat_max * DEG2RAD), 2);
    const double cmax_h = std::min(dx * dx * cos2_lat_max, dy * dy) / 6.0;
    const double cmax_v = dz * dz / 6.0;
    if (cmax_h <= 1e-12 || cmax_v <= 1e-12) return -2;   // :414-417
    const double dt = 1.0;
    // :425-434
    const int nstep_h = static_cast<int>(std::ceil(sigma_h * sigma_h / (2.0 * cmax_h * dt)));
    const int nstep_v = static_cast<int>(std::ceil(sigma_v * sigma_v / (2.0 * cmax_v * dt)));
    const int nstep = std::max({nstep_h, nstep_v, 1});
    *ch = sigma_h * sigma_h / (2.0 * nstep * dt);
    *cv = sigma_v * sigma_v / (2.0 * nstep * dt);
    return nstep;
}

extern "C" int orc_pde_smooth(int nx, int ny, int nz, double dx, double dy, double dz,
                              const double* ygrid, const double* zgrid, double sigma_h,
                              double sigma_v, double* field, int* nstep_out) {
    if (nx < 3 || ny < 3 || nz < 3) return -3;
    double ch = 0, cv = 0;
    const int nstep = orc_pde_smooth_nstep(ny, dx, dy, dz, ygrid[0], ygrid[ny - 1], sigma_h,
                                           sigma_v, &ch, &cv);
    if (nstep < 0) return nstep;
    if (nstep_out) *nstep_out = nstep;
    const size_t n = (size_t)nx * ny * nz;
    auto at = [&](int ix, int iy, int k) { return ((size_t)ix * ny + iy) * nz + k; };
    std::vector<double> u(field, field + n), lap(n);
    // :74-78
    const double dx2_inv = 1.0 / (dx * dx);
    const double dy2_inv = 1.0 / (dy * dy);
    const double dz2_inv = 1.0 / (dz * dz);
    const double dy_inv_half = 1.0 / (2.0 * dy);
    const double dz_inv_half = 1.0 / (2.0 * dz);
    for (int istep = 0; istep < nstep; ++istep) {
        std::fill(lap.begin(), lap.end(), 0.0);
        // :81-126 (single rank: ix in [1, nx-1), iy in [1, ny-1), all k).  The
        // expanded field has no depth halo: at k = 0 and nz-1 the reference's
        // row-major tensor reads the neighbouring column's first/last sample;
        // those planes are overwritten by the boundary copies below.
        const double* e = u.data();
        for (int ix = 1; ix < nx - 1; ++ix) {
            for (int iy = 1; iy < ny - 1; ++iy) {
                // y_loc_expd(iy) = ygrids(0) + iy * dgrid_j (src/decomposer.cpp:116-118)
                const double lat_rad = (ygrid[0] + iy * dy) * DEG2RAD;
                const double cos_lat = std::cos(lat_rad);
                const double dy2_corr_inv = 1.0 / (cos_lat * cos_lat);
                const double tan_lat = std::tan(lat_rad);
                for (int k = 0; k < nz; ++k) {
                    const size_t c = at(ix, iy, 0) + k;
                    const double center = e[c];
                    const double d2u_dx2 = ch * dx2_inv * dy2_corr_inv *
                                           (e[c + (size_t)ny * nz] + e[c - (size_t)ny * nz] - 2.0 * center);
                    const double u_jp1 = e[c + nz];
                    const double u_jm1 = e[c - nz];
                    const double d2u_dy2 = ch * dy2_inv * (u_jp1 + u_jm1 - 2.0 * center);
                    const double du_dy = ch * DEG2RAD * tan_lat * dy_inv_half * (u_jp1 - u_jm1);
                    const double lat_term = d2u_dy2 - du_dy;
                    const double u_kp1 = e[c + 1];
                    const double u_km1 = e[c - 1];
                    const double d2u_dz2 = cv * dz2_inv * (u_kp1 + u_km1 - 2.0 * center);
                    const double r_inv = 2.0 / (R_EARTH - zgrid[k]);
                    const double du_dz = cv * r_inv * dz_inv_half * (u_kp1 - u_km1);
                    const double depth_term = d2u_dz2 - du_dz;
                    lap[c] = d2u_dx2 + lat_term + depth_term;
                }
            }
        }
        // :453 smoothed_buf = smoothed_buf + dt * lap (dt = 1)
        for (size_t i = 0; i < n; ++i) u[i] = u[i] + 1.0 * lap[i];
        // :130-158
        for (int iy = 0; iy < ny; ++iy)
            for (int k = 0; k < nz; ++k) u[at(0, iy, k)] = u[at(1, iy, k)];
        for (int iy = 0; iy < ny; ++iy)
            for (int k = 0; k < nz; ++k) u[at(nx - 1, iy, k)] = u[at(nx - 2, iy, k)];
        for (int ix = 0; ix < nx; ++ix)
            for (int k = 0; k < nz; ++k) u[at(ix, 0, k)] = u[at(ix, 1, k)];
        for (int ix = 0; ix < nx; ++ix)
            for (int k = 0; k < nz; ++k) u[at(ix, ny - 1, k)] = u[at(ix, ny - 2, k)];
        for (int ix = 0; ix < nx; ++ix)
            for (int iy = 0; iy < ny; ++iy) {
                u[at(ix, iy, 0)] = u[at(ix, iy, 1)];
                u[at(ix, iy, nz - 1)] = u[at(ix, iy, nz - 2)];
            }
    }
    std::copy(u.begin(), u.end(), field);
    return 0;
}

// ---- multigrid smoothing (smooth_method 1) --------------------------------
// PostProc::InvGrid::init / fwd2inv / inv2fwd (src/postproc.cpp:160-386) and
// PostProc::smooth (:465-480): nset staggered coarse grids of
// (n_inv + 2) nodes per axis; the field is projected onto them and
// interpolated back, averaged over the sets.  Kept as the reference has it:
// fwd2inv adds each fine node to one corner only (the one of n = 7: its
// accumulation sits after the corner loop), and the coarse index uses the
// inner counts n_inv_J, n_inv_K as strides (I2V_INV_GRIDS,
// include/postproc.h:53-55).
namespace {
int locate_bissection(const double* v, int n, double x) {   // include/utils.h:39-60
    int low = 0, high = n - 1;
    if (x < v[0] || x > v[n - 1]) return -1;
    while (high - low > 1) {
        const int mid = (high + low) / 2;
        if (v[mid] > x) high = mid;
        else low = mid;
    }
    if (x == v[0]) return 0;
    if (x == v[n - 1]) return n - 2;
    return low;
}

struct InvGrid {
    int nI, nJ, nK, nset;
    std::vector<double> xinv, yinv, zinv;   // [set][node]
    int idx(int A, int B, int C, int D) const { return A * nK * nJ * nset + B * nK * nset + C * nset + D; }
};

InvGrid inv_grid_init(const double* x, int nx, const double* y, int ny, const double* z, int nz,
                      const int* n_inv, int nset) {
    InvGrid G{n_inv[0], n_inv[1], n_inv[2], nset, {}, {}, {}};
    auto axis = [&](const double* g, int n, int ninner, std::vector<double>& out) {
        const int m = ninner + 2;
        const double g0 = g[0], g1 = g[n - 1];
        const double d = (g1 - g0) / ninner;
        const double add = d / nset;
        const double beg = g0 - add, end = g1 + add;
        out.assign((size_t)m * nset, 0.0);
        for (int is = 0; is < nset; ++is) {
            double* o = out.data() + (size_t)is * m;
            o[0] = beg;
            o[m - 1] = end;
            for (int j = 1; j < m - 1; ++j) o[j] = (g0 + (j - 1) * d) + is * add;
        }
    };
    axis(x, nx, G.nI, G.xinv);
    axis(y, ny, G.nJ, G.yinv);
    axis(z, nz, G.nK, G.zinv);
    return G;
}
}  // namespace

// buf, out: (nx, ny, nz) row-major.  Returns -1 when a node lies outside a
// coarse grid (the reference aborts).
extern "C" int orc_multigrid_smooth(int nx, int ny, int nz, const double* x, const double* y,
                                    const double* z, const int* n_inv, int nset,
                                    const double* buf, double* out) {
    const InvGrid G = inv_grid_init(x, nx, y, ny, z, nz, n_inv, nset);
    const int mx = G.nI + 2, my = G.nJ + 2, mz = G.nK + 2;
    const size_t ngrid = (size_t)mx * my * mz * nset;
    std::vector<double> tmp(ngrid, 0.0), weight(ngrid, 0.0), arr(ngrid, 0.0);
    for (int ig = 0; ig < nset; ++ig) {
        const double* xi = G.xinv.data() + (size_t)ig * mx;
        const double* yi = G.yinv.data() + (size_t)ig * my;
        const double* zi = G.zinv.data() + (size_t)ig * mz;
        for (int i = 0; i < nx; ++i) {
            const int ix = locate_bissection(xi, mx, x[i]);
            if (ix < 0) return -1;
            const double wx = (x[i] - xi[ix]) / (xi[ix + 1] - xi[ix]);
            for (int j = 0; j < ny; ++j) {
                const int iy = locate_bissection(yi, my, y[j]);
                if (iy < 0) return -1;
                const double wy = (y[j] - yi[iy]) / (yi[iy + 1] - yi[iy]);
                for (int k = 0; k < nz; ++k) {
                    const int iz = locate_bissection(zi, mz, z[k]);
                    if (iz < 0) return -1;
                    const double wz = (z[k] - zi[iz]) / (zi[iz + 1] - zi[iz]);
                    const int m = G.idx(ix + 1, iy, iz + 1, ig);   // the n = 7 corner
                    const double wt = wx * (1.0 - wy) * wz;
                    weight[m] += wt;
                    tmp[m] += wt * buf[((size_t)i * ny + j) * nz + k];
                }
            }
        }
    }
    for (size_t i = 0; i < ngrid; ++i) arr[i] = weight[i] > 0.0 ? tmp[i] / weight[i] : 0.0;
    for (size_t i = 0; i < (size_t)nx * ny * nz; ++i) out[i] = 0.0;
    for (int ig = 0; ig < nset; ++ig) {
        const double* xi = G.xinv.data() + (size_t)ig * mx;
        const double* yi = G.yinv.data() + (size_t)ig * my;
        const double* zi = G.zinv.data() + (size_t)ig * mz;
        for (int i = 0; i < nx; ++i) {
            const int ix = locate_bissection(xi, mx, x[i]);
            const double wx = (x[i] - xi[ix]) / (xi[ix + 1] - xi[ix]);
            for (int j = 0; j < ny; ++j) {
                const int iy = locate_bissection(yi, my, y[j]);
                const double wy = (y[j] - yi[iy]) / (yi[iy + 1] - yi[iy]);
                for (int k = 0; k < nz; ++k) {
                    const int iz = locate_bissection(zi, mz, z[k]);
                    const double wz = (z[k] - zi[iz]) / (zi[iz + 1] - zi[iz]);
                    const int c[8][3] = {{ix, iy, iz},         {ix, iy + 1, iz},
                                         {ix + 1, iy + 1, iz}, {ix + 1, iy, iz},
                                         {ix, iy, iz + 1},     {ix, iy + 1, iz + 1},
                                         {ix + 1, iy + 1, iz + 1}, {ix + 1, iy, iz + 1}};
                    const double w[8] = {(1.0 - wx) * (1.0 - wy) * (1.0 - wz),
                                         (1.0 - wx) * wy * (1.0 - wz),
                                         wx * wy * (1.0 - wz),
                                         wx * (1.0 - wy) * (1.0 - wz),
                                         (1.0 - wx) * (1.0 - wy) * wz,
                                         (1.0 - wx) * wy * wz,
                                         wx * wy * wz,
                                         wx * (1.0 - wy) * wz};
                    double val = 0.0;
                    for (int n = 0; n < 8; ++n) val += w[n] * arr[G.idx(c[n][0], c[n][1], c[n][2], ig)];
                    out[((size_t)i * ny + j) * nz + k] += val;
                }
            }
        }
    }
    for (size_t i = 0; i < (size_t)nx * ny * nz; ++i) out[i] = out[i] / static_cast<double>(nset);
    return 0;
}
