// CPU oracle: factored-eikonal fast sweeping, its adjoint, the source mask and
// receiver interpolation.  TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Every expression keeps the reference's association so that, compiled with
// -ffp-contract=off, each intermediate rounds exactly as the reference source
// reads.  Citations are to the reference project.
#include "oracle.h"
#include "eik_state.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

constexpr double PI = 3.14159265358979323846264338327950288;   // include/config.h:54
constexpr double R_EARTH = 6371.0;                             // include/config.h:55
constexpr double DEG2RAD = PI / 180.0;                         // include/config.h:68

inline int at(int nx, int ix, int iy) { return ix + nx * iy; }

// include/utils.h:28-36
inline double bilinear(const double* M, int nx, int idx0, int idy0, double r1, double r2) {
    return (1 - r1) * (1 - r2) * M[at(nx, idx0, idy0)]
         + (1 - r1) * r2 * M[at(nx, idx0, idy0 + 1)]
         + r1 * (1 - r2) * M[at(nx, idx0 + 1, idy0)]
         + r1 * r2 * M[at(nx, idx0 + 1, idy0 + 1)];
}

}  // namespace

// src/eikonal_solver.cpp:22-318, with the stopping rule as a parameter:
// tol > 0 stops as the reference (L1 and Linf of the change below tol,
// reference value 1e-4); tol == 0 iterates to a fixed point (an iteration
// that changes no cell).  `st` (optional) receives the converged state for
// the discrete adjoint (eikonal_discrete.cpp).
int eik_fwd_core(int nx, int ny, const double* xx_deg, const double* yy_deg,
                 const double* spha, const double* sphb, const double* sphc, const double* fun,
                 double x0_deg, double y0_deg, double TOL, int MAXITER, double* T_out,
                 int* niter, EikState* st) {
    if (nx < 3 || ny < 3) return -1;
    const int n = nx * ny;

    std::vector<double> xx(nx), yy(ny);
    for (int i = 0; i < nx; i++) xx[i] = xx_deg[i] * DEG2RAD;
    for (int i = 0; i < ny; i++) yy[i] = yy_deg[i] * DEG2RAD;
    const double x0 = x0_deg * DEG2RAD;
    const double y0 = y0_deg * DEG2RAD;
    const double dx = xx[1] - xx[0];
    const double dy = yy[1] - yy[0];

    // :55-65
    std::vector<double> a(n), b(n), c(n);
    for (int iy = 0; iy < ny; iy++) {
        const double cos_y = std::cos(yy[iy]);
        const double cos2_y = cos_y * cos_y;
        const double R2 = R_EARTH * R_EARTH;
        for (int ix = 0; ix < nx; ix++) {
            const int k = at(nx, ix, iy);
            a[k] = spha[k] / (R2 * cos2_y);
            b[k] = sphb[k] / R2;
            c[k] = sphc[k] / (R_EARTH * R_EARTH * cos_y);
        }
    }

    // :71-82
    int idx0 = static_cast<int>(std::floor((x0 - xx[0]) / dx));
    int idy0 = static_cast<int>(std::floor((y0 - yy[0]) / dy));
    idx0 = std::max(0, std::min(idx0, nx - 2));
    idy0 = std::max(0, std::min(idy0, ny - 2));
    const double r1 = std::min(1.0, (x0 - xx[idx0]) / dx);
    const double r2 = std::min(1.0, (y0 - yy[idy0]) / dy);
    const double fun0 = bilinear(fun, nx, idx0, idy0, r1, r2);

    // :91-131
    std::vector<double> T0(n), T0x(n), T0y(n), tau(n), G(n), Gx(n), Gy(n);
    std::vector<unsigned char> ischange(n, 1);
    for (int ix = 0; ix < nx; ix++) {
        for (int iy = 0; iy < ny; iy++) {
            const int k = at(nx, ix, iy);
            const double dlon = xx[ix] - x0;
            const double tmp = std::sin(yy[iy]) * std::sin(y0)
                             + std::cos(yy[iy]) * std::cos(y0) * std::cos(dlon);
            const double tmp_c = std::max(-1.0, std::min(1.0, tmp));
            // T0 = G fun0 etc., the products associated as the reference
            // writes them (fun0 multiplies last)
            G[k] = std::acos(tmp_c) * R_EARTH;
            T0[k] = G[k] * fun0;
            const double sin_d = std::sqrt(std::max(0.0, 1.0 - tmp_c * tmp_c));
            if (sin_d < 1e-14) {
                Gx[k] = 0.0;
                Gy[k] = 0.0;
                T0x[k] = 0.0;
                T0y[k] = 0.0;
            } else {
                Gx[k] = std::cos(yy[iy]) * std::cos(y0) * std::sin(dlon) / sin_d * R_EARTH;
                Gy[k] = -(std::cos(yy[iy]) * std::sin(y0)
                          - std::sin(yy[iy]) * std::cos(y0) * std::cos(dlon))
                        / sin_d * R_EARTH;
                T0x[k] = Gx[k] * fun0;
                T0y[k] = Gy[k] * fun0;
            }
            if (std::abs((xx[ix] - x0) / dx) <= 1.0 && std::abs((yy[iy] - y0) / dy) <= 1.0) {
                tau[k] = 1.0;
                ischange[k] = 0;
            } else {
                tau[k] = 10.0;
                ischange[k] = 1;
            }
        }
    }

    // :137-140 sweep table
    const int SX0[4] = {0, 0, nx - 1, nx - 1};
    const int SX1[4] = {nx - 1, nx - 1, 0, 0};
    const int SY0[4] = {0, ny - 1, 0, ny - 1};
    const int SY1[4] = {ny - 1, 0, ny - 1, 0};
    const int SXQ[4] = {-1, -1, +1, +1};
    const int SYQ[4] = {-1, +1, -1, +1};

    std::vector<double> tau_old(n);
    double candidates[24];
    int iter = 0;
    int iters_run = 0;
    for (iter = 0; iter < MAXITER; iter++) {
        tau_old = tau;
        iters_run = iter + 1;
        for (int s = 0; s < 4; s++) {
            const int xd = (SX1[s] >= SX0[s]) ? 1 : -1;
            const int yd = (SY1[s] >= SY0[s]) ? 1 : -1;
            for (int ix = SX0[s]; ix != SX1[s] + xd; ix += xd) {
                for (int iy = SY0[s]; iy != SY1[s] + yd; iy += yd) {
                    const int k = at(nx, ix, iy);
                    if (ischange[k] == 0) continue;
                    const double t0 = T0[k];
                    const double t0x = T0x[k];
                    const double t0y = T0y[k];
                    const double aij = a[k];
                    const double bij = b[k];
                    const double cij = c[k];
                    const double fij = fun[k];
                    const double det = aij * bij - cij * cij;
                    int ncand = 0;
                    // A. two-point quadrant stencils, :176-219
                    for (int q = 0; q < 4; q++) {
                        const int sx = SXQ[q], sy = SYQ[q];
                        const int nix = ix + sx, niy = iy + sy;
                        if (nix < 0 || nix >= nx || niy < 0 || niy >= ny) continue;
                        const double px = t0x - sx * (t0 / dx);
                        const double qx = sx * (t0 / dx) * tau[at(nx, ix + sx, iy)];
                        const double py = t0y - sy * (t0 / dy);
                        const double qy = sy * (t0 / dy) * tau[at(nx, ix, iy + sy)];
                        const double eq_a = aij * px * px + bij * py * py - 2.0 * cij * px * py;
                        const double eq_b = 2.0 * (aij * px * qx + bij * py * qy - cij * (px * qy + py * qx));
                        const double eq_c = aij * qx * qx + bij * qy * qy - 2.0 * cij * qx * qy - fij * fij;
                        const double Delta = eq_b * eq_b - 4.0 * eq_a * eq_c;
                        if (Delta < 0.0 || std::abs(eq_a) < 1e-30) continue;
                        const double sq = std::sqrt(Delta);
                        const double two_a = 2.0 * eq_a;
                        for (int sgn = 0; sgn < 2; sgn++) {
                            const double tmp_tau = (-eq_b + (sgn == 0 ? sq : -sq)) / two_a;
                            const double Tx = px * tmp_tau + qx;
                            const double Ty = py * tmp_tau + qy;
                            const double char_x = aij * Tx - cij * Ty;
                            const double char_y = bij * Ty - cij * Tx;
                            if (-sx * char_x >= 0.0 && -sy * char_y >= 0.0)
                                candidates[ncand++] = tmp_tau;
                        }
                    }
                    // B. one-point axis stencils, :224-279
                    if (ix > 0) {
                        const int kn = at(nx, ix - 1, iy);
                        const double px = t0x + t0 / dx;
                        const double qx = -(t0 / dx) * tau[kn];
                        if (det > 0.0) {
                            const double dis = std::sqrt(fij * fij * bij / det);
                            for (int sgn = 0; sgn < 2; sgn++) {
                                const double tmp_tau = ((sgn == 0 ? dis : -dis) - qx) / px;
                                if (tmp_tau * t0 >= tau[kn] * T0[kn] && tmp_tau > tau[kn] * 0.5)
                                    candidates[ncand++] = tmp_tau;
                            }
                        }
                    }
                    if (ix < nx - 1) {
                        const int kn = at(nx, ix + 1, iy);
                        const double px = t0x - t0 / dx;
                        const double qx = (t0 / dx) * tau[kn];
                        if (det > 0.0) {
                            const double dis = std::sqrt(fij * fij * bij / det);
                            for (int sgn = 0; sgn < 2; sgn++) {
                                const double tmp_tau = ((sgn == 0 ? dis : -dis) - qx) / px;
                                if (tmp_tau * t0 >= tau[kn] * T0[kn] && tmp_tau > tau[kn] * 0.5)
                                    candidates[ncand++] = tmp_tau;
                            }
                        }
                    }
                    if (iy > 0) {
                        const int kn = at(nx, ix, iy - 1);
                        const double py = t0y + t0 / dy;
                        const double qy = -(t0 / dy) * tau[kn];
                        if (det > 0.0) {
                            const double dis = std::sqrt(fij * fij * aij / det);
                            for (int sgn = 0; sgn < 2; sgn++) {
                                const double tmp_tau = ((sgn == 0 ? dis : -dis) - qy) / py;
                                if (tmp_tau * t0 >= tau[kn] * T0[kn] && tmp_tau > tau[kn] * 0.5)
                                    candidates[ncand++] = tmp_tau;
                            }
                        }
                    }
                    if (iy < ny - 1) {
                        const int kn = at(nx, ix, iy + 1);
                        const double py = t0y - t0 / dy;
                        const double qy = (t0 / dy) * tau[kn];
                        if (det > 0.0) {
                            const double dis = std::sqrt(fij * fij * aij / det);
                            for (int sgn = 0; sgn < 2; sgn++) {
                                const double tmp_tau = ((sgn == 0 ? dis : -dis) - qy) / py;
                                if (tmp_tau * t0 >= tau[kn] * T0[kn] && tmp_tau > tau[kn] * 0.5)
                                    candidates[ncand++] = tmp_tau;
                            }
                        }
                    }
                    for (int ci = 0; ci < ncand; ci++) tau[k] = std::min(tau[k], candidates[ci]);
                }
            }
        }
        // :292-302
        double L1_dif = 0.0, Linf_dif = 0.0;
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                const int k = at(nx, ix, iy);
                const double d = std::abs(tau[k] - tau_old[k]) * T0[k];
                L1_dif += d;
                Linf_dif = std::max(Linf_dif, d);
            }
        L1_dif /= static_cast<double>(nx * ny);
        if (TOL > 0.0 ? (L1_dif < TOL && Linf_dif < TOL) : (tau == tau_old)) break;
    }
    if (niter) *niter = iters_run;
    for (int k = 0; k < n; k++) T_out[k] = tau[k] * T0[k];
    if (st) {
        st->nx = nx;
        st->ny = ny;
        st->dx = dx;
        st->dy = dy;
        st->fun0 = fun0;
        st->idx0 = idx0;
        st->idy0 = idy0;
        st->r1 = r1;
        st->r2 = r2;
        st->a = std::move(a);
        st->b = std::move(b);
        st->c = std::move(c);
        st->T0 = std::move(T0);
        st->T0x = std::move(T0x);
        st->T0y = std::move(T0y);
        st->G = std::move(G);
        st->Gx = std::move(Gx);
        st->Gy = std::move(Gy);
        st->tau = std::move(tau);
        st->ischange = std::move(ischange);
    }
    return 0;
}

extern "C" int orc_eik_fwd(int nx, int ny, const double* xx_deg, const double* yy_deg,
                           const double* spha, const double* sphb, const double* sphc,
                           const double* fun, double x0_deg, double y0_deg,
                           double* T_out, int* niter) {
    return eik_fwd_core(nx, ny, xx_deg, yy_deg, spha, sphb, sphc, fun, x0_deg, y0_deg, 1e-4,
                        2000, T_out, niter, nullptr);
}

extern "C" int orc_eik_fwd_tol(int nx, int ny, const double* xx_deg, const double* yy_deg,
                               const double* spha, const double* sphb, const double* sphc,
                               const double* fun, double x0_deg, double y0_deg, double tol,
                               int maxiter, double* T_out, int* niter) {
    return eik_fwd_core(nx, ny, xx_deg, yy_deg, spha, sphb, sphc, fun, x0_deg, y0_deg, tol,
                        maxiter, T_out, niter, nullptr);
}

// src/eikonal_solver.cpp:323-511
extern "C" int orc_eik_adj(int nx, int ny, const double* xx_deg, const double* yy_deg,
                           const double* spha, const double* sphb, const double* sphc,
                           const double* T, int nr, const double* xrec_deg,
                           const double* yrec_deg, const double* source_adj,
                           double* Ta_out, int* niter) {
    const double eps = 1e-14;
    const double tol = 1e-9;
    const int maxiter = 1000;
    const int n = nx * ny;

    std::vector<double> xx(nx), yy(ny);
    for (int i = 0; i < nx; i++) xx[i] = xx_deg[i] * DEG2RAD;
    for (int i = 0; i < ny; i++) yy[i] = yy_deg[i] * DEG2RAD;
    const double dx = xx[1] - xx[0];
    const double dy = yy[1] - yy[0];

    // :354-375
    std::vector<double> delta(n, 0.0);
    for (int ir = 0; ir < nr; ir++) {
        const double xrec = xrec_deg[ir] * DEG2RAD;
        const double yrec = yrec_deg[ir] * DEG2RAD;
        int idx0 = static_cast<int>(std::floor((xrec - xx[0]) / dx));
        int idy0 = static_cast<int>(std::floor((yrec - yy[0]) / dy));
        idx0 = std::max(0, std::min(idx0, nx - 2));
        idy0 = std::max(0, std::min(idy0, ny - 2));
        const double r1 = std::min(1.0, (xrec - xx[idx0]) / dx);
        const double r2 = std::min(1.0, (yrec - yy[idy0]) / dy);
        const double area = dx * R_EARTH * std::cos(yrec) * dy * R_EARTH;
        const double w = source_adj[ir] / area;
        delta[at(nx, idx0, idy0)] += w * (1 - r1) * (1 - r2);
        delta[at(nx, idx0, idy0 + 1)] += w * (1 - r1) * r2;
        delta[at(nx, idx0 + 1, idy0)] += w * r1 * (1 - r2);
        delta[at(nx, idx0 + 1, idy0 + 1)] += w * r1 * r2;
    }

    // :380-389
    std::vector<double> a(n), b(n), c(n);
    for (int ix = 0; ix < nx; ix++)
        for (int iy = 0; iy < ny; iy++) {
            const int k = at(nx, ix, iy);
            const double cos_y = std::cos(yy[iy]);
            const double R2 = R_EARTH * R_EARTH;
            a[k] = spha[k] / (R2 * cos_y * cos_y);
            b[k] = sphb[k] / R2;
            c[k] = sphc[k] / (R2 * cos_y);
        }

    // :404-441
    std::vector<double> a1m(n), a1p(n), a2m(n), a2p(n), b1m(n), b1p(n), b2m(n), b2p(n);
    auto Tt = [&](int ix, int iy) { return T[at(nx, ix, iy)]; };
    auto A = [&](int ix, int iy) { return a[at(nx, ix, iy)]; };
    auto B = [&](int ix, int iy) { return b[at(nx, ix, iy)]; };
    auto C = [&](int ix, int iy) { return c[at(nx, ix, iy)]; };
    for (int ix = 1; ix < nx - 1; ix++) {
        for (int iy = 1; iy < ny - 1; iy++) {
            const int k = at(nx, ix, iy);
            const double a1 =
                -(Tt(ix, iy) - Tt(ix - 1, iy)) / dx * (A(ix, iy) + A(ix - 1, iy)) / 2.0
                + (Tt(ix, iy + 1) - Tt(ix, iy - 1) + Tt(ix - 1, iy + 1) - Tt(ix - 1, iy - 1)) / (4.0 * dy)
                  * (C(ix, iy) + C(ix - 1, iy)) / 2.0;
            a1m[k] = (a1 - std::abs(a1)) / 2.0;
            a1p[k] = (a1 + std::abs(a1)) / 2.0;
            const double a2 =
                -(Tt(ix + 1, iy) - Tt(ix, iy)) / dx * (A(ix + 1, iy) + A(ix, iy)) / 2.0
                + (Tt(ix + 1, iy + 1) - Tt(ix + 1, iy - 1) + Tt(ix, iy + 1) - Tt(ix, iy - 1)) / (4.0 * dy)
                  * (C(ix + 1, iy) + C(ix, iy)) / 2.0;
            a2m[k] = (a2 - std::abs(a2)) / 2.0;
            a2p[k] = (a2 + std::abs(a2)) / 2.0;
            const double b1 =
                -(Tt(ix, iy) - Tt(ix, iy - 1)) / dy * (B(ix, iy) + B(ix, iy - 1)) / 2.0
                + (Tt(ix + 1, iy) - Tt(ix - 1, iy) + Tt(ix + 1, iy - 1) - Tt(ix - 1, iy - 1)) / (4.0 * dx)
                  * (C(ix, iy) + C(ix, iy - 1)) / 2.0;
            b1m[k] = (b1 - std::abs(b1)) / 2.0;
            b1p[k] = (b1 + std::abs(b1)) / 2.0;
            const double b2 =
                -(Tt(ix, iy + 1) - Tt(ix, iy)) / dy * (B(ix, iy + 1) + B(ix, iy)) / 2.0
                + (Tt(ix + 1, iy + 1) - Tt(ix - 1, iy + 1) + Tt(ix + 1, iy) - Tt(ix - 1, iy)) / (4.0 * dx)
                  * (C(ix, iy + 1) + C(ix, iy)) / 2.0;
            b2m[k] = (b2 - std::abs(b2)) / 2.0;
            b2p[k] = (b2 + std::abs(b2)) / 2.0;
        }
    }

    // :446-449
    std::vector<double> Ta(n, 0.0);
    for (int ix = 1; ix < nx - 1; ix++)
        for (int iy = 1; iy < ny - 1; iy++) Ta[at(nx, ix, iy)] = 100.0;

    const int IX0[4] = {1, 1, nx - 2, nx - 2};
    const int IX1[4] = {nx - 2, nx - 2, 1, 1};
    const int IY0[4] = {1, ny - 2, 1, ny - 2};
    const int IY1[4] = {ny - 2, 1, ny - 2, 1};

    std::vector<double> Ta_old(n);
    int iters_run = 0;
    for (int iter = 0; iter < maxiter; iter++) {
        Ta_old = Ta;
        iters_run = iter + 1;
        for (int s = 0; s < 4; s++) {
            const int xd = (IX1[s] >= IX0[s]) ? 1 : -1;
            const int yd = (IY1[s] >= IY0[s]) ? 1 : -1;
            for (int ix = IX0[s]; ix != IX1[s] + xd; ix += xd) {
                for (int iy = IY0[s]; iy != IY1[s] + yd; iy += yd) {
                    const int k = at(nx, ix, iy);
                    const double d = (a2p[k] - a1m[k]) / dx + (b2p[k] - b1m[k]) / dy;
                    if (std::abs(d) < eps) {
                        Ta[k] = 0.0;
                    } else {
                        const double e =
                            (Ta[at(nx, ix - 1, iy)] * a1p[k] - Ta[at(nx, ix + 1, iy)] * a2m[k]) / dx +
                            (Ta[at(nx, ix, iy - 1)] * b1p[k] - Ta[at(nx, ix, iy + 1)] * b2m[k]) / dy;
                        Ta[k] = (delta[k] + e) / d;
                    }
                }
            }
        }
        double L1_dif = 0.0, Linf_dif = 0.0;
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                const int k = at(nx, ix, iy);
                const double dd = std::abs(Ta[k] - Ta_old[k]);
                L1_dif += dd;
                Linf_dif = std::max(Linf_dif, dd);
            }
        L1_dif /= static_cast<double>(nx * ny);
        if (L1_dif < tol && Linf_dif < tol) break;
    }
    if (niter) *niter = iters_run;
    std::copy(Ta.begin(), Ta.end(), Ta_out);
    return 0;
}

// src/eikonal_solver.cpp:514-536
extern "C" void orc_mask_uniform_grid(int nx, int ny, const double* xx, const double* yy,
                                      double* table, double x0, double y0) {
    if (nx < 2 || ny < 2) return;
    const double dx = xx[1] - xx[0];
    const double dy = yy[1] - yy[0];
    const int ix_lo = std::max(0, static_cast<int>(std::floor((x0 - 1.5 * dx - xx[0]) / dx)) + 1);
    const int ix_hi = std::min(nx - 1, static_cast<int>(std::ceil((x0 + 1.5 * dx - xx[0]) / dx)) - 1);
    const int iy_lo = std::max(0, static_cast<int>(std::floor((y0 - 1.5 * dy - yy[0]) / dy)) + 1);
    const int iy_hi = std::min(ny - 1, static_cast<int>(std::ceil((y0 + 1.5 * dy - yy[0]) / dy)) - 1);
    if (ix_lo <= ix_hi && iy_lo <= iy_hi) {
        for (int iy = iy_lo; iy <= iy_hi; iy++)
            for (int ix = ix_lo; ix <= ix_hi; ix++) table[at(nx, ix, iy)] = 0.0;
    }
}

// include/utils.h:358-409
extern "C" void orc_interp2d(int nx, int ny, const double* xgrid, const double* ygrid,
                             const double* z, int nq, const double* xq, const double* yq,
                             double* zq) {
    for (int k = 0; k < nq; ++k) {
        const double qx = xq[k];
        const double qy = yq[k];
        if (qx < xgrid[0] || qx > xgrid[nx - 1] || qy < ygrid[0] || qy > ygrid[ny - 1]) {
            zq[k] = std::nan("");
            continue;
        }
        int i = static_cast<int>(std::lower_bound(xgrid, xgrid + nx, qx) - xgrid);
        if (i == nx) --i;
        if (i > 0 && xgrid[i] > qx) --i;
        i = std::clamp(i, 0, nx - 2);
        int j = static_cast<int>(std::lower_bound(ygrid, ygrid + ny, qy) - ygrid);
        if (j == ny) --j;
        if (j > 0 && ygrid[j] > qy) --j;
        j = std::clamp(j, 0, ny - 2);
        const double x1 = xgrid[i], x2 = xgrid[i + 1];
        const double y1 = ygrid[j], y2 = ygrid[j + 1];
        const double tx = (qx - x1) / (x2 - x1);
        const double ty = (qy - y1) / (y2 - y1);
        zq[k] = (1 - tx) * (1 - ty) * z[at(nx, i, j)]
              + (tx) * (1 - ty) * z[at(nx, i + 1, j)]
              + (1 - tx) * (ty) * z[at(nx, i, j + 1)]
              + (tx) * (ty) * z[at(nx, i + 1, j + 1)];
    }
}
