// CPU oracle: the exact discrete adjoint of the factored-eikonal forward
// solve.  TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// The reference's adjoint (src/eikonal_solver.cpp:323-511) discretises the
// continuous adjoint transport equation; its kernel differs from the
// derivative of the discrete forward map by the discretisation error.  This
// file differentiates the discrete map itself.  At a fixed point of the fast
// sweeping iteration (src/eikonal_solver.cpp:145-303) every free cell k
// satisfies tau_k = Phi_k(tau_x, tau_y, f_k, t0_k, t0x_k, t0y_k): the
// smallest admissible candidate of :176-279, a root of the quadrant
// quadratic (two upwind neighbours) or an axis update (one neighbour).  With
// T = tau T0 (:317), T0 = G fun0, fun0 the bilinear slowness at the source
// (:71-82), and the receiver times by interp2d (include/utils.h:358-409):
//   lambda = g + J^T lambda,  g_k = sum_r dchi/dT_r beta_rk T0_k,
//   J_kj = dPhi_k / dtau_j (j one of the winning candidate's neighbours),
//   dchi/dfun_m = lambda_m dPhi_m/df_m + alpha_m S,
//   S = sum_k lambda_k (dPhi_k/dt0 G_k + dPhi_k/dt0x Gx_k + dPhi_k/dt0y Gy_k)
//       + sum_r dchi/dT_r sum_k beta_rk tau_k G_k,
// alpha_m the source's bilinear weights.  Partials of a quadrant root of
// Q(tau) = A tau^2 + B tau + C, by implicit differentiation
// (dtau/dtheta = -Q_theta / Q_tau, Q_tau = 2 A tau + B):
//   Q_tau_x = 2 char_x sx t0/dx,  Q_tau_y = 2 char_y sy t0/dy,  Q_f = -2 f,
//   Q_t0 = 2 char_x sx (tau_x - tau)/dx + 2 char_y sy (tau_y - tau)/dy,
//   Q_t0x = 2 tau char_x,  Q_t0y = 2 tau char_y,
// char_x = a Tx - c Ty, char_y = b Ty - c Tx, Tx = px tau + qx,
// Ty = py tau + qy (the characteristic of :210-214).  An axis update
// tau = (s_dis dis - q)/p with p = t0x - s t0/dx, q = s (t0/dx) tau_n gives
//   dtau/dtau_n = -(s t0/dx)/p, dtau/df = s_dis (dis/f)/p,
//   dtau/dt0 = s (tau - tau_n)/(dx p), dtau/dt0x = -tau/p
// (y likewise).  lambda is found by Jacobi iteration, exact after as many
// iterations as the longest dependency chain.
#include "oracle.h"
#include "eik_state.h"

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace {

inline int at(int nx, int ix, int iy) { return ix + nx * iy; }

// The winning candidate of a converged cell and its partials.
struct Win {
    bool ok = false;      // tau is this candidate (else tau is a constant)
    int jx = -1, jy = -1; // neighbours the candidate reads (-1: none)
    double dx_ = 0, dy_ = 0, df = 0, dt0 = 0, dt0x = 0, dt0y = 0;
};

// Candidates in the order of src/eikonal_solver.cpp:176-279; the smallest
// one (the first of equal ones) wins.  The forward keeps min(tau,
// candidates), so at a fixed point tau is the smallest candidate up to
// rounding: it was set from neighbour values that later moved by a few
// ulps, so the candidate recomputed now can exceed it by that much.  A cell
// whose smallest candidate is farther from tau (never reached, tau still
// its initial 10) does not depend on its neighbours.
Win winner(const EikState& S, const double* fun, int ix, int iy) {
    const int nx = S.nx, ny = S.ny;
    const int k = at(nx, ix, iy);
    const double tau = S.tau[k];
    const double t0 = S.T0[k], t0x = S.T0x[k], t0y = S.T0y[k];
    const double aij = S.a[k], bij = S.b[k], cij = S.c[k], fij = fun[k];
    const double det = aij * bij - cij * cij;
    const double dx = S.dx, dy = S.dy;
    Win best;
    double bv = HUGE_VAL;
    auto take = [&](double v, const Win& w) {
        if (v < bv) {
            bv = v;
            best = w;
        }
    };
    const int SXQ[4] = {-1, -1, +1, +1};
    const int SYQ[4] = {-1, +1, -1, +1};
    for (int q = 0; q < 4; q++) {
        const int sx = SXQ[q], sy = SYQ[q];
        const int nix = ix + sx, niy = iy + sy;
        if (nix < 0 || nix >= nx || niy < 0 || niy >= ny) continue;
        const int jx = at(nx, ix + sx, iy), jy = at(nx, ix, iy + sy);
        const double tx = S.tau[jx], ty = S.tau[jy];
        const double px = t0x - sx * (t0 / dx);
        const double qx = sx * (t0 / dx) * tx;
        const double py = t0y - sy * (t0 / dy);
        const double qy = sy * (t0 / dy) * ty;
        const double eq_a = aij * px * px + bij * py * py - 2.0 * cij * px * py;
        const double eq_b = 2.0 * (aij * px * qx + bij * py * qy - cij * (px * qy + py * qx));
        const double eq_c = aij * qx * qx + bij * qy * qy - 2.0 * cij * qx * qy - fij * fij;
        const double Delta = eq_b * eq_b - 4.0 * eq_a * eq_c;
        if (Delta < 0.0 || std::abs(eq_a) < 1e-30) continue;
        const double sq = std::sqrt(Delta);
        const double two_a = 2.0 * eq_a;
        for (int sgn = 0; sgn < 2; sgn++) {
            const double tt = (-eq_b + (sgn == 0 ? sq : -sq)) / two_a;
            const double Tx = px * tt + qx;
            const double Ty = py * tt + qy;
            const double char_x = aij * Tx - cij * Ty;
            const double char_y = bij * Ty - cij * Tx;
            if (!(-sx * char_x >= 0.0 && -sy * char_y >= 0.0)) continue;
            const double Qt = 2.0 * eq_a * tt + eq_b;
            Win w;
            w.ok = true;
            w.jx = jx;
            w.jy = jy;
            w.dx_ = -(2.0 * char_x * sx * t0 / dx) / Qt;
            w.dy_ = -(2.0 * char_y * sy * t0 / dy) / Qt;
            w.df = (2.0 * fij) / Qt;
            w.dt0 = -(2.0 * char_x * sx * (tx - tt) / dx + 2.0 * char_y * sy * (ty - tt) / dy) / Qt;
            w.dt0x = -(2.0 * tt * char_x) / Qt;
            w.dt0y = -(2.0 * tt * char_y) / Qt;
            take(tt, w);
        }
    }
    // axis updates: (neighbour offset, side s, along x?)
    struct Ax {
        int ox, oy, s;
        bool xdir;
        bool ok;
    };
    const Ax axes[4] = {{-1, 0, -1, true, ix > 0},
                        {+1, 0, +1, true, ix < nx - 1},
                        {0, -1, -1, false, iy > 0},
                        {0, +1, +1, false, iy < ny - 1}};
    for (const Ax& A : axes) {
        if (!A.ok || !(det > 0.0)) continue;
        const int kn = at(nx, ix + A.ox, iy + A.oy);
        const double h = A.xdir ? dx : dy;
        const double g = A.xdir ? t0x : t0y;
        const double p = g - A.s * (t0 / h);
        const double qv = A.s * (t0 / h) * S.tau[kn];
        const double dis = std::sqrt(fij * fij * (A.xdir ? bij : aij) / det);
        for (int sgn = 0; sgn < 2; sgn++) {
            const double sd = sgn == 0 ? 1.0 : -1.0;
            const double tt = (sd * dis - qv) / p;
            if (!(tt * t0 >= S.tau[kn] * S.T0[kn] && tt > S.tau[kn] * 0.5)) continue;
            Win w;
            w.ok = true;
            if (A.xdir) {
                w.jx = kn;
                w.dx_ = -(A.s * t0 / h) / p;
                w.dt0x = -tt / p;
            } else {
                w.jy = kn;
                w.dy_ = -(A.s * t0 / h) / p;
                w.dt0y = -tt / p;
            }
            w.df = sd * (dis / fij) / p;
            w.dt0 = A.s * (tt - S.tau[kn]) / (h * p);
            take(tt, w);
        }
    }
    if (!(std::abs(bv - tau) <= 1e-9 * std::abs(tau))) best.ok = false;
    return best;
}

// interp2d's cell and weights for one receiver (include/utils.h:358-409);
// false outside the grid
bool interp_weights(int nx, int ny, const double* xg, const double* yg, double qx, double qy,
                    int* idx, double* w) {
    if (qx < xg[0] || qx > xg[nx - 1] || qy < yg[0] || qy > yg[ny - 1]) return false;
    int i = static_cast<int>(std::lower_bound(xg, xg + nx, qx) - xg);
    if (i == nx) --i;
    if (i > 0 && xg[i] > qx) --i;
    i = std::clamp(i, 0, nx - 2);
    int j = static_cast<int>(std::lower_bound(yg, yg + ny, qy) - yg);
    if (j == ny) --j;
    if (j > 0 && yg[j] > qy) --j;
    j = std::clamp(j, 0, ny - 2);
    const double tx = (qx - xg[i]) / (xg[i + 1] - xg[i]);
    const double ty = (qy - yg[j]) / (yg[j + 1] - yg[j]);
    idx[0] = at(nx, i, j);
    idx[1] = at(nx, i + 1, j);
    idx[2] = at(nx, i, j + 1);
    idx[3] = at(nx, i + 1, j + 1);
    w[0] = (1 - tx) * (1 - ty);
    w[1] = tx * (1 - ty);
    w[2] = (1 - tx) * ty;
    w[3] = tx * ty;
    return true;
}

}  // namespace

// One event: forward to the stopping rule `tol` (0: fixed point), receiver
// times syn[nr], and, when dchi_dT is given (dchi/dT_r per receiver; NaN or
// receivers outside the grid contribute nothing), grad_fun[nx*ny] =
// dchi/dfun.  Returns 0, -1 for a grid below 3x3, -2 when the forward did
// not reach its stopping rule within maxiter iterations.
extern "C" int orc_eik_discrete_grad(int nx, int ny, const double* xx_deg, const double* yy_deg,
                                     const double* spha, const double* sphb, const double* sphc,
                                     const double* fun, double x0_deg, double y0_deg,
                                     double tol, int maxiter, int nr, const double* xrec_deg,
                                     const double* yrec_deg, const double* dchi_dT,
                                     double* syn, double* grad_fun, int* niter) {
    const int n = nx * ny;
    EikState S;
    std::vector<double> T(n);
    int it = 0;
    const int rc = eik_fwd_core(nx, ny, xx_deg, yy_deg, spha, sphb, sphc, fun, x0_deg, y0_deg,
                                tol, maxiter, T.data(), &it, &S);
    if (rc) return rc;
    if (niter) *niter = it;
    std::vector<int> ridx(4 * static_cast<size_t>(nr));
    std::vector<double> rw(4 * static_cast<size_t>(nr));
    std::vector<char> rin(nr);
    for (int r = 0; r < nr; r++) {
        rin[r] = interp_weights(nx, ny, xx_deg, yy_deg, xrec_deg[r], yrec_deg[r], &ridx[4 * r],
                                &rw[4 * r]);
        if (syn) {
            // the association of interp2d (orc_interp2d)
            syn[r] = rin[r] ? rw[4 * r] * T[ridx[4 * r]] + rw[4 * r + 1] * T[ridx[4 * r + 1]]
                                  + rw[4 * r + 2] * T[ridx[4 * r + 2]]
                                  + rw[4 * r + 3] * T[ridx[4 * r + 3]]
                            : std::nan("");
        }
    }
    if (!grad_fun) return it >= maxiter ? -2 : 0;
    // adjoint source and the explicit fun0 term of the receivers
    std::vector<double> g(n, 0.0);
    double Srec = 0.0;
    for (int r = 0; r < nr; r++) {
        const double d = dchi_dT[r];
        if (!rin[r] || !std::isfinite(d)) continue;
        for (int q = 0; q < 4; q++) {
            const int k = ridx[4 * r + q];
            g[k] += d * rw[4 * r + q] * S.T0[k];
            Srec += d * rw[4 * r + q] * S.tau[k] * S.G[k];
        }
    }
    std::vector<Win> W(n);
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++) {
            const int k = at(nx, ix, iy);
            if (S.ischange[k]) W[k] = winner(S, fun, ix, iy);
        }
    // lambda = g + J^T lambda by Jacobi iteration
    std::vector<double> lam = g, nxt(n);
    for (int pass = 0; pass <= n; pass++) {
        nxt = g;
        for (int k = 0; k < n; k++) {
            if (!W[k].ok || lam[k] == 0.0) continue;
            if (W[k].jx >= 0) nxt[W[k].jx] += W[k].dx_ * lam[k];
            if (W[k].jy >= 0) nxt[W[k].jy] += W[k].dy_ * lam[k];
        }
        const bool same = nxt == lam;
        lam.swap(nxt);
        if (same) break;
    }
    double Sfun0 = Srec;
    for (int k = 0; k < n; k++) {
        grad_fun[k] = 0.0;
        if (!W[k].ok) continue;
        grad_fun[k] = lam[k] * W[k].df;
        Sfun0 += lam[k] * (W[k].dt0 * S.G[k] + W[k].dt0x * S.Gx[k] + W[k].dt0y * S.Gy[k]);
    }
    // fun0 = bilinear(fun) at the source (src/eikonal_solver.cpp:71-82)
    const double r1 = S.r1, r2 = S.r2;
    grad_fun[at(nx, S.idx0, S.idy0)] += (1 - r1) * (1 - r2) * Sfun0;
    grad_fun[at(nx, S.idx0, S.idy0 + 1)] += (1 - r1) * r2 * Sfun0;
    grad_fun[at(nx, S.idx0 + 1, S.idy0)] += r1 * (1 - r2) * Sfun0;
    grad_fun[at(nx, S.idx0 + 1, S.idy0 + 1)] += r1 * r2 * Sfun0;
    return it >= maxiter ? -2 : 0;
}

// Every event of a batch as preproc::forward_for_event with the exact
// discrete gradient: chi = 0.5 sum w (T - Tobs)^2 (or, with sadj, the
// vector-Jacobian product of the receiver times with sadj), grad_svel
// [nper][ny][nx] += dchi/dsvel = -dchi/dfun fun^2 (fun = 1/svel,
// src/preproc.cpp:97-98), syn the receiver times.  tol as above; events
// round-robin over nthreads workers, planes summed in worker order.
extern "C" int orc_discrete_for_events(int nx, int ny, int nper, const double* xx_deg,
                                       const double* yy_deg, const double* svel,
                                       const double* m11, const double* m12,
                                       const double* m22, int ne, const double* evlo,
                                       const double* evla, const int* iper, const int* rec_ptr,
                                       const int* rec_idx, const double* stlo,
                                       const double* stla, const double* tt_obs,
                                       const double* weight, const double* sadj, double tol,
                                       int maxiter, double* syn, double* grad_svel,
                                       double* chi, int* fwd_iters, int nthreads) {
    const int n = nx * ny;
    const size_t plane = static_cast<size_t>(n) * nper;
    if (nthreads < 1) nthreads = 1;
    std::vector<std::vector<double>> acc(nthreads);
    std::vector<double> chis(nthreads, 0.0);
    std::vector<int> bad(nthreads, 0);
    auto work = [&](int t) {
        if (grad_svel) acc[t].assign(plane, 0.0);
        std::vector<double> fun(n), sphc(n), gf(n);
        for (int ie = t; ie < ne; ie += nthreads) {
            const int ip = iper[ie];
            const double* sv = svel + static_cast<size_t>(ip) * n;
            const double* a11 = m11 + static_cast<size_t>(ip) * n;
            const double* a12 = m12 + static_cast<size_t>(ip) * n;
            const double* a22 = m22 + static_cast<size_t>(ip) * n;
            for (int k = 0; k < n; k++) {
                fun[k] = (1.0 / sv[k]) * 1.0;
                sphc[k] = -a12[k];
            }
            const int r0 = rec_ptr[ie], nr = rec_ptr[ie + 1] - r0;
            std::vector<double> xr(nr), yr(nr), ts(nr), d(nr);
            for (int i = 0; i < nr; i++) {
                xr[i] = stlo[rec_idx[r0 + i]];
                yr[i] = stla[rec_idx[r0 + i]];
            }
            int it = 0;
            int rc = orc_eik_discrete_grad(nx, ny, xx_deg, yy_deg, a11, a22, sphc.data(),
                                           fun.data(), evlo[ie], evla[ie], tol, maxiter, nr,
                                           xr.data(), yr.data(), nullptr, ts.data(), nullptr,
                                           &it);
            if (rc) bad[t] = rc;
            if (fwd_iters) fwd_iters[ie] = it;
            double s = 0.0;
            for (int i = 0; i < nr; i++) {
                if (syn) syn[r0 + i] = ts[i];
                const double r = ts[i] - (tt_obs ? tt_obs[r0 + i] : 0.0);
                if (tt_obs) s += weight[r0 + i] * (r * r);
                d[i] = sadj ? sadj[r0 + i] : weight[r0 + i] * r;
            }
            chis[t] += 0.5 * s;
            if (!grad_svel) continue;
            rc = orc_eik_discrete_grad(nx, ny, xx_deg, yy_deg, a11, a22, sphc.data(), fun.data(),
                                       evlo[ie], evla[ie], tol, maxiter, nr, xr.data(),
                                       yr.data(), d.data(), nullptr, gf.data(), nullptr);
            if (rc) bad[t] = rc;
            double* out = acc[t].data() + static_cast<size_t>(ip) * n;
            for (int k = 0; k < n; k++) out[k] += -gf[k] * (fun[k] * fun[k]);
        }
    };
    if (nthreads == 1) {
        work(0);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; t++) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    double c = 0.0;
    for (int t = 0; t < nthreads; t++) {
        c += chis[t];
        if (grad_svel)
            for (size_t i = 0; i < plane; i++) grad_svel[i] += acc[t][i];
    }
    if (chi) *chi = c;
    for (int t = 0; t < nthreads; t++)
        if (bad[t]) return bad[t];
    return 0;
}
