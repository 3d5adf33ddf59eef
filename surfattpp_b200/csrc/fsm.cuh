// Sweep policies: the factored-eikonal forward update and the adjoint
// transport update, templated on the sweep precision S.
//   S = double: rounds exactly as the reference's FP64 code (the translation
//               unit is compiled with -fmad=false; IEEE division and sqrt).
//   S = float:  the same update in FP32 (fast division/sqrt); travel times,
//               adjoint coefficients, residuals and accumulation stay FP64.
#pragma once
#include "common.cuh"
#include "systolic.cuh"

namespace sa {

__device__ __forceinline__ double abs_(double x) { return fabs(x); }
__device__ __forceinline__ float abs_(float x) { return fabsf(x); }

// One cell update of eikonal::FSM_UW_PS_lonlat_2d (src/eikonal_solver.cpp:157-283).
// xm/xp/ym/yp carry tau and T0 of the axis neighbours (ix-1, ix+1, iy-1, iy+1).
template <class S>
__device__ __forceinline__ S fsm_update(S tau, S t0, S t0x, S t0y, S aij, S bij, S cij, S fij,
                                        S dx, S dy, const Nb<S, S>& xm, const Nb<S, S>& xp,
                                        const Nb<S, S>& ym, const Nb<S, S>& yp) {
    const S det = aij * bij - cij * cij;
    const S tdx = t0 / dx;
    const S tdy = t0 / dy;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int sx = (k < 2) ? -1 : 1;
        const int sy = (k & 1) ? 1 : -1;
        const Nb<S, S>& nxn = (sx < 0) ? xm : xp;
        const Nb<S, S>& nyn = (sy < 0) ? ym : yp;
        if (!(nxn.has && nyn.has)) continue;
        const S px = t0x - sx * tdx;
        const S qx = sx * tdx * nxn.v;
        const S py = t0y - sy * tdy;
        const S qy = sy * tdy * nyn.v;
        const S eq_a = aij * px * px + bij * py * py - S(2.0) * cij * px * py;
        const S eq_b = S(2.0) * (aij * px * qx + bij * py * qy - cij * (px * qy + py * qx));
        const S eq_c = aij * qx * qx + bij * qy * qy - S(2.0) * cij * qx * qy - fij * fij;
        const S Delta = eq_b * eq_b - S(4.0) * eq_a * eq_c;
        if (Delta < S(0) || abs_(eq_a) < S(1e-30)) continue;
        const S sq = sqrt(Delta);
        const S two_a = S(2.0) * eq_a;
#pragma unroll
        for (int sgn = 0; sgn < 2; sgn++) {
            const S tmp_tau = (-eq_b + (sgn == 0 ? sq : -sq)) / two_a;
            const S Tx = px * tmp_tau + qx;
            const S Ty = py * tmp_tau + qy;
            const S char_x = aij * Tx - cij * Ty;
            const S char_y = bij * Ty - cij * Tx;
            if (-sx * char_x >= S(0) && -sy * char_y >= S(0))
                if (tmp_tau < tau) tau = tmp_tau;
        }
    }
    if (det > S(0)) {
        const S disx = sqrt(fij * fij * bij / det);
        const S disy = sqrt(fij * fij * aij / det);
        if (xm.has) {
            const S px = t0x + t0 / dx;
            const S qx = -(t0 / dx) * xm.v;
#pragma unroll
            for (int sgn = 0; sgn < 2; sgn++) {
                const S tmp_tau = ((sgn == 0 ? disx : -disx) - qx) / px;
                if (tmp_tau * t0 >= xm.v * xm.x && tmp_tau > xm.v * S(0.5))
                    if (tmp_tau < tau) tau = tmp_tau;
            }
        }
        if (xp.has) {
            const S px = t0x - t0 / dx;
            const S qx = (t0 / dx) * xp.v;
#pragma unroll
            for (int sgn = 0; sgn < 2; sgn++) {
                const S tmp_tau = ((sgn == 0 ? disx : -disx) - qx) / px;
                if (tmp_tau * t0 >= xp.v * xp.x && tmp_tau > xp.v * S(0.5))
                    if (tmp_tau < tau) tau = tmp_tau;
            }
        }
        if (ym.has) {
            const S py = t0y + t0 / dy;
            const S qy = -(t0 / dy) * ym.v;
#pragma unroll
            for (int sgn = 0; sgn < 2; sgn++) {
                const S tmp_tau = ((sgn == 0 ? disy : -disy) - qy) / py;
                if (tmp_tau * t0 >= ym.v * ym.x && tmp_tau > ym.v * S(0.5))
                    if (tmp_tau < tau) tau = tmp_tau;
            }
        }
        if (yp.has) {
            const S py = t0y - t0 / dy;
            const S qy = (t0 / dy) * yp.v;
#pragma unroll
            for (int sgn = 0; sgn < 2; sgn++) {
                const S tmp_tau = ((sgn == 0 ? disy : -disy) - qy) / py;
                if (tmp_tau * t0 >= yp.v * yp.x && tmp_tau > yp.v * S(0.5))
                    if (tmp_tau < tau) tau = tmp_tau;
            }
        }
    }
    return tau;
}

// Forward sweep policy.  Field: tau (sweep precision S) in the warp's
// scratch slot; tau_start holds the field at the start of the iteration for
// the convergence test (src/eikonal_solver.cpp:147, :292-302).
template <class S>
struct FwdPolicy {
    using V = S;
    using X = S;
    struct Cell {
        S v;    // tau before this update
        S x;    // T0 of the cell
        S gx, gy, f, a, b, c, vs;
    };
    int nx, ny;
    S dx, dy, fun0;
    const S* G;
    const S* Gx;
    const S* Gy;
    const S* fun;        // period plane
    const S* a_row;      // iso: [ny]
    S b_iso;
    const S* a_pl;       // general planes or null
    const S* b_pl;
    const S* c_pl;
    S* tau;
    S* tau_start;
    int fix_x0, fix_x1;  // fixed source columns [fix_x0, fix_x1]
    const double* yy;
    double y0, dy64;
    // per-row state
    bool row_fixed;
    S row_a;

    __device__ int nrows() const { return ny; }
    __device__ int ncols() const { return nx; }
    __device__ int row(int rp, int yd) const { return yd > 0 ? rp : ny - 1 - rp; }
    __device__ int col(int cp, int xd) const { return xd > 0 ? cp : nx - 1 - cp; }
    __device__ void begin_row(int iy, bool act) {
        if (!act) return;
        row_fixed = fabs((yy[iy] - y0) / dy64) <= 1.0;
        row_a = a_pl ? S(0) : a_row[iy];
    }
    __device__ Cell load(int iy, int ix, bool last) const {
        const size_t k = (size_t)iy * nx + ix;
        Cell c;
        c.v = tau[k];
        c.x = G[k] * fun0;
        c.gx = Gx[k];
        c.gy = Gy[k];
        c.f = fun[k];
        if (a_pl) {
            c.a = a_pl[k];
            c.b = b_pl[k];
            c.c = c_pl[k];
        } else {
            c.a = row_a;
            c.b = b_iso;
            c.c = S(0);
        }
        c.vs = last ? tau_start[k] : S(0);
        return c;
    }
    __device__ Cell load_nb(int iy, int ix) const {
        const size_t k = (size_t)iy * nx + ix;
        Cell c{};
        c.v = tau[k];
        c.x = G[k] * fun0;
        return c;
    }
    __device__ S update(const Cell& cur, int iy, int ix, const Nb<S, S>& xm, const Nb<S, S>& xp,
                        const Nb<S, S>& ym, const Nb<S, S>& yp, bool last, double& l1,
                        double& linf) const {
        if (row_fixed && ix >= fix_x0 && ix <= fix_x1) return cur.v;   // ischange == 0
        const S t0x = cur.gx * fun0;
        const S t0y = cur.gy * fun0;
        const S nv = fsm_update<S>(cur.v, cur.x, t0x, t0y, cur.a, cur.b, cur.c, cur.f, dx, dy,
                                   xm, xp, ym, yp);
        if (last) {
            const double d = fabs((double)nv - (double)cur.vs) * (double)cur.x;
            l1 += d;
            linf = fmax(linf, d);
        }
        return nv;
    }
    __device__ void store(int iy, int ix, S v, bool last) const {
        const size_t k = (size_t)iy * nx + ix;
        tau[k] = v;
        if (last) tau_start[k] = v;
    }
};

// FP32 forward update in increment form.  The stored field is u = tau - 1
// (tau ~ 1 everywhere, so u keeps ~20x more absolute resolution than tau),
// and each stencil is solved for the increment D = u - u_neighbour.  This is
// the same discretisation as fsm_update (same stencils, same causality
// tests, same fixed point), rearranged so that no FP32 quantity carries the
// (t0/dx)^2 magnitudes whose cancellation ruins the direct quadratic:
//   Tx = A0 + A1*D,  Ty = B0 + B1*D,
//   A0 = t0x*(1+u_x), A1 = t0x - sx*t0/dx,
//   B0 = t0y*(1+u_x) - sy*(t0/dy)*(u_x - u_y), B1 = t0y - sy*t0/dy,
// solved with the cancellation-free quadratic formula.
__device__ __forceinline__ float fsm_update_delta(float u, float t0, float t0x, float t0y,
                                                  float aij, float bij, float cij, float fij,
                                                  float idx, float idy,
                                                  const Nb<float, float>& xm,
                                                  const Nb<float, float>& xp,
                                                  const Nb<float, float>& ym,
                                                  const Nb<float, float>& yp) {
    const float det = aij * bij - cij * cij;
    const float k = t0 * idx;
    const float m = t0 * idy;
    const float f2 = fij * fij;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int sx = (q < 2) ? -1 : 1;
        const int sy = (q & 1) ? 1 : -1;
        const Nb<float, float>& nxn = (sx < 0) ? xm : xp;
        const Nb<float, float>& nyn = (sy < 0) ? ym : yp;
        if (!(nxn.has && nyn.has)) continue;
        const float ux = nxn.v, uy = nyn.v;
        const float tx1 = fmaf(t0x, ux, t0x);
        const float A0 = tx1;
        const float A1 = t0x - sx * k;
        const float B0 = fmaf(t0y, ux, t0y) - sy * m * (ux - uy);
        const float B1 = t0y - sy * m;
        const float al = aij * A1 * A1 + bij * B1 * B1 - 2.f * cij * A1 * B1;
        const float be = 2.f * (aij * A0 * A1 + bij * B0 * B1 - cij * (A0 * B1 + A1 * B0));
        const float ga = aij * A0 * A0 + bij * B0 * B0 - 2.f * cij * A0 * B0 - f2;
        const float disc = be * be - 4.f * al * ga;
        if (disc < 0.f || fabsf(al) < 1e-30f) continue;
        const float sq = sqrtf(disc);
        const float qq = -0.5f * (be + copysignf(sq, be));
        float Dr[2];
        Dr[0] = qq / al;
        Dr[1] = (qq != 0.f) ? ga / qq : Dr[0];
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const float D = Dr[r];
            const float Tx = fmaf(A1, D, A0);
            const float Ty = fmaf(B1, D, B0);
            const float char_x = aij * Tx - cij * Ty;
            const float char_y = bij * Ty - cij * Tx;
            if (-sx * char_x >= 0.f && -sy * char_y >= 0.f) {
                const float c = ux + D;
                if (c < u) u = c;
            }
        }
    }
    if (det > 0.f) {
        const float disx = sqrtf(f2 * bij / det);
        const float disy = sqrtf(f2 * aij / det);
        auto one_point = [&](const Nb<float, float>& n, float g, float kk, int s, float dis) {
            // (T0 tau)_axis = g*tau - s*kk*(tau - tau_n) = +-dis
            const float g1 = fmaf(g, n.v, g);
            const float den = g - s * kk;
#pragma unroll
            for (int sgn = 0; sgn < 2; sgn++) {
                const float D = ((sgn == 0 ? dis : -dis) - g1) / den;
                const float c = n.v + D;
                // (1+c)*t0 >= (1+u_n)*T0_n  and  1+c > 0.5*(1+u_n)
                const float lhs = (t0 - n.x) + (c * t0 - n.v * n.x);
                if (lhs >= 0.f && c > 0.5f * n.v - 0.5f)
                    if (c < u) u = c;
            }
        };
        if (xm.has) one_point(xm, t0x, k, -1, disx);
        if (xp.has) one_point(xp, t0x, k, +1, disx);
        if (ym.has) one_point(ym, t0y, m, -1, disy);
        if (yp.has) one_point(yp, t0y, m, +1, disy);
    }
    return u;
}

// FP32 forward policy: field u = tau - 1.
struct FwdPolicyDelta32 {
    using V = float;
    using X = float;
    struct Cell {
        float v;    // u before this update
        float x;    // T0 of the cell
        float gx, gy, f, a, b, c, vs;
    };
    int nx, ny;
    float idx, idy, fun0;
    const float* G;
    const float* Gx;
    const float* Gy;
    const float* fun;
    const float* a_row;
    float b_iso;
    const float* a_pl;
    const float* b_pl;
    const float* c_pl;
    float* tau;         // holds u
    float* tau_start;
    int fix_x0, fix_x1;
    const double* yy;
    double y0, dy64;
    bool row_fixed;
    float row_a;

    __device__ int nrows() const { return ny; }
    __device__ int ncols() const { return nx; }
    __device__ int row(int rp, int yd) const { return yd > 0 ? rp : ny - 1 - rp; }
    __device__ int col(int cp, int xd) const { return xd > 0 ? cp : nx - 1 - cp; }
    __device__ void begin_row(int iy, bool act) {
        if (!act) return;
        row_fixed = fabs((yy[iy] - y0) / dy64) <= 1.0;
        row_a = a_pl ? 0.f : a_row[iy];
    }
    __device__ Cell load(int iy, int ix, bool last) const {
        const size_t k = (size_t)iy * nx + ix;
        Cell c;
        c.v = tau[k];
        c.x = G[k] * fun0;
        c.gx = Gx[k];
        c.gy = Gy[k];
        c.f = fun[k];
        if (a_pl) {
            c.a = a_pl[k];
            c.b = b_pl[k];
            c.c = c_pl[k];
        } else {
            c.a = row_a;
            c.b = b_iso;
            c.c = 0.f;
        }
        c.vs = last ? tau_start[k] : 0.f;
        return c;
    }
    __device__ Cell load_nb(int iy, int ix) const {
        const size_t k = (size_t)iy * nx + ix;
        Cell c{};
        c.v = tau[k];
        c.x = G[k] * fun0;
        return c;
    }
    __device__ float update(const Cell& cur, int iy, int ix, const Nb<float, float>& xm,
                            const Nb<float, float>& xp, const Nb<float, float>& ym,
                            const Nb<float, float>& yp, bool last, double& l1,
                            double& linf) const {
        if (row_fixed && ix >= fix_x0 && ix <= fix_x1) return cur.v;
        const float nv = fsm_update_delta(cur.v, cur.x, cur.gx * fun0, cur.gy * fun0, cur.a,
                                          cur.b, cur.c, cur.f, idx, idy, xm, xp, ym, yp);
        if (last) {
            const double d = fabs((double)nv - (double)cur.vs) * (double)cur.x;
            l1 += d;
            linf = fmax(linf, d);
        }
        return nv;
    }
    __device__ void store(int iy, int ix, float v, bool last) const {
        const size_t k = (size_t)iy * nx + ix;
        tau[k] = v;
        if (last) tau_start[k] = v;
    }
};

// Adjoint sweep policy, exact FP64 form (src/eikonal_solver.cpp:471-509),
// over the interior.  A(ix,iy) = a1 (left-face flux) for ix in [1,nx-1] and
// a2(ix) == A(ix+1); B(ix,iy) = b1 (bottom-face flux) for iy in [1,ny-1] and
// b2(iy) == B(iy+1) (identical expressions in the reference).  D = diagonal.
struct AdjPolicyExact {
    using V = double;
    using X = float;      // no auxiliary neighbour data
    struct Cell {
        double v;
        float x;
        double vs;
    };
    int nx, ny;
    double dx, dy;
    const double* A;
    const double* B;
    const double* D;
    const double* delta;
    double* Ta;
    double* Ta_start;

    __device__ int nrows() const { return ny - 2; }
    __device__ int ncols() const { return nx - 2; }
    __device__ int row(int rp, int yd) const { return yd > 0 ? 1 + rp : ny - 2 - rp; }
    __device__ int col(int cp, int xd) const { return xd > 0 ? 1 + cp : nx - 2 - cp; }
    __device__ void begin_row(int, bool) {}
    __device__ Cell load(int iy, int ix, bool last) const {
        const size_t k = (size_t)iy * nx + ix;
        Cell c;
        c.v = Ta[k];
        c.x = 0.f;
        c.vs = last ? Ta_start[k] : 0.0;
        return c;
    }
    __device__ Cell load_nb(int iy, int ix) const {
        Cell c{};
        c.v = Ta[(size_t)iy * nx + ix];
        return c;
    }
    __device__ double update(const Cell& cur, int iy, int ix, const Nb<double, float>& xm,
                             const Nb<double, float>& xp, const Nb<double, float>& ym,
                             const Nb<double, float>& yp, bool last, double& l1,
                             double& linf) const {
        const size_t k = (size_t)iy * nx + ix;
        const double d = D[k];
        double nv;
        if (fabs(d) < 1e-14) {
            nv = 0.0;
        } else {
            const double a1 = A[k], a2 = A[k + 1];
            const double b1 = B[k], b2 = B[k + nx];
            const double a1p = (a1 + fabs(a1)) / 2.0;
            const double a2m = (a2 - fabs(a2)) / 2.0;
            const double b1p = (b1 + fabs(b1)) / 2.0;
            const double b2m = (b2 - fabs(b2)) / 2.0;
            const double txm = xm.has ? xm.v : 0.0;
            const double txp = xp.has ? xp.v : 0.0;
            const double tym = ym.has ? ym.v : 0.0;
            const double typ = yp.has ? yp.v : 0.0;
            const double e = (txm * a1p - txp * a2m) / dx + (tym * b1p - typ * b2m) / dy;
            nv = (delta[k] + e) / d;
        }
        if (last) {
            const double dd = fabs(nv - cur.vs);
            l1 += dd;
            linf = fmax(linf, dd);
        }
        return nv;
    }
    __device__ void store(int iy, int ix, double v, bool last) const {
        const size_t k = (size_t)iy * nx + ix;
        Ta[k] = v;
        if (last) Ta_start[k] = v;
    }
};

// Adjoint sweep policy, FP32 weight form: the same Gauss-Seidel update
// rewritten as Ta = c0 + wxm*Ta(ix-1) + wxp*Ta(ix+1) + wym*Ta(iy-1) + wyp*Ta(iy+1)
// with FP32 weights precomputed in FP64 (W plane = 5 floats per cell).
struct AdjPolicyW32 {
    using V = float;
    using X = float;
    struct Cell {
        float v;
        float x;
        float c0, wxm, wxp, wym, wyp;
        float vs;
    };
    int nx, ny;
    const float* W;     // [5][ny][nx]
    float* Ta;
    float* Ta_start;
    float* vmax;        // unused placeholder

    __device__ int nrows() const { return ny - 2; }
    __device__ int ncols() const { return nx - 2; }
    __device__ int row(int rp, int yd) const { return yd > 0 ? 1 + rp : ny - 2 - rp; }
    __device__ int col(int cp, int xd) const { return xd > 0 ? 1 + cp : nx - 2 - cp; }
    __device__ void begin_row(int, bool) {}
    __device__ Cell load(int iy, int ix, bool last) const {
        const size_t n = (size_t)nx * ny;
        const size_t k = (size_t)iy * nx + ix;
        Cell c;
        c.v = Ta[k];
        c.x = 0.f;
        c.c0 = W[k];
        c.wxm = W[n + k];
        c.wxp = W[2 * n + k];
        c.wym = W[3 * n + k];
        c.wyp = W[4 * n + k];
        c.vs = last ? Ta_start[k] : 0.f;
        return c;
    }
    __device__ Cell load_nb(int iy, int ix) const {
        Cell c{};
        c.v = Ta[(size_t)iy * nx + ix];
        return c;
    }
    __device__ float update(const Cell& cur, int, int, const Nb<float, float>& xm,
                            const Nb<float, float>& xp, const Nb<float, float>& ym,
                            const Nb<float, float>& yp, bool last, double& l1,
                            double& linf) const {
        const float txm = xm.has ? xm.v : 0.f;
        const float txp = xp.has ? xp.v : 0.f;
        const float tym = ym.has ? ym.v : 0.f;
        const float typ = yp.has ? yp.v : 0.f;
        const float nv = cur.c0 + cur.wxm * txm + cur.wxp * txp + cur.wym * tym + cur.wyp * typ;
        if (last) {
            const double dd = fabs((double)nv - (double)cur.vs);
            l1 += dd;
            linf = fmax(linf, dd);
        }
        return nv;
    }
    __device__ void store(int iy, int ix, float v, bool last) const {
        const size_t k = (size_t)iy * nx + ix;
        Ta[k] = v;
        if (last) Ta_start[k] = v;
    }
};

}  // namespace sa
