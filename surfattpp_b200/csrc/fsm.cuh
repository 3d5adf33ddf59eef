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

// Four values of precision S loaded with 16-byte vector loads (one load for
// FP32, two for FP64): the per-cell operands of a sweep are packed so that a
// lane fetches its next cell with one or two instructions.
template <class S>
struct Q4 {
    S x, y, z, w;
};
__device__ __forceinline__ Q4<float> ld4(const Q4<float>* p) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ Q4<double> ld4(const Q4<double>* p) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    return {a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ void st4(Q4<float>* p, float x, float y, float z, float w) {
    *reinterpret_cast<float4*>(p) = make_float4(x, y, z, w);
}
__device__ __forceinline__ void st4(Q4<double>* p, double x, double y, double z, double w) {
    reinterpret_cast<double2*>(p)[0] = make_double2(x, y);
    reinterpret_cast<double2*>(p)[1] = make_double2(z, w);
}

// One cell update of eikonal::FSM_UW_PS_lonlat_2d (src/eikonal_solver.cpp:157-283).
// xm/xp/ym/yp carry tau and T0 of the axis neighbours (ix-1, ix+1, iy-1, iy+1).
// ISO: flat isotropic surface, c == +0 exactly.  The c terms are then
// signed zeros added to non-zero values and are dropped without changing any
// rounded result or comparison.
template <class S, bool ISO>
__device__ __forceinline__ S fsm_update(S tau, S t0, S t0x, S t0y, S aij, S bij, S cij, S fij,
                                        S dx, S dy, const Nb<S, S>& xm, const Nb<S, S>& xp,
                                        const Nb<S, S>& ym, const Nb<S, S>& yp) {
    const S det = ISO ? aij * bij : aij * bij - cij * cij;
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
        S eq_a, eq_b, eq_c;
        if (ISO) {
            eq_a = aij * px * px + bij * py * py;
            eq_b = S(2.0) * (aij * px * qx + bij * py * qy);
            eq_c = aij * qx * qx + bij * qy * qy - fij * fij;
        } else {
            eq_a = aij * px * px + bij * py * py - S(2.0) * cij * px * py;
            eq_b = S(2.0) * (aij * px * qx + bij * py * qy - cij * (px * qy + py * qx));
            eq_c = aij * qx * qx + bij * qy * qy - S(2.0) * cij * qx * qy - fij * fij;
        }
        const S Delta = eq_b * eq_b - S(4.0) * eq_a * eq_c;
        if (Delta < S(0) || abs_(eq_a) < S(1e-30)) continue;
        const S sq = sqrt(Delta);
        const S two_a = S(2.0) * eq_a;
#pragma unroll
        for (int sgn = 0; sgn < 2; sgn++) {
            const S tmp_tau = (-eq_b + (sgn == 0 ? sq : -sq)) / two_a;
            const S Tx = px * tmp_tau + qx;
            const S Ty = py * tmp_tau + qy;
            const S char_x = ISO ? aij * Tx : aij * Tx - cij * Ty;
            const S char_y = ISO ? bij * Ty : bij * Ty - cij * Tx;
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

// Forward sweep policies.  Per cell the sweep reads one packed record
// pk = {T0, T0x, T0y, fun} (built per event) and, for a general metric, one
// record mt = {a, b, c, 0} (built per period); the evolving field is a
// separate plane.  tau_start holds the field at the start of the iteration
// for the convergence test (src/eikonal_solver.cpp:147, :292-302).
template <class S, bool ISO>
struct MetricCell {
    S a, b, c;
};
template <class S>
struct MetricCell<S, true> {};

#ifndef SA_FWD_LEAD
#define SA_FWD_LEAD 1
#endif
// ROLLED: one copy of the sweep step with register moves (the default) or
// the step unrolled with statically rotated buffers (systolic.cuh).
template <class S, bool ISO, bool ROLLED = true>
struct FwdBase {
    using V = S;
    using X = S;
    static constexpr int kLead = SA_FWD_LEAD;
    static constexpr bool kRolled = ROLLED;
    // per-cell skip flags (systolic.cuh) where the update is expensive enough
    // to pay for them: the FP64 update (IEEE division and sqrt); the FP32
    // march updates every cell of its range (10 % faster on C3)
    static constexpr bool kFlags = sizeof(S) == sizeof(double);
    // the FP32 sweeps can run as a team (systolic.cuh)
    static constexpr bool kCoop = sizeof(S) == sizeof(float);
    struct Cell {
        S v;    // field before this update
        S x;    // T0 of the cell
        S gx, gy, f, vs;
        unsigned fl;     // sweep flags (systolic.cuh)
        MetricCell<S, ISO> m;
    };
    int nx, ny;
    unsigned char* flags;  // per event
    int2* rng;           // per row: x range of flag bit 0 (systolic.cuh)
    int2* crng;          // per row: x range changed in this iteration
    int2* rng2;          // next sweep's ranges (flag-free march)
    const Q4<S>* pk;     // per event
    const Q4<S>* mt;     // per period (general metric) or null
    const S* a_row;      // iso: [ny]
    S b_iso;
    S* tau;
    S* tau_start;
    int fix_x0, fix_x1;  // fixed source columns [fix_x0, fix_x1]
    int fy0, fy1;        // fixed source rows [fy0, fy1]
    bool row_fixed;
    S row_a;

    __device__ int nrows() const { return ny; }
    __device__ int ncols() const { return nx; }
    __device__ int stride() const { return nx; }
    __device__ int row(int rp, int yd) const { return yd > 0 ? rp : ny - 1 - rp; }
    __device__ int col(int cp, int xd) const { return xd > 0 ? cp : nx - 1 - cp; }
    __device__ int cp_of(int ix, int xd) const { return xd > 0 ? ix : nx - 1 - ix; }
    __device__ void begin_row(int iy, bool act) {
        if (!act) return;
        row_fixed = iy >= fy0 && iy <= fy1;
        if (ISO) row_a = a_row[iy];
    }
    __device__ Cell load(int k, bool last) const {
        Cell c;
        c.v = tau[k];
        const Q4<S> q = ld4(pk + k);
        c.x = q.x;
        c.gx = q.y;
        c.gy = q.z;
        c.f = q.w;
        if constexpr (!ISO) {
            const Q4<S> m = ld4(mt + k);
            c.m.a = m.x;
            c.m.b = m.y;
            c.m.c = m.z;
        }
        c.vs = last ? tau_start[k] : S(0);
        c.fl = kFlags ? flags[k] : 0u;
        return c;
    }
    __device__ S ca(const Cell& c) const {
        if constexpr (ISO) return row_a; else return c.m.a;
    }
    __device__ S cb(const Cell& c) const {
        if constexpr (ISO) return b_iso; else return c.m.b;
    }
    __device__ S cc(const Cell& c) const {
        if constexpr (ISO) return S(0); else return c.m.c;
    }
    __device__ Cell load_nb(int k) const {
        Cell c{};
        c.v = tau[k];
        c.x = pk[k].x;
        c.fl = kFlags ? flags[k] : 0u;
        return c;
    }
    __device__ void store(int k, S v, bool write_v, bool write_start) const {
        if (write_v) tau[k] = v;
        if (write_start) tau_start[k] = v;
    }
    __device__ void store_flag(int k, unsigned f) const { flags[k] = (unsigned char)f; }
};

// FP64 forward: field tau, exact reference update.
template <bool ISO>
struct FwdPolicy64 : FwdBase<double, ISO> {
    using Base = FwdBase<double, ISO>;
    using Cell = typename Base::Cell;
    using Base::row_fixed;
    using Base::fix_x0;
    using Base::fix_x1;
    double dx, dy;
    // Neighbours come in sweep order (xm / ym upwind).  The update is
    // evaluated in the sweep's reflected frame x' = xd*x, y' = yd*y: T0x,
    // T0y and the cross term c change sign, every intermediate is the
    // reference's own value times +-1 (exact), and the set of candidates is
    // the same, so the result is bit-identical to the unreflected update.
    __device__ double update(const Cell& cur, int ix, const Nb<double, double>& xm,
                             const Nb<double, double>& xp, const Nb<double, double>& ym,
                             const Nb<double, double>& yp, int xd, int yd) const {
        if (row_fixed && ix >= fix_x0 && ix <= fix_x1) return cur.v;   // ischange == 0
        return fsm_update<double, ISO>(cur.v, cur.x, (double)xd * cur.gx, (double)yd * cur.gy,
                                       this->ca(cur), this->cb(cur),
                                       (double)(xd * yd) * this->cc(cur), cur.f, dx, dy, xm, xp,
                                       ym, yp);
    }
    // convergence sums of src/eikonal_solver.cpp:292-302, last sweep only
    __device__ void account(const Cell& cur, double nv, double& l1, double& linf) const {
        const double d = fabs(nv - cur.vs) * cur.x;
        l1 += d;
        linf = fmax(linf, d);
    }
};

// FP32 arithmetic of the sweeps, spelled out: every product, sum and fused
// multiply-add is an explicit round-to-nearest operation, so no compiled copy
// of the sweep (the batch kernel's variants, a tail team's out-of-line copy)
// contracts differently from another, and all round identically.
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ff(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// approximate reciprocal (hardware, 1 ulp; flushes subnormals): divisions
// of the FP32 forward update are a * rcp(b), |b| in [1e-30, 2^126]
__device__ __forceinline__ float frcp(float b) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
    return r;
}
__device__ __forceinline__ float fdiv(float a, float b) { return __fmul_rn(a, frcp(b)); }
__device__ __forceinline__ float fsqrt(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

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
// Evaluated without control flow: every stencil is computed, invalid ones
// (missing neighbour, negative discriminant, degenerate quadratic, failed
// causality) are masked out of the minimum, so the compiler interleaves the
// eight independent stencils instead of running them one after another
// (12 % faster than the branched form on the batch workload).
template <bool ISO>
__device__ __forceinline__ float fsm_update_delta(float u, float t0, float t0x, float t0y,
                                                  float aij, float bij, float cij, float fij,
                                                  float idx, float idy,
                                                  const Nb<float, float>& xm,
                                                  const Nb<float, float>& xp,
                                                  const Nb<float, float>& ym,
                                                  const Nb<float, float>& yp) {
    const float det = ISO ? fm(aij, bij) : ff(aij, bij, -fm(cij, cij));
    const float k = fm(t0, idx);
    const float m = fm(t0, idy);
    const float f2 = fm(fij, fij);
    const float c2 = fm(2.f, cij);
    float best = u;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int sx = (q < 2) ? -1 : 1;
        const int sy = (q & 1) ? 1 : -1;
        const Nb<float, float>& nxn = (sx < 0) ? xm : xp;
        const Nb<float, float>& nyn = (sy < 0) ? ym : yp;
        const float ux = nxn.v, uy = nyn.v;
        const float A0 = ff(t0x, ux, t0x);
        const float A1 = sx < 0 ? fa(t0x, k) : fs(t0x, k);
        const float B0 = ff(sy < 0 ? m : -m, fs(ux, uy), ff(t0y, ux, t0y));
        const float B1 = sy < 0 ? fa(t0y, m) : fs(t0y, m);
        const float aA0 = fm(aij, A0), bB0 = fm(bij, B0);
        float al, be, ga;
        if (ISO) {
            al = ff(fm(aij, A1), A1, fm(fm(bij, B1), B1));
            be = fm(2.f, ff(aA0, A1, fm(bB0, B1)));
            ga = ff(aA0, A0, ff(bB0, B0, -f2));
        } else {
            al = ff(fm(aij, A1), A1, ff(fm(bij, B1), B1, -fm(fm(c2, A1), B1)));
            be = fm(2.f, ff(aA0, A1, ff(bB0, B1, -fm(cij, ff(A0, B1, fm(A1, B0))))));
            ga = ff(aA0, A0, ff(bB0, B0, ff(-fm(c2, A0), B0, -f2)));
        }
        const float disc = ff(be, be, -fm(fm(4.f, al), ga));
        const bool ok = nxn.has && nyn.has && disc >= 0.f && fabsf(al) >= 1e-30f;
        const float sq = fsqrt(fmaxf(disc, 0.f));
        const float qq = fm(-0.5f, fa(be, copysignf(sq, be)));
        // the second root as ga / qq also when qq == 0: then it is +-inf or
        // NaN and fails the tests below, and the first root is the only one
        float Dr[2];
        Dr[0] = fdiv(qq, al);
        Dr[1] = fdiv(ga, qq);
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const float D = Dr[r];
            const float Tx = ff(A1, D, A0);
            const float Ty = ff(B1, D, B0);
            const float char_x = ISO ? Tx : ff(aij, Tx, -fm(cij, Ty));
            const float char_y = ISO ? Ty : ff(bij, Ty, -fm(cij, Tx));
            // both characteristic components point away from the neighbours
            // (a NaN root makes both NaN and fails)
            const bool take = ok && fminf(-sx * char_x, -sy * char_y) >= 0.f;
            best = take ? fminf(best, fa(ux, D)) : best;
        }
    }
    const bool okd = det > 0.f;
    const float disx = fsqrt(fmaxf(fdiv(fm(f2, bij), det), 0.f));
    const float disy = fsqrt(fmaxf(fdiv(fm(f2, aij), det), 0.f));
    auto one_point = [&](const Nb<float, float>& n, float g, float kk, int s, float dis) {
        // (T0 tau)_axis = g*tau - s*kk*(tau - tau_n) = +-dis
        const float g1 = ff(g, n.v, g);
        const float rden = frcp(s < 0 ? fa(g, kk) : fs(g, kk));
        const bool ok = okd && n.has;
        // (1+c)*t0 >= (1+u_n)*T0_n  and  1+c > 0.5*(1+u_n)
        const float kn = fs(t0, ff(n.v, n.x, n.x));
        const float half = ff(0.5f, n.v, -0.5f);
#pragma unroll
        for (int sgn = 0; sgn < 2; sgn++) {
            const float c = ff(fs(sgn == 0 ? dis : -dis, g1), rden, n.v);
            const bool take = ok && ff(c, t0, kn) >= 0.f && c > half;
            best = take ? fminf(best, c) : best;
        }
    };
    one_point(xm, t0x, k, -1, disx);
    one_point(xp, t0x, k, +1, disx);
    one_point(ym, t0y, m, -1, disy);
    one_point(yp, t0y, m, +1, disy);
    return best;
}

// Pairs of FP32 values in one 64-bit register, for the packed FP32
// operations of sm_100 (add / sub / mul / fma .rn.f32x2).  Each half rounds
// exactly as the scalar operation of the same name, so an update written
// with them returns the scalar update's bits.
struct F2 {
    unsigned long long v;
};
__device__ __forceinline__ F2 p2(float a, float b) {
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ F2 b2(float a) { return p2(a, a); }
__device__ __forceinline__ void u2(F2 x, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x.v));
}
__device__ __forceinline__ F2 fa2(F2 a, F2 b) {
    F2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 fs2(F2 a, F2 b) {
    F2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 fm2(F2 a, F2 b) {
    F2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 ff2(F2 a, F2 b, F2 c) {
    F2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return d;
}
// exact negation of both halves (signs of zeros included)
__device__ __forceinline__ F2 neg2(F2 a) { return {a.v ^ 0x8000000080000000ull}; }

// fsm_update_delta with the arithmetic of two stencils in each packed
// operation: the quadrants sharing an x neighbour (y neighbour below /
// above) and the axis updates of one axis (neighbour before / after), every
// candidate then tested and folded into the minimum in the scalar form's
// order.  Same operations, operands and order per stencil as
// fsm_update_delta: the result is bit for bit the same.
template <bool ISO>
__device__ __forceinline__ float fsm_update_delta2(float u, float t0, float t0x, float t0y,
                                                   float aij, float bij, float cij, float fij,
                                                   float idx, float idy,
                                                   const Nb<float, float>& xm,
                                                   const Nb<float, float>& xp,
                                                   const Nb<float, float>& ym,
                                                   const Nb<float, float>& yp) {
    const float det = ISO ? fm(aij, bij) : ff(aij, bij, -fm(cij, cij));
    const float k = fm(t0, idx);
    const float m = fm(t0, idy);
    const float f2 = fm(fij, fij);
    const float c2 = fm(2.f, cij);
    float best = u;
    // members: sy = -1 (ym), sy = +1 (yp)
    const F2 uy = p2(ym.v, yp.v);
    const F2 msy = p2(m, -m);
    const F2 B1 = fa2(b2(t0y), msy);
#pragma unroll
    for (int px = 0; px < 2; px++) {   // sx = -1: quadrants 0, 1; sx = +1: 2, 3
        const int sx = px == 0 ? -1 : 1;
        const Nb<float, float>& nxn = (sx < 0) ? xm : xp;
        const float ux = nxn.v;
        const float A0 = ff(t0x, ux, t0x);
        const float A1 = sx < 0 ? fa(t0x, k) : fs(t0x, k);
        const F2 B0 = ff2(msy, fs2(b2(ux), uy), b2(ff(t0y, ux, t0y)));
        const float aA0 = fm(aij, A0);
        const F2 bB0 = fm2(b2(bij), B0);
        F2 al, be, ga;
        if (ISO) {
            al = ff2(b2(fm(aij, A1)), b2(A1), fm2(fm2(b2(bij), B1), B1));
            be = fm2(b2(2.f), ff2(b2(aA0), b2(A1), fm2(bB0, B1)));
            ga = ff2(b2(aA0), b2(A0), ff2(bB0, B0, b2(-f2)));
        } else {
            al = ff2(b2(fm(aij, A1)), b2(A1),
                     ff2(fm2(b2(bij), B1), B1, neg2(fm2(b2(fm(c2, A1)), B1))));
            be = fm2(b2(2.f),
                     ff2(b2(aA0), b2(A1),
                         ff2(bB0, B1, neg2(fm2(b2(cij), ff2(b2(A0), B1, fm2(b2(A1), B0)))))));
            ga = ff2(b2(aA0), b2(A0), ff2(bB0, B0, ff2(b2(-fm(c2, A0)), B0, b2(-f2))));
        }
        const F2 disc = ff2(be, be, neg2(fm2(fm2(b2(4.f), al), ga)));
        float dv[2], alv[2], bev[2];
        u2(disc, dv[0], dv[1]);
        u2(al, alv[0], alv[1]);
        u2(be, bev[0], bev[1]);
        bool ok[2];
        float sq[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
            ok[e] = nxn.has && (e == 0 ? ym.has : yp.has) && dv[e] >= 0.f &&
                    fabsf(alv[e]) >= 1e-30f;
            sq[e] = copysignf(fsqrt(fmaxf(dv[e], 0.f)), bev[e]);
        }
        const F2 qq = fm2(b2(-0.5f), fa2(be, p2(sq[0], sq[1])));
        float qv[2];
        u2(qq, qv[0], qv[1]);
        // the second root as ga / qq also when qq == 0 (see fsm_update_delta)
        F2 Dr[2];
        Dr[0] = fm2(qq, p2(frcp(alv[0]), frcp(alv[1])));
        Dr[1] = fm2(ga, p2(frcp(qv[0]), frcp(qv[1])));
        bool take[2][2];
        float cand[2][2];
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const F2 Tx = ff2(b2(A1), Dr[r], b2(A0));
            const F2 Ty = ff2(B1, Dr[r], B0);
            F2 chx = Tx, chy = Ty;
            if (!ISO) {
                chx = ff2(b2(aij), Tx, neg2(fm2(b2(cij), Ty)));
                chy = ff2(b2(bij), Ty, neg2(fm2(b2(cij), Tx)));
            }
            float xv[2], yv[2], cv[2];
            u2(chx, xv[0], xv[1]);
            u2(chy, yv[0], yv[1]);
            u2(fa2(b2(ux), Dr[r]), cv[0], cv[1]);
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int sy = e == 0 ? -1 : 1;
                take[r][e] = ok[e] && fminf(-sx * xv[e], -sy * yv[e]) >= 0.f;
                cand[r][e] = cv[e];
            }
        }
#pragma unroll
        for (int e = 0; e < 2; e++)
#pragma unroll
            for (int r = 0; r < 2; r++) best = take[r][e] ? fminf(best, cand[r][e]) : best;
    }
    const bool okd = det > 0.f;
    const float disx = fsqrt(fmaxf(fdiv(fm(f2, bij), det), 0.f));
    const float disy = fsqrt(fmaxf(fdiv(fm(f2, aij), det), 0.f));
    // axis updates, the neighbours before (s = -1) and after (s = +1) of one
    // axis in one pair: (T0 tau)_axis = g*tau - s*kk*(tau - tau_n) = +-dis
    auto axis_pair = [&](const Nb<float, float>& n0, const Nb<float, float>& n1, float g, float kk,
                         float dis) {
        const F2 nv = p2(n0.v, n1.v), nx = p2(n0.x, n1.x);
        const F2 g1 = ff2(b2(g), nv, b2(g));
        float den[2];
        u2(fa2(b2(g), p2(kk, -kk)), den[0], den[1]);
        const F2 rden = p2(frcp(den[0]), frcp(den[1]));
        // (1+c)*t0 >= (1+u_n)*T0_n  and  1+c > 0.5*(1+u_n)
        const F2 kn = fs2(b2(t0), ff2(nv, nx, nx));
        float hv[2];
        u2(ff2(b2(0.5f), nv, b2(-0.5f)), hv[0], hv[1]);
        float cv[2][2], tv[2][2];
#pragma unroll
        for (int sgn = 0; sgn < 2; sgn++) {
            const F2 c = ff2(fs2(b2(sgn == 0 ? dis : -dis), g1), rden, nv);
            u2(c, cv[sgn][0], cv[sgn][1]);
            u2(ff2(c, b2(t0), kn), tv[sgn][0], tv[sgn][1]);
        }
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const bool ok = okd && (e == 0 ? n0.has : n1.has);
#pragma unroll
            for (int sgn = 0; sgn < 2; sgn++) {
                const bool take = ok && tv[sgn][e] >= 0.f && cv[sgn][e] > hv[e];
                best = take ? fminf(best, cv[sgn][e]) : best;
            }
        }
    };
    axis_pair(xm, xp, t0x, k, disx);
    axis_pair(ym, yp, t0y, m, disy);
    return best;
}

// FSM_PACKED 1: the forward update in packed FP32 pairs (fsm_update_delta2),
// 0: the scalar form; both give the same bits.
#ifndef FSM_PACKED
#define FSM_PACKED 1
#endif

// FP32 forward: field u = tau - 1, increment-form update.
template <bool ISO, bool ROLLED = true>
struct FwdPolicyDelta32 : FwdBase<float, ISO, ROLLED> {
    using Base = FwdBase<float, ISO, ROLLED>;
    using Cell = typename Base::Cell;
    using Base::row_fixed;
    using Base::fix_x0;
    using Base::fix_x1;
    float idx, idy;
    // neighbours in sweep order, evaluated in the reflected frame (see
    // FwdPolicy64::update)
    __device__ float update(const Cell& cur, int ix, const Nb<float, float>& xm,
                            const Nb<float, float>& xp, const Nb<float, float>& ym,
                            const Nb<float, float>& yp, int xd, int yd) const {
        if (row_fixed && ix >= fix_x0 && ix <= fix_x1) return cur.v;
#if FSM_PACKED
        return fsm_update_delta2<ISO>(cur.v, cur.x, (float)xd * cur.gx, (float)yd * cur.gy,
                                      this->ca(cur), this->cb(cur),
                                      (float)(xd * yd) * this->cc(cur), cur.f, idx, idy, xm, xp,
                                      ym, yp);
#else
        return fsm_update_delta<ISO>(cur.v, cur.x, (float)xd * cur.gx, (float)yd * cur.gy,
                                     this->ca(cur), this->cb(cur),
                                     (float)(xd * yd) * this->cc(cur), cur.f, idx, idy, xm, xp,
                                     ym, yp);
#endif
    }
    __device__ void account(const Cell& cur, float nv, double& l1, double& linf) const {
        const double d = __dmul_rn(fabs(__dsub_rn((double)nv, (double)cur.vs)), (double)cur.x);
        l1 = __dadd_rn(l1, d);
        linf = fmax(linf, d);
    }
};

// Adjoint sweep policy, exact FP64 form (src/eikonal_solver.cpp:471-509),
// over the interior.  Per cell: aq = {a1p, a2m, b1p, b2m} (the positive /
// negative parts of the left/right/bottom/top face fluxes, :404-441) and
// dd = {delta, d} with d = (a2p - a1m)/dx + (b2p - b1m)/dy (:479-481).
struct AdjPolicyExact {
    using V = double;
    using X = float;      // no auxiliary neighbour data
    static constexpr int kLead = 2;
    static constexpr bool kRolled = false;
    static constexpr bool kFlags = false;   // ranges from changes (systolic.cuh)
    static constexpr bool kCoop = false;
    struct Cell {
        double v;
        float x;
        Q4<double> q;
        double2 de;
        double vs;
        unsigned fl;
    };
    int nx, ny;
    double dx, dy;
    int2* rng;
    int2* crng;
    int2* rng2;          // next sweep's ranges (flag-free march)
    const Q4<double>* aq;
    const double2* dd;
    double* Ta;
    double* Ta_start;

    __device__ int nrows() const { return ny - 2; }
    __device__ int ncols() const { return nx - 2; }
    __device__ int stride() const { return nx; }
    __device__ int row(int rp, int yd) const { return yd > 0 ? 1 + rp : ny - 2 - rp; }
    __device__ int col(int cp, int xd) const { return xd > 0 ? 1 + cp : nx - 2 - cp; }
    __device__ int cp_of(int ix, int xd) const { return xd > 0 ? ix - 1 : nx - 2 - ix; }
    __device__ void begin_row(int, bool) {}
    __device__ Cell load(int k, bool last) const {
        Cell c;
        c.v = Ta[k];
        c.x = 0.f;
        c.q = ld4(aq + k);
        c.de = dd[k];
        c.vs = last ? Ta_start[k] : 0.0;
        c.fl = 0u;
        return c;
    }
    __device__ Cell load_nb(int k) const {
        Cell c{};
        c.v = Ta[k];
        return c;
    }
    // um / dm: upwind / downwind x neighbour in sweep order (likewise uy /
    // dy_), mapped back to the grid's left/right and bottom/top
    __device__ double update(const Cell& cur, int, const Nb<double, float>& um,
                             const Nb<double, float>& dm, const Nb<double, float>& uy,
                             const Nb<double, float>& dy_, int xd, int yd) const {
        const Nb<double, float>& xm = xd > 0 ? um : dm;
        const Nb<double, float>& xp = xd > 0 ? dm : um;
        const Nb<double, float>& ym = yd > 0 ? uy : dy_;
        const Nb<double, float>& yp = yd > 0 ? dy_ : uy;
        const double2 de = cur.de;
        double nv;
        if (fabs(de.y) < 1e-14) {
            nv = 0.0;
        } else {
            const Q4<double>& q = cur.q;
            const double txm = xm.has ? xm.v : 0.0;
            const double txp = xp.has ? xp.v : 0.0;
            const double tym = ym.has ? ym.v : 0.0;
            const double typ = yp.has ? yp.v : 0.0;
            const double e = (txm * q.x - txp * q.y) / dx + (tym * q.z - typ * q.w) / dy;
            nv = (de.x + e) / de.y;
        }
        return nv;
    }
    // src/eikonal_solver.cpp:498-507
    __device__ void account(const Cell& cur, double nv, double& l1, double& linf) const {
        const double dv = fabs(nv - cur.vs);
        l1 += dv;
        linf = fmax(linf, dv);
    }
    __device__ void store(int k, double v, bool write_v, bool write_start) const {
        if (write_v) Ta[k] = v;
        if (write_start) Ta_start[k] = v;
    }
};

// Sweep policy of the exact discrete adjoint (batch.cuh, discrete_adjoint):
// lambda = c0 + wxm lambda(ix-1) + wxp lambda(ix+1) + wym lambda(iy-1) +
// wyp lambda(iy+1) over the whole grid, FP64, the weights being the partial
// derivatives of the neighbours' winning forward stencils with respect to
// this cell's tau (zero where a neighbour's stencil does not read it).
struct AdjPolicyLinear64 {
    using V = double;
    using X = float;
    static constexpr int kLead = 2;
    static constexpr bool kRolled = false;
    static constexpr bool kFlags = false;
    static constexpr bool kCoop = false;
    struct Cell {
        double v;
        float x;
        Q4<double> w;
        double c0;
        double vs;
        unsigned fl;
    };
    int nx, ny;
    int2* rng;
    int2* crng;
    int2* rng2;
    const Q4<double>* W;
    const double* C0;
    double* Ta;
    double* Ta_start;

    __device__ int nrows() const { return ny; }
    __device__ int ncols() const { return nx; }
    __device__ int stride() const { return nx; }
    __device__ int row(int rp, int yd) const { return yd > 0 ? rp : ny - 1 - rp; }
    __device__ int col(int cp, int xd) const { return xd > 0 ? cp : nx - 1 - cp; }
    __device__ int cp_of(int ix, int xd) const { return xd > 0 ? ix : nx - 1 - ix; }
    __device__ void begin_row(int, bool) {}
    __device__ Cell load(int k, bool last) const {
        Cell c;
        c.v = Ta[k];
        c.x = 0.f;
        c.w = ld4(W + k);
        c.c0 = C0[k];
        c.vs = last ? Ta_start[k] : 0.0;
        c.fl = 0u;
        return c;
    }
    __device__ Cell load_nb(int k) const {
        Cell c{};
        c.v = Ta[k];
        return c;
    }
    __device__ double update(const Cell& cur, int, const Nb<double, float>& um,
                             const Nb<double, float>& dm, const Nb<double, float>& uy,
                             const Nb<double, float>& dy_, int xd, int yd) const {
        const Nb<double, float>& xm = xd > 0 ? um : dm;
        const Nb<double, float>& xp = xd > 0 ? dm : um;
        const Nb<double, float>& ym = yd > 0 ? uy : dy_;
        const Nb<double, float>& yp = yd > 0 ? dy_ : uy;
        const double txm = xm.has ? xm.v : 0.0;
        const double txp = xp.has ? xp.v : 0.0;
        const double tym = ym.has ? ym.v : 0.0;
        const double typ = yp.has ? yp.v : 0.0;
        return cur.c0 + cur.w.x * txm + cur.w.y * txp + cur.w.z * tym + cur.w.w * typ;
    }
    __device__ void account(const Cell& cur, double nv, double& l1, double& linf) const {
        const double dv = fabs(nv - cur.vs);
        l1 += dv;
        linf = fmax(linf, dv);
    }
    __device__ void store(int k, double v, bool write_v, bool write_start) const {
        if (write_v) Ta[k] = v;
        if (write_start) Ta_start[k] = v;
    }
};

// Adjoint sweep policy, FP32 weight form: the same Gauss-Seidel update
// rewritten as Ta = c0 + wxm*Ta(ix-1) + wxp*Ta(ix+1) + wym*Ta(iy-1) + wyp*Ta(iy+1)
// with FP32 weights computed in FP64 (w = {wxm, wxp, wym, wyp}, c0 separate).
// LEAD: how many steps ahead the sweep loads (2 by default).
template <int LEAD = 2>
struct AdjPolicyW32 {
    using V = float;
    using X = float;
    static constexpr int kLead = LEAD;
    static constexpr bool kRolled = false;
    static constexpr bool kFlags = false;   // ranges from changes (systolic.cuh)
    static constexpr bool kCoop = true;
    struct Cell {
        float v;
        float x;
        Q4<float> w;
        float c0;
        float vs;
        unsigned fl;
    };
    int nx, ny;
    int2* rng;
    int2* crng;
    int2* rng2;          // next sweep's ranges (flag-free march)
    const Q4<float>* W;
    const float* C0;
    float* Ta;
    float* Ta_start;

    __device__ int nrows() const { return ny - 2; }
    __device__ int ncols() const { return nx - 2; }
    __device__ int stride() const { return nx; }
    __device__ int row(int rp, int yd) const { return yd > 0 ? 1 + rp : ny - 2 - rp; }
    __device__ int col(int cp, int xd) const { return xd > 0 ? 1 + cp : nx - 2 - cp; }
    __device__ int cp_of(int ix, int xd) const { return xd > 0 ? ix - 1 : nx - 2 - ix; }
    __device__ void begin_row(int, bool) {}
    __device__ Cell load(int k, bool last) const {
        Cell c;
        c.v = Ta[k];
        c.x = 0.f;
        c.w = ld4(W + k);
        c.c0 = C0[k];
        c.vs = last ? Ta_start[k] : 0.f;
        c.fl = 0u;
        return c;
    }
    __device__ Cell load_nb(int k) const {
        Cell c{};
        c.v = Ta[k];
        return c;
    }
    // neighbours in sweep order, mapped back as in AdjPolicyExact::update
    __device__ float update(const Cell& cur, int, const Nb<float, float>& um,
                            const Nb<float, float>& dm, const Nb<float, float>& uy,
                            const Nb<float, float>& dy_, int xd, int yd) const {
        const Nb<float, float>& xm = xd > 0 ? um : dm;
        const Nb<float, float>& xp = xd > 0 ? dm : um;
        const Nb<float, float>& ym = yd > 0 ? uy : dy_;
        const Nb<float, float>& yp = yd > 0 ? dy_ : uy;
        const float txm = xm.has ? xm.v : 0.f;
        const float txp = xp.has ? xp.v : 0.f;
        const float tym = ym.has ? ym.v : 0.f;
        const float typ = yp.has ? yp.v : 0.f;
        return ff(cur.w.w, typ, ff(cur.w.z, tym, ff(cur.w.y, txp, ff(cur.w.x, txm, cur.c0))));
    }
    __device__ void account(const Cell& cur, float nv, double& l1, double& linf) const {
        const double dv = fabs(__dsub_rn((double)nv, (double)cur.vs));
        l1 = __dadd_rn(l1, dv);
        linf = fmax(linf, dv);
    }
    __device__ void store(int k, float v, bool write_v, bool write_start) const {
        if (write_v) Ta[k] = v;
        if (write_start) Ta_start[k] = v;
    }
};

}  // namespace sa
