// Persistent (source, period) batch kernel, templated on the sweep precision.
//
// One warp per event, events pulled from a device work queue (atomicAdd on a
// counter), so solves of uneven iteration count balance across the GPU.  Per
// event, fused: forward FSM -> T = tau*T0 -> receiver interpolation ->
// residuals and misfit -> adjoint source -> face fluxes -> adjoint FSM ->
// source mask -> adj_s += Ta * svel^-3 (FP64 atomics).
// Reference: preproc::forward_for_event (src/preproc.cpp:71-148).
#pragma once
#include "common.cuh"
#include "event_common.cuh"
#include "fsm.cuh"
#include "launch.h"

#include <type_traits>

// Resident 128-thread blocks per SM the register allocation is sized for.
#ifndef SA_MINB64
#define SA_MINB64 3
#endif
#ifndef SA_MINB32
#define SA_MINB32 4
#endif

namespace sa {

template <class S>
struct BatchArgs {
    Grid g;
    int iso;
    const S* fun;          // sweep-precision slowness planes
    const double* fun64;   // FP64 slowness planes (fun0, T0 for T)
    const double* inv3;
    const S* a_f_row;
    const double* a_a_row64;
    S b_iso;
    double b_iso64;
    const Q4<S>* mt;       // general metric {a, b, c, 0} per period (or null)
    const double* b_p64;
    const double* a_a64;
    const double* c_a64;
    const S* G;
    const S* Gx;
    const S* Gy;
    const double* G64;
    Events ev;
    Outputs out;
    Scratch sc;
    int maxr;              // largest receiver count of any event
    int mode;
    int discrete;          // BatchDesc::discrete
};

// Scratch slot layout (bytes, every plane 256-byte aligned).  The packed
// forward operands (PK) and the packed adjoint coefficients share one region:
// the forward planes are dead once T is formed.
struct SlotLayout {
    size_t tau, tst, T, delta, PK, AQ, DD, W, C0, Ta, sadj, syn, flags, rng, team, total;
};
template <class S>
__host__ __device__ inline SlotLayout slot_layout(int nx, int ny, int maxr) {
    const size_t n = (size_t)nx * ny;
    const size_t r = (size_t)(maxr > 0 ? maxr : 1);
    SlotLayout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o += align_up(bytes, 256);
        return at;
    };
    L.tau = take(n * sizeof(S));
    L.tst = take(n * sizeof(S));
    L.T = take(n * sizeof(double));
    L.delta = take(n * sizeof(double));
    L.PK = take(n * 4 * sizeof(S));
    L.AQ = L.PK;      // FP64: {a1p, a2m, b1p, b2m} (same size as PK)
    L.W = L.PK;       // FP32: {wxm, wxp, wym, wyp} (same size as PK)
    if (sizeof(S) == sizeof(double)) {
        L.DD = take(n * 2 * sizeof(double));
        L.C0 = 0;
    } else {
        L.C0 = take(n * sizeof(float));
        L.DD = 0;
    }
    L.Ta = take(n * sizeof(S));
    L.sadj = take(r * sizeof(double));
    L.syn = take(r * sizeof(double));
    L.flags = take(n);   // per-cell sweep flags of the FP64 forward (systolic.cuh)
    // per-row x ranges (systolic.cuh): [0, ny) cells that can change in the
    // current sweep, [ny, 2 ny) cells changed in the current iteration,
    // [2 ny, 3 ny) the adjoint's ranges for the next sweep
    L.rng = take(3 * (size_t)ny * sizeof(int2));
    // tail teams (systolic.cuh, Team): per strip its record and the last
    // sweep's L1 partials of its 32 lanes
    const size_t nstrip = ((size_t)ny + 31) / 32;
    L.team = take(nstrip * sizeof(int4) + nstrip * 32 * sizeof(double));
    L.total = o;
    return L;
}

// Launch variants of the FP32 kernel (kBatchVariants, chosen per plan by
// sa_plan_autotune): bit 0 = unrolled forward step (else one rolled copy),
// bit 1 = FP32 adjoint loads 3 steps ahead (else 2), bit 2 = tail teams
// (below).  The FP64 kernel has variant 0 only.
__host__ __device__ constexpr bool variant_fwd_rolled(int v) { return (v & 1) == 0; }
__host__ __device__ constexpr int variant_adj_lead(int v) { return (v & 2) ? 3 : 2; }
__host__ __device__ constexpr bool variant_teams(int v) { return (v & 4) != 0; }

// Tail teams (FP32 kernel, variant bit 2).  A warp whose queue pull finds no
// event left offers itself to the warps of its block still solving one; at
// its next iteration start such an owner takes the warps on offer, and the
// team marches that iteration's four sweeps together (systolic.cuh, Team).
// The owner keeps its team to the end of the forward (or adjoint)
// iterations, then releases it.  Results are those of the warp alone (the
// same cell updates; the L1 sums added per strip in strip order).  Every
// wait is bounded; one that gives up sets the block's error flag, after
// which no team forms and the events report ST_TEAM.
constexpr int kTeamPolBytes = 256;
struct TeamRec {
    unsigned long long word[4];   // the members' progress words (systolic.cuh)
    double linf[4];               // members' Linf of the iteration
    int4* sinfo;                  // the owner's strip records and L1 partials
    double* sums;
    alignas(16) unsigned char pol[kTeamPolBytes];   // the owner's sweep policy
};
struct BlockTeams {
    unsigned idle;      // bit w: warp w is on offer
    int busy;           // warps that may still take a team
    int err;
    unsigned mail[4];   // per warp: job from an owner (0: none)
    TeamRec rec[4];     // per owner warp
};
constexpr unsigned kMailRelease = 0x80000000u;
constexpr long long kOfferNs = 30000000000ll;   // an offer is withdrawn after 30 s

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.cta.shared.u32 %0, [%1];"
                 : "=r"(v)
                 : "r"((unsigned)__cvta_generic_to_shared(p))
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.cta.shared.u32 [%0], %1;"
                 :
                 : "r"((unsigned)__cvta_generic_to_shared(p)), "r"(v)
                 : "memory");
}
__device__ __forceinline__ unsigned mail_job(int owner, int role, int W, int kind) {
    return 1u | (unsigned)owner << 1 | (unsigned)role << 3 | (unsigned)W << 5 |
           (unsigned)kind << 8;
}

// Owner, at an iteration start: takes the warps on offer, posts the
// iteration to its members and returns the team (W = 1: alone).  kind 0 =
// forward sweeps, 1 = adjoint sweeps.
template <class Pol>
__device__ __forceinline__ Team team_begin(BlockTeams* bt, unsigned& helpers, int kind,
                                           const Pol& P, int ny) {
    const int lane = threadIdx.x & 31, me = threadIdx.x >> 5;
    TeamRec& R = bt->rec[me];
    // the slot's team region follows its range planes (slot_layout)
    unsigned char* tr =
        reinterpret_cast<unsigned char*>(P.rng) + align_up(3 * (size_t)ny * sizeof(int2), 256);
    int4* sinfo = reinterpret_cast<int4*>(tr);
    double* sums = reinterpret_cast<double*>(tr + (size_t)((ny + 31) / 32) * sizeof(int4));
    Team T{1, 0, R.word, sinfo, sums, &bt->err};
    const bool ok = __shfl_sync(FULL_MASK, *(volatile int*)&bt->err, 0) == 0;
    if (ok && __popc(helpers) < 3) {
        unsigned got = 0;
        if (lane == 0) {
            unsigned m = *(volatile unsigned*)&bt->idle & ~(1u << me);
            while (m) {
                const int b = __ffs(m) - 1;
                m &= m - 1;
                if (atomicAnd(&bt->idle, ~(1u << b)) & (1u << b)) got |= 1u << b;
            }
        }
        helpers |= __shfl_sync(FULL_MASK, got, 0);
    }
    if (!ok || helpers == 0) return T;
    T.W = 1 + __popc(helpers);
    static_assert(sizeof(Pol) <= kTeamPolBytes, "sweep policy larger than its team copy");
    if (lane == 0) {
        *reinterpret_cast<Pol*>(R.pol) = P;
        R.sinfo = sinfo;
        R.sums = sums;
    }
    if (lane < T.W) R.word[lane] = 0ull;
    __threadfence_block();
    __syncwarp();
    if (lane == 0) {
        int role = 1;
        for (unsigned m = helpers; m; m &= m - 1)
            st_release_u32(&bt->mail[__ffs(m) - 1], mail_job(me, role++, T.W, kind));
    }
    return T;
}

// Owner, after the team's sweeps: waits for every member, folds in their
// Linf and forms the L1 sum in strip order (as the warp alone adds it).
__device__ __forceinline__ void team_end(BlockTeams* bt, const Team& T, int nstrip, double& l1,
                                         double& linf) {
    const int lane = threadIdx.x & 31, me = threadIdx.x >> 5;
    for (int r = 1; r < T.W; r++) {
        team_wait(T, r, kTeamEnd - 1, kStripDone);
        linf = fmax(linf, bt->rec[me].linf[r]);
    }
    double s = 0.0;
    for (int j = 0; j < nstrip; j++) s += T.sums[j * 32 + lane];
    l1 = s;
}

// One team iteration (four sweeps) of a member: out of line, so that owner
// and helpers run one copy of the team sweeps (two copies of the long
// forward step in flight on an SM thrash its instruction cache).  Returns the
// member's Linf; the L1 partials go to the strip sums.
template <class Pol>
__device__ __noinline__ double team_sweeps(const Pol* pol, const Team T) {
    Pol P = *pol;
    double l1 = 0.0, linf = 0.0;
    for (int sw = 0; sw < 4; sw++)
        systolic_sweep(P, sweep_xd(sw), sweep_yd(sw), sw == 3, l1, linf, &T, sw);
    return linf;
}

__device__ __forceinline__ void team_release(BlockTeams* bt, unsigned& helpers) {
    if ((threadIdx.x & 31) == 0)
        for (unsigned m = helpers; m; m &= m - 1) st_release_u32(&bt->mail[__ffs(m) - 1], kMailRelease);
    helpers = 0;
    __syncwarp();
}

// A warp without events: on offer until every warp of the block is done;
// runs the iterations its owners post.
template <class PolF, class PolA>
__device__ __forceinline__ void team_serve(BlockTeams* bt) {
    const int lane = threadIdx.x & 31, me = threadIdx.x >> 5;
    if (lane == 0) atomicOr(&bt->idle, 1u << me);
    __syncwarp();
    long long t0 = __shfl_sync(FULL_MASK, global_ns(), 0);
    bool offered = true;
    for (;;) {
        const unsigned m = __shfl_sync(FULL_MASK, ld_acquire_u32(&bt->mail[me]), 0);
        const long long now = __shfl_sync(FULL_MASK, global_ns(), 0);
        if (m == 0u) {
            if (__shfl_sync(FULL_MASK, *(volatile int*)&bt->busy, 0) == 0) break;
            if (now - t0 > (offered ? kOfferNs : kTeamWaitNs)) {
                if (!offered) {   // taken, but no job came
                    if (lane == 0) atomicExch(&bt->err, 1);
                    break;
                }
                // withdraw the offer; if an owner took it already, its job follows
                unsigned old = 0;
                if (lane == 0) old = atomicAnd(&bt->idle, ~(1u << me));
                if (!((__shfl_sync(FULL_MASK, old, 0) >> me) & 1u)) {
                    offered = false;
                    t0 = now;
                    continue;
                }
                break;
            }
            __nanosleep(256);
            continue;
        }
        if (lane == 0) bt->mail[me] = 0u;
        __syncwarp();
        t0 = now;
        if (m == kMailRelease) {
            if (lane == 0) atomicOr(&bt->idle, 1u << me);
            offered = true;
            __syncwarp();
            continue;
        }
        const int o = (m >> 1) & 3, role = (m >> 3) & 3, W = (m >> 5) & 7, kind = (m >> 8) & 1;
        TeamRec& R = bt->rec[o];
        const Team T{W, role, R.word, R.sinfo, R.sums, &bt->err};
        double linf = kind == 0 ? team_sweeps(reinterpret_cast<const PolF*>(R.pol), T)
                                : team_sweeps(reinterpret_cast<const PolA*>(R.pol), T);
        linf = warp_max(linf);
        if (lane == 0) R.linf[role] = linf;
        __threadfence_block();
        __syncwarp();
        if (lane == 0) st_release_u64(&R.word[role], team_word(kTeamEnd, 0));
        offered = false;
    }
}

template <class S, bool ISO, int VAR>
__device__ __forceinline__ double fwd_solve(const BatchArgs<S>& B, const SrcInfo& si, int ip,
                                            int src, S* tau, S* tst, Q4<S>* pk,
                                            unsigned char* flags, int2* rng, double* T,
                                            int& iters, int& status, BlockTeams* bt) {
    const Grid& g = B.g;
    const int nx = g.nx, ny = g.ny;
    const size_t n = (size_t)nx * ny;
    const int lane = threadIdx.x & 31;
    const double fun0_64 = bilinear64(B.fun64 + (size_t)ip * n, nx, si.idx0, si.idy0, si.r1, si.r2);
    using Pol = typename std::conditional<sizeof(S) == sizeof(double), FwdPolicy64<ISO>,
                                          FwdPolicyDelta32<ISO, variant_fwd_rolled(VAR)>>::type;
    Pol P;
    P.nx = nx;
    P.ny = ny;
    if constexpr (sizeof(S) == sizeof(double)) {
        P.dx = g.dx;
        P.dy = g.dy;
    } else {
        P.idx = (float)(1.0 / g.dx);
        P.idy = (float)(1.0 / g.dy);
    }
    // packed per-cell operands {T0, T0x, T0y, fun}; T0 = G*fun0 etc. exactly
    // as src/eikonal_solver.cpp:102-115 multiplies by fun0 last
    const S fun0 = (S)fun0_64;
    {
        const S* G = B.G + (size_t)src * n;
        const S* Gx = B.Gx + (size_t)src * n;
        const S* Gy = B.Gy + (size_t)src * n;
        const S* fn = B.fun + (size_t)ip * n;
        for (size_t k = lane; k < n; k += 32)
            st4(pk + k, G[k] * fun0, Gx[k] * fun0, Gy[k] * fun0, fn[k]);
    }
    P.pk = pk;
    P.mt = ISO ? nullptr : B.mt + (size_t)ip * n;
    P.a_row = B.a_f_row;
    P.b_iso = B.b_iso;
    P.tau = tau;
    P.tau_start = tst;
    P.flags = flags;
    P.rng = rng;
    P.crng = rng + ny;
    P.rng2 = rng + 2 * ny;
    P.fix_x0 = si.fix_x0;
    P.fix_x1 = si.fix_x1;
    // rows with |(yy - y0)/dy| <= 1 (src/eikonal_solver.cpp:118-129, :162):
    // one contiguous range, yy being monotone
    int fy0 = ny, fy1 = -1;
    for (int iy = lane; iy < ny; iy += 32)
        if (fabs((g.yy[iy] - si.y0) / g.dy) <= 1.0) {
            fy0 = min(fy0, iy);
            fy1 = max(fy1, iy);
        }
    for (int o = 16; o > 0; o >>= 1) {
        fy0 = min(fy0, __shfl_xor_sync(FULL_MASK, fy0, o));
        fy1 = max(fy1, __shfl_xor_sync(FULL_MASK, fy1, o));
    }
    P.fy0 = fy0;
    P.fy1 = fy1;
    // initial tau (src/eikonal_solver.cpp:118-129); FP32 stores u = tau - 1
    const S off = (sizeof(S) == sizeof(double)) ? S(0) : S(1);
    for_cells(nx, n, lane, [&](size_t k, int ix, int iy) {
        const bool fixed = iy >= fy0 && iy <= fy1 && ix >= si.fix_x0 && ix <= si.fix_x1;
        const S v = (fixed ? S(1) : S(10)) - off;
        tau[k] = v;
        tst[k] = v;
        if (Pol::kFlags) flags[k] = 1;
    });
    for (int iy = lane; iy < ny; iy += 32) {
        rng[iy] = make_int2(0, nx - 1);
        rng[ny + iy] = make_int2(0x7fffffff, -1);   // crng: nothing changed yet
        rng[2 * ny + iy] = make_int2(0x7fffffff, -1);
    }
    __syncwarp();
    iters = 0;
    // stopping rule: the reference's (src/eikonal_solver.cpp:292-303), or,
    // for the exact discrete adjoint, a fixed point (an iteration in which
    // no cell changed: every cell's change times T0 is zero, T0 > 0 off the
    // fixed source cells)
    unsigned helpers = 0;   // tail team (FP32 variants with teams)
    for (int iter = 0; iter < 2000; iter++) {
        double l1 = 0.0, linf = 0.0;
        if constexpr (variant_teams(VAR) && sizeof(S) == sizeof(float)) {
            // (alone: the sweeps of the variants without teams, the same code)
            const Team tm = bt ? team_begin(bt, helpers, 0, P, ny)
                               : Team{1, 0, nullptr, nullptr, nullptr, nullptr};
            if (tm.W > 1) {
                linf = team_sweeps(reinterpret_cast<const Pol*>(bt->rec[threadIdx.x >> 5].pol), tm);
                team_end(bt, tm, (ny + 31) >> 5, l1, linf);
            } else {
                for (int sw = 0; sw < 4; sw++)
                    systolic_sweep(P, sweep_xd(sw), sweep_yd(sw), sw == 3, l1, linf);
            }
        } else {
            for (int sw = 0; sw < 4; sw++)
                systolic_sweep(P, sweep_xd(sw), sweep_yd(sw), sw == 3, l1, linf);
        }
        iters = iter + 1;
        const double L1 = warp_sum(l1) / (double)(nx * ny);
        const double Linf = warp_max(linf);
        if (B.discrete ? (Linf == 0.0) : (L1 < 1e-4 && Linf < 1e-4)) break;
        if (iter == 1999) status = ST_NOCONV;
    }
    if constexpr (variant_teams(VAR) && sizeof(S) == sizeof(float)) {
        if (bt) {
            team_release(bt, helpers);
            if (__shfl_sync(FULL_MASK, *(volatile int*)&bt->err, 0)) status = ST_TEAM;
        }
    }
    // T = tau * T0 in FP64 (src/eikonal_solver.cpp:317)
    const double* G64 = B.G64 + (size_t)src * n;
    bool finite = true;
    for (size_t k = lane; k < n; k += 32) {
        const double t0 = G64[k] * fun0_64;
        const double t = (sizeof(S) == sizeof(double)) ? (double)tau[k] * t0
                                                         : t0 + (double)tau[k] * t0;
        T[k] = t;
        if (!isfinite(t)) finite = false;
    }
    if (!__all_sync(FULL_MASK, finite)) status = ST_NONFINITE;
    __syncwarp();
    return fun0_64;
}

// ---------------------------------------------------------------------------
// Exact discrete adjoint of the factored forward solve (FP64 plans, no
// reference counterpart: the reference's adjoint, src/eikonal_solver.cpp:
// 323-511, discretises the continuous adjoint equation).  At a fixed point of
// the forward iteration every free cell satisfies tau_k = Phi_k(tau_x, tau_y,
// f_k, t0_k, t0x_k, t0y_k), Phi_k its smallest admissible candidate of
// :176-279 (a quadrant root, two upwind neighbours, or an axis update, one).
// With T = tau T0 and T0 = G fun0 (fun0 the bilinear slowness at the source):
//   lambda = g + J^T lambda,   g_k = sum_r dchi/dT_r beta_rk T0_k,
//   dchi/dfun_m = lambda_m dPhi_m/df_m + alpha_m S,
//   S = sum_k lambda_k (dPhi/dt0 G + dPhi/dt0x Gx + dPhi/dt0y Gy)_k
//       + sum_r dchi/dT_r sum_k beta_rk tau_k G_k,
// beta the receivers' interp2d weights, alpha the source's bilinear weights;
// the partials by implicit differentiation of the quadratic (quadrant) or
// of the axis formula.  lambda is swept to its fixed point with the same
// engine (AdjPolicyLinear64), whose weights at cell j are the partials of the
// neighbours' winning stencils with respect to tau_j.  The result,
// dchi/dsvel = -dchi/dfun fun^2, is added to adj_s (or the event's
// contribution plane).
// Scratch reuse (after the forward): T -> dPhi/dtau of the x neighbour,
// delta -> of the y neighbour (zeroed again at the end), DD -> {dPhi/df,
// dPhi/dfun0}, flags -> which neighbours the winner reads, tau -> the
// adjoint source g, PK -> the sweep weights, Ta / tst -> lambda.
// ---------------------------------------------------------------------------
struct WinD {
    int dirx, diry;   // 0: none, 1: the neighbour at -1, 2: at +1
    double jx, jy, df, dt0, dt0x, dt0y;
    bool ok;
};

// The smallest admissible candidate of cell (ix, iy) and its partials; not
// ok when that candidate is farther than 1e-9 relative from tau (the cell
// was never reached).
__device__ inline WinD discrete_winner(const double* tau, const Q4<double>* pk, int nx, int ny,
                                       int ix, int iy, double aij, double bij, double cij,
                                       double dx, double dy) {
    const int k = iy * nx + ix;
    const Q4<double> c0 = pk[k];
    const double t0 = c0.x, t0x = c0.y, t0y = c0.z, fij = c0.w;
    const double det = aij * bij - cij * cij;
    WinD best{};
    best.ok = false;
    double bv = HUGE_VAL;
#pragma unroll 1
    for (int q = 0; q < 4; q++) {
        const int sx = (q < 2) ? -1 : 1;
        const int sy = (q & 1) ? 1 : -1;
        if (ix + sx < 0 || ix + sx >= nx || iy + sy < 0 || iy + sy >= ny) continue;
        const double tx = tau[k + sx], ty = tau[k + sy * nx];
        const double px = t0x - sx * (t0 / dx);
        const double qx = sx * (t0 / dx) * tx;
        const double py = t0y - sy * (t0 / dy);
        const double qy = sy * (t0 / dy) * ty;
        const double ea = aij * px * px + bij * py * py - 2.0 * cij * px * py;
        const double eb = 2.0 * (aij * px * qx + bij * py * qy - cij * (px * qy + py * qx));
        const double ec = aij * qx * qx + bij * qy * qy - 2.0 * cij * qx * qy - fij * fij;
        const double Delta = eb * eb - 4.0 * ea * ec;
        if (Delta < 0.0 || fabs(ea) < 1e-30) continue;
        const double sq = sqrt(Delta);
#pragma unroll 1
        for (int sgn = 0; sgn < 2; sgn++) {
            const double tt = (-eb + (sgn == 0 ? sq : -sq)) / (2.0 * ea);
            const double Tx = px * tt + qx, Ty = py * tt + qy;
            const double chx = aij * Tx - cij * Ty, chy = bij * Ty - cij * Tx;
            if (!(-sx * chx >= 0.0 && -sy * chy >= 0.0) || !(tt < bv)) continue;
            const double Qt = 2.0 * ea * tt + eb;
            bv = tt;
            best.dirx = sx < 0 ? 1 : 2;
            best.diry = sy < 0 ? 1 : 2;
            best.jx = -(2.0 * chx * sx * t0 / dx) / Qt;
            best.jy = -(2.0 * chy * sy * t0 / dy) / Qt;
            best.df = (2.0 * fij) / Qt;
            best.dt0 = -(2.0 * chx * sx * (tx - tt) / dx + 2.0 * chy * sy * (ty - tt) / dy) / Qt;
            best.dt0x = -(2.0 * tt * chx) / Qt;
            best.dt0y = -(2.0 * tt * chy) / Qt;
        }
    }
    if (det > 0.0) {
#pragma unroll 1
        for (int a = 0; a < 4; a++) {
            const bool xdir = a < 2;
            const int s = (a & 1) ? 1 : -1;
            if (xdir ? (ix + s < 0 || ix + s >= nx) : (iy + s < 0 || iy + s >= ny)) continue;
            const int kn = xdir ? k + s : k + s * nx;
            const double h = xdir ? dx : dy;
            const double p = (xdir ? t0x : t0y) - s * (t0 / h);
            const double qv = s * (t0 / h) * tau[kn];
            const double dis = sqrt(fij * fij * (xdir ? bij : aij) / det);
            const double tn = tau[kn], T0n = pk[kn].x;
#pragma unroll 1
            for (int sgn = 0; sgn < 2; sgn++) {
                const double sd = sgn == 0 ? 1.0 : -1.0;
                const double tt = (sd * dis - qv) / p;
                if (!(tt * t0 >= tn * T0n && tt > tn * 0.5) || !(tt < bv)) continue;
                bv = tt;
                best.dirx = xdir ? (s < 0 ? 1 : 2) : 0;
                best.diry = xdir ? 0 : (s < 0 ? 1 : 2);
                best.jx = xdir ? -(s * t0 / h) / p : 0.0;
                best.jy = xdir ? 0.0 : -(s * t0 / h) / p;
                best.df = sd * (dis / fij) / p;
                best.dt0 = s * (tt - tn) / (h * p);
                best.dt0x = xdir ? -tt / p : 0.0;
                best.dt0y = xdir ? 0.0 : -tt / p;
            }
        }
    }
    best.ok = fabs(bv - tau[k]) <= 1e-9 * fabs(tau[k]);
    return best;
}

template <bool ISO>
__device__ inline void discrete_adjoint(const BatchArgs<double>& B, unsigned int e,
                                        unsigned char* base, const SrcInfo& si, int ip, int nr,
                                        int& status) {
    const Grid& g = B.g;
    const int nx = g.nx, ny = g.ny;
    const size_t n = (size_t)nx * ny;
    const int lane = threadIdx.x & 31;
    const SlotLayout L = slot_layout<double>(nx, ny, B.maxr);
    double* tau = reinterpret_cast<double*>(base + L.tau);
    double* tst = reinterpret_cast<double*>(base + L.tst);
    double* Jx = reinterpret_cast<double*>(base + L.T);
    double* Jy = reinterpret_cast<double*>(base + L.delta);
    double2* DD = reinterpret_cast<double2*>(base + L.DD);
    Q4<double>* PK = reinterpret_cast<Q4<double>*>(base + L.PK);
    unsigned char* fl = base + L.flags;
    double* lam = reinterpret_cast<double*>(base + L.Ta);
    const double* sadj = reinterpret_cast<const double*>(base + L.sadj);
    int2* rng = reinterpret_cast<int2*>(base + L.rng);
    const int src = B.ev.src[e];
    const double* G = B.G + (size_t)src * n;
    const double* Gx = B.Gx + (size_t)src * n;
    const double* Gy = B.Gy + (size_t)src * n;
    const Q4<double>* mt = ISO ? nullptr : B.mt + (size_t)ip * n;
    const int r0 = B.ev.rec_ptr[e];
    // fixed source cells (src/eikonal_solver.cpp:118-129)
    int fy0 = ny, fy1 = -1;
    for (int iy = lane; iy < ny; iy += 32)
        if (fabs((g.yy[iy] - si.y0) / g.dy) <= 1.0) {
            fy0 = min(fy0, iy);
            fy1 = max(fy1, iy);
        }
    for (int o = 16; o > 0; o >>= 1) {
        fy0 = min(fy0, __shfl_xor_sync(FULL_MASK, fy0, o));
        fy1 = max(fy1, __shfl_xor_sync(FULL_MASK, fy1, o));
    }
    // 1. the winning stencils and their partials
    for_cells(nx, n, lane, [&](size_t k, int ix, int iy) {
        const bool fixed = iy >= fy0 && iy <= fy1 && ix >= si.fix_x0 && ix <= si.fix_x1;
        WinD w{};
        w.ok = false;
        if (!fixed) {
            const double aij = ISO ? B.a_f_row[iy] : mt[k].x;
            const double bij = ISO ? B.b_iso : mt[k].y;
            const double cij = ISO ? 0.0 : mt[k].z;
            w = discrete_winner(tau, PK, nx, ny, ix, iy, aij, bij, cij, g.dx, g.dy);
        }
        if (w.ok) {
            fl[k] = (unsigned char)(16u | (unsigned)w.dirx | ((unsigned)w.diry << 2));
            Jx[k] = w.jx;
            Jy[k] = w.jy;
            DD[k] = make_double2(w.df, w.dt0 * G[k] + w.dt0x * Gx[k] + w.dt0y * Gy[k]);
        } else {
            fl[k] = 0;
            Jx[k] = 0.0;
            Jy[k] = 0.0;
            DD[k] = make_double2(0.0, 0.0);
        }
    });
    __syncwarp();
    // 2. the receivers' explicit fun0 term, then the adjoint source g in the
    // tau plane (tau is no longer needed)
    double srec = 0.0;
    if (lane == 0)
        for (int ir = 0; ir < nr; ir++) {
            const double d = sadj[ir];
            const int st = B.ev.rec_idx[r0 + ir];
            size_t kq[4];
            double wq[4];
            if (!isfinite(d) ||
                !interp2d_weights(g.xx_deg, nx, g.yy_deg, ny, B.ev.stlo[st], B.ev.stla[st], kq, wq))
                continue;
            for (int q = 0; q < 4; q++) srec += d * wq[q] * tau[kq[q]] * G[kq[q]];
        }
    srec = __shfl_sync(FULL_MASK, srec, 0);
    __syncwarp();
    for (size_t k = lane; k < n; k += 32) tau[k] = 0.0;
    __syncwarp();
    if (lane == 0)
        for (int ir = 0; ir < nr; ir++) {
            const double d = sadj[ir];
            const int st = B.ev.rec_idx[r0 + ir];
            size_t kq[4];
            double wq[4];
            if (!isfinite(d) ||
                !interp2d_weights(g.xx_deg, nx, g.yy_deg, ny, B.ev.stlo[st], B.ev.stla[st], kq, wq))
                continue;
            for (int q = 0; q < 4; q++) tau[kq[q]] += d * wq[q] * PK[kq[q]].x;
        }
    __syncwarp();
    // 3. the sweep weights at every cell: the partials of the neighbours'
    // winners that read this cell
    for_cells(nx, n, lane, [&](size_t k, int ix, int iy) {
        const double wxm = (ix > 0 && (fl[k - 1] & 3u) == 2u) ? Jx[k - 1] : 0.0;
        const double wxp = (ix < nx - 1 && (fl[k + 1] & 3u) == 1u) ? Jx[k + 1] : 0.0;
        const double wym = (iy > 0 && ((fl[k - nx] >> 2) & 3u) == 2u) ? Jy[k - nx] : 0.0;
        const double wyp = (iy < ny - 1 && ((fl[k + nx] >> 2) & 3u) == 1u) ? Jy[k + nx] : 0.0;
        st4(PK + k, wxm, wxp, wym, wyp);
        lam[k] = 0.0;
        tst[k] = 0.0;
    });
    for (int iy = lane; iy < ny; iy += 32) {
        rng[iy] = make_int2(0, nx - 1);
        rng[ny + iy] = make_int2(0x7fffffff, -1);
        rng[2 * ny + iy] = make_int2(0x7fffffff, -1);
    }
    __syncwarp();
    // 4. lambda to its fixed point
    AdjPolicyLinear64 Q;
    Q.nx = nx;
    Q.ny = ny;
    Q.rng = rng;
    Q.crng = rng + ny;
    Q.rng2 = rng + 2 * ny;
    Q.W = PK;
    Q.C0 = tau;
    Q.Ta = lam;
    Q.Ta_start = tst;
    int iters = 0;
    for (int iter = 0; iter < 2000; iter++) {
        double l1 = 0.0, linf = 0.0;
        for (int sw = 0; sw < 4; sw++) systolic_sweep(Q, sweep_xd(sw), sweep_yd(sw), sw == 3, l1, linf);
        iters = iter + 1;
        if (warp_max(linf) == 0.0) break;
        if (iter == 1999) status = ST_NOCONV;
    }
    if (lane == 0 && B.out.adj_iters) B.out.adj_iters[e] = iters;
    // 5. dchi/dsvel = -dchi/dfun fun^2
    const double* fun = B.fun64 + (size_t)ip * n;
    double* acc = B.out.adj_s ? B.out.adj_s + (size_t)ip * n : nullptr;
    double* con = B.out.contrib ? B.out.contrib + (size_t)(e - B.out.contrib_e0) * n : nullptr;
    double s0 = 0.0;
    bool finite = true;
    for (size_t k = lane; k < n; k += 32) {
        const double lk = lam[k];
        s0 += lk * DD[k].y;
        const double gf = (fl[k] & 16u) ? lk * DD[k].x : 0.0;
        const double v = -gf * (fun[k] * fun[k]);
        if (!isfinite(v)) finite = false;
        if (con) con[k] = v;
        else if (acc && v != 0.0) atomicAdd(acc + k, v);
    }
    const double S = srec + warp_sum(s0);
    __syncwarp();
    if (lane == 0) {
        const int i0 = si.idx0, j0 = si.idy0;
        const size_t kk[4] = {(size_t)j0 * nx + i0, (size_t)(j0 + 1) * nx + i0,
                              (size_t)j0 * nx + i0 + 1, (size_t)(j0 + 1) * nx + i0 + 1};
        const double al[4] = {(1 - si.r1) * (1 - si.r2), (1 - si.r1) * si.r2,
                              si.r1 * (1 - si.r2), si.r1 * si.r2};
        for (int q = 0; q < 4; q++) {
            const double v = -(al[q] * S) * (fun[kk[q]] * fun[kk[q]]);
            if (!isfinite(v)) finite = false;
            if (con) con[kk[q]] += v;
            else if (acc && v != 0.0) atomicAdd(acc + kk[q], v);
        }
    }
    if (!__all_sync(FULL_MASK, finite)) status = ST_NONFINITE;
    // the delta plane is zero between events
    for (size_t k = lane; k < n; k += 32) Jy[k] = 0.0;
    __syncwarp();
}

// One event of the batch on the warp's scratch slot `base` (laid out for
// this event's grid).  Shared by the single-grid persistent kernel and the
// multi-grid one (one launch over plans of different grid sizes).
// `clear_delta`: the slot last held an event of another grid size, whose
// planes overlap this grid's adjoint-source plane, so it is zeroed first (in
// a single-grid launch it is zero between events by construction).
template <class S, bool ISO, int VAR>
__device__ __forceinline__ void batch_event(const BatchArgs<S>& B, unsigned int e,
                                            unsigned char* base, bool clear_delta = false,
                                            BlockTeams* bt = nullptr) {
    const int lane = threadIdx.x & 31;
    const Grid& g = B.g;
    const int nx = g.nx, ny = g.ny;
    const size_t n = (size_t)nx * ny;
    const SlotLayout L = slot_layout<S>(nx, ny, B.maxr);
    S* P_tau = reinterpret_cast<S*>(base + L.tau);
    S* P_tst = reinterpret_cast<S*>(base + L.tst);
    double* P_T = reinterpret_cast<double*>(base + L.T);
    double* P_delta = reinterpret_cast<double*>(base + L.delta);   // zero between events
    double* P_sadj = reinterpret_cast<double*>(base + L.sadj);
    double* P_syn = reinterpret_cast<double*>(base + L.syn);
    Q4<S>* P_pk = reinterpret_cast<Q4<S>*>(base + L.PK);
    unsigned char* P_fl = base + L.flags;
    int2* P_rng = reinterpret_cast<int2*>(base + L.rng);
    {
        const int ip = B.ev.iper[e];
        const int r0 = B.ev.rec_ptr[e];
        const int nr = B.ev.rec_ptr[e + 1] - r0;
        const SrcInfo si = source_info(g, B.ev.evlo[e], B.ev.evla[e]);
        int status = ST_OK;
        const double* T = P_T;

        if (B.mode != MODE_ADJ_ONLY) {
            int iters = 0;
            fwd_solve<S, ISO, VAR>(B, si, ip, B.ev.src[e], P_tau, P_tst, P_pk, P_fl, P_rng,
                                   P_T, iters, status, bt);
            if (lane == 0 && B.out.fwd_iters) B.out.fwd_iters[e] = iters;
            if (B.out.T_out)
                for (size_t k = lane; k < n; k += 32) B.out.T_out[(size_t)e * n + k] = P_T[k];
            // synthetic times at the receivers (src/preproc.cpp:105-115)
            for (int ir = lane; ir < nr; ir += 32) {
                const int st = B.ev.rec_idx[r0 + ir];
                const double ts =
                    interp2d_pt(g.xx_deg, nx, g.yy_deg, ny, P_T, B.ev.stlo[st], B.ev.stla[st]);
                if (B.out.syn) B.out.syn[r0 + ir] = ts;
                P_syn[ir] = ts;
                // residual adjoint source (src/preproc.cpp:111-115), or a
                // caller-given one (the vector-Jacobian product of T_rec)
                // (a forward-only run reads neither: tt_obs, weight may be NULL)
                P_sadj[ir] = B.ev.sadj ? B.ev.sadj[r0 + ir]
                             : B.mode == MODE_FWD
                                 ? 0.0
                                 : B.ev.weight[r0 + ir] * (ts - B.ev.tt_obs[r0 + ir]);
            }
            __syncwarp();
            if (B.mode == MODE_FWD_ADJ && lane == 0 && B.out.chi_ev) {
                double s = 0.0;   // src/preproc.cpp:142, receivers in order
                for (int ir = 0; ir < nr; ir++) {
                    const double r = P_syn[ir] - B.ev.tt_obs[r0 + ir];
                    s += B.ev.weight[r0 + ir] * (r * r);
                }
                B.out.chi_ev[e] = 0.5 * s;
            }
        } else {
            T = B.ev.T_in + (size_t)e * n;
            for (int ir = lane; ir < nr; ir += 32) P_sadj[ir] = B.ev.sadj[r0 + ir];
            __syncwarp();
        }

        // pass 0: the adjoint of the residuals (or the given source); pass 1
        // (is_kden): the kernel-density adjoint, source -w at every receiver,
        // not masked and accumulated into kden_s (src/preproc.cpp:128-137)
        // the exact discrete adjoint replaces the passes (FP64 plans)
        bool discrete = false;
        if constexpr (sizeof(S) == sizeof(double)) {
            if (B.discrete && B.mode == MODE_FWD_ADJ) {
                discrete_adjoint<ISO>(B, e, base, si, ip, nr, status);
                discrete = true;
            }
        }
        const int npass = (B.mode == MODE_FWD || discrete) ? 0
                          : (B.mode == MODE_FWD_ADJ && B.out.kden_s && !B.ev.sadj) ? 2
                                                                                   : 1;
        if (clear_delta && npass > 0) {
            for (size_t k = lane; k < n; k += 32) P_delta[k] = 0.0;
            __syncwarp();
        }
        for (int pass = 0; pass < npass; pass++) {
            if (pass == 1) {
                for (int ir = lane; ir < nr; ir += 32) P_sadj[ir] = -B.ev.weight[r0 + ir] * 1.0;
                __syncwarp();
            }
            // adjoint source (src/eikonal_solver.cpp:354-375), receivers in order
            if (lane == 0) spread_delta(g, B.ev, r0, nr, P_sadj, P_delta, false);
            __syncwarp();
            const double* a_a = ISO ? nullptr : B.a_a64 + (size_t)ip * n;
            const double* b_p = ISO ? nullptr : B.b_p64 + (size_t)ip * n;
            const double* c_a = ISO ? nullptr : B.c_a64 + (size_t)ip * n;
            auto faceA = [&](int ix, int iy) -> double {
                if constexpr (ISO) return face_a1_iso(T, B.a_a_row64[iy], nx, ix, iy, g.dx, g.dy);
                else return face_a1(T, a_a, c_a, nx, ix, iy, g.dx, g.dy);
            };
            auto faceB = [&](int ix, int iy) -> double {
                if constexpr (ISO) return face_b1_iso(T, B.b_iso64, B.b_iso64, nx, ix, iy, g.dx, g.dy);
                else return face_b1(T, b_p, c_a, nx, ix, iy, g.dx, g.dy);
            };
            int iters = 0;
            const bool big = nx >= 3 && ny >= 3;
            if constexpr (sizeof(S) == sizeof(double)) {
                Q4<double>* P_AQ = reinterpret_cast<Q4<double>*>(base + L.AQ);
                double2* P_DD = reinterpret_cast<double2*>(base + L.DD);
                double* P_Ta = reinterpret_cast<double*>(base + L.Ta);
                double* P_Tst = reinterpret_cast<double*>(P_tst);
                // face fluxes (src/eikonal_solver.cpp:404-441): a2(ix) is a1(ix+1)
                // and b2(iy) is b1(iy+1), identical expressions in the reference
                for_cells(nx, n, lane, [&](size_t k, int ix, int iy) {
                    const bool interior = ix >= 1 && ix <= nx - 2 && iy >= 1 && iy <= ny - 2;
                    double a1p = 0, a2m = 0, b1p = 0, b2m = 0, d = 0;
                    if (interior) {
                        const double a1 = faceA(ix, iy), a2 = faceA(ix + 1, iy);
                        const double b1 = faceB(ix, iy), b2 = faceB(ix, iy + 1);
                        const double a1m = (a1 - fabs(a1)) / 2.0;
                        a1p = (a1 + fabs(a1)) / 2.0;
                        a2m = (a2 - fabs(a2)) / 2.0;
                        const double a2p = (a2 + fabs(a2)) / 2.0;
                        const double b1m = (b1 - fabs(b1)) / 2.0;
                        b1p = (b1 + fabs(b1)) / 2.0;
                        b2m = (b2 - fabs(b2)) / 2.0;
                        const double b2p = (b2 + fabs(b2)) / 2.0;
                        d = (a2p - a1m) / g.dx + (b2p - b1m) / g.dy;   // :479-481
                    }
                    st4(P_AQ + k, a1p, a2m, b1p, b2m);
                    P_DD[k] = make_double2(P_delta[k], d);
                    const double v0 = interior ? 100.0 : 0.0;   // :446-449
                    P_Ta[k] = v0;
                    P_Tst[k] = v0;
                });
                for (int iy = lane; iy < ny; iy += 32) {
                    P_rng[iy] = make_int2(1, nx - 2);
                    P_rng[ny + iy] = make_int2(0x7fffffff, -1);
                    P_rng[2 * ny + iy] = make_int2(0x7fffffff, -1);
                }
                __syncwarp();
                AdjPolicyExact Q;
                Q.nx = nx;
                Q.ny = ny;
                Q.dx = g.dx;
                Q.dy = g.dy;
                Q.aq = P_AQ;
                Q.dd = P_DD;
                Q.Ta = P_Ta;
                Q.Ta_start = P_Tst;
                Q.rng = P_rng;
                Q.crng = P_rng + ny;
                Q.rng2 = P_rng + 2 * ny;
                if (big)
                    for (int iter = 0; iter < 1000; iter++) {
                        double l1 = 0.0, linf = 0.0;
                        for (int sw = 0; sw < 4; sw++)
                            systolic_sweep(Q, sweep_xd(sw), sweep_yd(sw), sw == 3, l1, linf);
                        iters = iter + 1;
                        const double L1 = warp_sum(l1) / (double)(nx * ny);
                        const double Linf = warp_max(linf);
                        if (L1 < 1e-9 && Linf < 1e-9) break;
                    }
            } else {
                Q4<float>* P_W = reinterpret_cast<Q4<float>*>(base + L.W);
                float* P_C0 = reinterpret_cast<float*>(base + L.C0);
                float* P_Ta = reinterpret_cast<float*>(base + L.Ta);
                // weights of the rewritten update, computed in FP64 from FP64 T
                // (FP32 path: reciprocals instead of divisions)
                const double idx = 1.0 / g.dx, idy = 1.0 / g.dy;
                const double i4dx = 1.0 / (4.0 * g.dx), i4dy = 1.0 / (4.0 * g.dy);
                // (isotropic media: no cross term, whose c is zero)
                auto fA = [&](int ix, int iy) -> double {
                    const size_t k = (size_t)iy * nx + ix;
                    if constexpr (ISO) return -(T[k] - T[k - 1]) * idx * B.a_a_row64[iy];
                    const double av = 0.5 * (a_a[k] + a_a[k - 1]);
                    const double cv = 0.5 * (c_a[k] + c_a[k - 1]);
                    return -(T[k] - T[k - 1]) * idx * av
                           + (T[k + nx] - T[k - nx] + T[k - 1 + nx] - T[k - 1 - nx]) * i4dy * cv;
                };
                auto fB = [&](int ix, int iy) -> double {
                    const size_t k = (size_t)iy * nx + ix;
                    if constexpr (ISO) return -(T[k] - T[k - nx]) * idy * B.b_iso64;
                    const double bv = 0.5 * (b_p[k] + b_p[k - nx]);
                    const double cv = 0.5 * (c_a[k] + c_a[k - nx]);
                    return -(T[k] - T[k - nx]) * idy * bv
                           + (T[k + 1] - T[k - 1] + T[k + 1 - nx] - T[k - 1 - nx]) * i4dx * cv;
                };
                for_cells(nx, n, lane, [&](size_t k, int ix, int iy) {
                    const bool interior = ix >= 1 && ix <= nx - 2 && iy >= 1 && iy <= ny - 2;
                    float c0 = 0.f, wxm = 0.f, wxp = 0.f, wym = 0.f, wyp = 0.f;
                    if (interior) {
                        const double a1 = fA(ix, iy), a2 = fA(ix + 1, iy);
                        const double b1 = fB(ix, iy), b2 = fB(ix, iy + 1);
                        const double a1p = fmax(a1, 0.0), a1m = fmin(a1, 0.0);
                        const double a2p = fmax(a2, 0.0), a2m = fmin(a2, 0.0);
                        const double b1p = fmax(b1, 0.0), b1m = fmin(b1, 0.0);
                        const double b2p = fmax(b2, 0.0), b2m = fmin(b2, 0.0);
                        const double d = (a2p - a1m) * idx + (b2p - b1m) * idy;
                        if (!(fabs(d) < 1e-14)) {
                            const double id = 1.0 / d;
                            c0 = (float)(P_delta[k] * id);
                            wxm = (float)(a1p * idx * id);
                            wxp = (float)(-a2m * idx * id);
                            wym = (float)(b1p * idy * id);
                            wyp = (float)(-b2m * idy * id);
                        }
                    }
                    st4(P_W + k, wxm, wxp, wym, wyp);
                    P_C0[k] = c0;
                    const float v0 = interior ? 100.f : 0.f;
                    P_Ta[k] = v0;
                    P_tst[k] = v0;
                });
                for (int iy = lane; iy < ny; iy += 32) {
                    P_rng[iy] = make_int2(1, nx - 2);
                    P_rng[ny + iy] = make_int2(0x7fffffff, -1);
                    P_rng[2 * ny + iy] = make_int2(0x7fffffff, -1);
                }
                __syncwarp();
                AdjPolicyW32<variant_adj_lead(VAR)> Q;
                Q.nx = nx;
                Q.ny = ny;
                Q.W = P_W;
                Q.C0 = P_C0;
                Q.Ta = P_Ta;
                Q.Ta_start = P_tst;
                Q.rng = P_rng;
                Q.crng = P_rng + ny;
                Q.rng2 = P_rng + 2 * ny;
                unsigned helpers = 0;   // tail team (variants with teams)
                if (big)
                    for (int iter = 0; iter < 1000; iter++) {
                        double l1 = 0.0, linf = 0.0;
                        if constexpr (variant_teams(VAR)) {
                            const Team tm = bt ? team_begin(bt, helpers, 1, Q, ny)
                                               : Team{1, 0, nullptr, nullptr, nullptr, nullptr};
                            if (tm.W > 1) {
                                using PolA = AdjPolicyW32<variant_adj_lead(VAR)>;
                                linf = team_sweeps(
                                    reinterpret_cast<const PolA*>(bt->rec[threadIdx.x >> 5].pol), tm);
                                team_end(bt, tm, (ny - 2 + 31) >> 5, l1, linf);
                            } else {
                                for (int sw = 0; sw < 4; sw++)
                                    systolic_sweep(Q, sweep_xd(sw), sweep_yd(sw), sw == 3, l1,
                                                   linf);
                            }
                        } else {
                            for (int sw = 0; sw < 4; sw++)
                                systolic_sweep(Q, sweep_xd(sw), sweep_yd(sw), sw == 3, l1, linf);
                        }
                        iters = iter + 1;
                        const double L1 = warp_sum(l1) / (double)(nx * ny);
                        const double Linf = warp_max(linf);
                        if (L1 < 1e-9 && Linf < 1e-9) break;
                        // FP32 fixed point: no cell changed by more than a few
                        // ulps of the field's largest magnitude
                        float vm = 0.f;
                        const float4* T4 = reinterpret_cast<const float4*>(P_Ta);
                        for (size_t k = lane; k < n / 4; k += 32) {
                            const float4 q = T4[k];
                            vm = fmaxf(vm, fmaxf(fmaxf(fabsf(q.x), fabsf(q.y)),
                                                 fmaxf(fabsf(q.z), fabsf(q.w))));
                        }
                        for (size_t k = (n / 4) * 4 + lane; k < n; k += 32)
                            vm = fmaxf(vm, fabsf(P_Ta[k]));
                        const double vmax = warp_max((double)vm);
                        if (Linf <= 4.0 * 5.960464477539063e-08 * vmax) break;
                    }
                if constexpr (variant_teams(VAR)) {
                    if (bt) {
                        team_release(bt, helpers);
                        if (__shfl_sync(FULL_MASK, *(volatile int*)&bt->err, 0)) status = ST_TEAM;
                    }
                }
            }
            if (lane == 0 && B.out.adj_iters && pass == 0) B.out.adj_iters[e] = iters;
            if (lane == 0) spread_delta(g, B.ev, r0, nr, P_sadj, P_delta, true);
            bool finite = true;
            const S* TaS = reinterpret_cast<const S*>(base + L.Ta);
            if (pass == 1) {
                const double* inv3 = B.inv3 + (size_t)ip * n;
                double* acc = B.out.kden_s + (size_t)ip * n;
                for (size_t k = lane; k < n; k += 32) {
                    const double v = (double)TaS[k];
                    if (!isfinite(v)) finite = false;
                    const double c = v * inv3[k];
                    if (c != 0.0) atomicAdd(acc + k, c);
                }
            } else if (B.mode == MODE_ADJ_ONLY) {
                for (size_t k = lane; k < n; k += 32) {
                    const double v = (double)TaS[k];
                    if (!isfinite(v)) finite = false;
                    if (B.out.Ta_out) B.out.Ta_out[(size_t)e * n + k] = v;
                }
            } else {
                // mask (src/eikonal_solver.cpp:514-536) + accumulate (src/preproc.cpp:28-31)
                const MaskBox mb = mask_box(g, B.ev.evlo[e], B.ev.evla[e]);
                const double* inv3 = B.inv3 + (size_t)ip * n;
                double* acc = B.out.adj_s ? B.out.adj_s + (size_t)ip * n : nullptr;
                double* con = B.out.contrib
                                  ? B.out.contrib + (size_t)(e - B.out.contrib_e0) * n
                                  : nullptr;
                for_cells(nx, n, lane, [&](size_t k, int ix, int iy) {
                    double v = (double)TaS[k];
                    if (ix >= mb.ix_lo && ix <= mb.ix_hi && iy >= mb.iy_lo && iy <= mb.iy_hi) v = 0.0;
                    if (!isfinite(v)) finite = false;
                    if (B.out.Ta_out) B.out.Ta_out[(size_t)e * n + k] = v;
                    const double c = v * inv3[k];
                    if (con) con[k] = c;
                    else if (acc && c != 0.0) atomicAdd(acc + k, c);
                });
            }
            if (!__all_sync(FULL_MASK, finite)) status = ST_NONFINITE;
            __syncwarp();
        }
        if (lane == 0 && B.out.status) B.out.status[e] = status;
        __syncwarp();
    }
}

// Body of the persistent batch kernel (below), shared with the FP64 variant
// that reads the grid spacing from device memory (eik64.cu): one warp per
// scratch slot pulls events from the queue until it is empty.
template <class S, bool ISO, int VAR>
__device__ __forceinline__ void batch_body(const BatchArgs<S>& B) {
    if constexpr (variant_teams(VAR) && sizeof(S) == sizeof(float)) {
        // tail teams: block-shared offers, jobs and progress words.  Slots
        // are numbered across the blocks first (warp w of block b: slot
        // w * blocks + b), so that fewer slots in use than warps leave every
        // block with owners and helpers (one slot per block: a block per solve)
        const int slot = (int)(threadIdx.x >> 5) * (int)gridDim.x + (int)blockIdx.x;
        __shared__ BlockTeams bt;
        if (threadIdx.x == 0) {
            int owners = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++)
                owners += (w * (int)gridDim.x + (int)blockIdx.x) < B.sc.nslots;
            bt.idle = 0u;
            bt.busy = owners;
            bt.err = 0;
            for (int w = 0; w < 4; w++) bt.mail[w] = 0u;
        }
        __syncthreads();
        using PolF = FwdPolicyDelta32<ISO, variant_fwd_rolled(VAR)>;
        using PolA = AdjPolicyW32<variant_adj_lead(VAR)>;
        if (slot < B.sc.nslots) {
            unsigned char* base = B.sc.base + (size_t)slot * B.sc.slot_bytes;
            for (;;) {
                const unsigned int qi = warp_next_event(B.sc.queue);
                if (qi >= (unsigned)B.ev.ne) break;
                const unsigned int e = B.sc.order ? (unsigned)B.sc.order[qi] : qi;
                batch_event<S, ISO, VAR>(B, e, base, false, &bt);
            }
            if ((threadIdx.x & 31) == 0) atomicSub(&bt.busy, 1);
        }
        team_serve<PolF, PolA>(&bt);
    } else {
        const int slot = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        if (slot >= B.sc.nslots) return;
        unsigned char* base = B.sc.base + (size_t)slot * B.sc.slot_bytes;
        for (;;) {
            const unsigned int qi = warp_next_event(B.sc.queue);
            if (qi >= (unsigned)B.ev.ne) break;
            const unsigned int e = B.sc.order ? (unsigned)B.sc.order[qi] : qi;
            batch_event<S, ISO, VAR>(B, e, base);
        }
    }
}

template <class S, bool ISO, int VAR>
__global__ void __launch_bounds__(128, sizeof(S) == sizeof(double) ? SA_MINB64 : SA_MINB32)
batch_kernel(BatchArgs<S> B) {
    batch_body<S, ISO, VAR>(B);
}

// One persistent launch over the events of several plans (grid levels of
// different size): queue position qi -> code[qi] = level << 24 | event, each
// level's arguments in device memory, scratch slots sized for the largest
// level.  `code` is ordered by work across levels, so the long solves of the
// fine grids start first and the short ones fill the tail.
template <class S, bool ISO, int VAR>
__global__ void __launch_bounds__(128, sizeof(S) == sizeof(double) ? SA_MINB64 : SA_MINB32)
batch_multi_kernel(const BatchArgs<S>* __restrict__ levels, unsigned int ntotal,
                   const unsigned int* __restrict__ code, Scratch sc) {
    const int slot = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (slot >= sc.nslots) return;
    unsigned char* base = sc.base + (size_t)slot * sc.slot_bytes;
    for (;;) {
        const unsigned int qi = warp_next_event(sc.queue);
        if (qi >= ntotal) break;
        const unsigned int c = code[qi];
        batch_event<S, ISO, VAR>(levels[c >> 24], c & 0xffffffu, base, true);
    }
}

template <class S>
inline BatchArgs<S> make_batch_args(const BatchDesc& d);

template <>
inline BatchArgs<double> make_batch_args<double>(const BatchDesc& d) {
    BatchArgs<double> B{};
    B.g = d.g;
    B.iso = d.iso;
    B.fun = d.fun64;
    B.fun64 = d.fun64;
    B.inv3 = d.inv3;
    B.a_f_row = d.a_f_row64;
    B.a_a_row64 = d.a_a_row64;
    B.b_iso = d.b_iso;
    B.b_iso64 = d.b_iso;
    B.mt = reinterpret_cast<const Q4<double>*>(d.mt64);
    B.b_p64 = d.b_p64;
    B.a_a64 = d.a_a64;
    B.c_a64 = d.c_a64;
    B.G = d.G64;
    B.Gx = d.Gx64;
    B.Gy = d.Gy64;
    B.G64 = d.G64;
    B.ev = d.ev;
    B.out = d.out;
    B.sc = d.sc;
    B.maxr = d.maxr;
    B.mode = d.mode;
    B.discrete = d.discrete;
    return B;
}

template <>
inline BatchArgs<float> make_batch_args<float>(const BatchDesc& d) {
    BatchArgs<float> B{};
    B.g = d.g;
    B.iso = d.iso;
    B.fun = d.fun32;
    B.fun64 = d.fun64;
    B.inv3 = d.inv3;
    B.a_f_row = d.a_f_row32;
    B.a_a_row64 = d.a_a_row64;
    B.b_iso = d.b_iso32;
    B.b_iso64 = d.b_iso;
    B.mt = reinterpret_cast<const Q4<float>*>(d.mt32);
    B.b_p64 = d.b_p64;
    B.a_a64 = d.a_a64;
    B.c_a64 = d.c_a64;
    B.G = d.G32;
    B.Gx = d.Gx32;
    B.Gy = d.Gy32;
    B.G64 = d.G64;
    B.ev = d.ev;
    B.out = d.out;
    B.sc = d.sc;
    B.maxr = d.maxr;
    B.mode = d.mode;
    B.discrete = d.discrete;
    return B;
}

}  // namespace sa
