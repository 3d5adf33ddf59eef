// Warp-systolic Gauss-Seidel sweep.
//
// One warp owns one (source, period) solve.  A sweep in direction (xd, yd)
// visits the grid in the reference's raster order (x outer, y inner, see
// src/eikonal_solver.cpp:149-154).  Each cell reads its 4 axis neighbours:
// the two upwind ones already updated in this sweep and the two downwind ones
// still holding the previous sweep's values.  Cells on one anti-diagonal
// (in sweep order) are therefore independent, and processing anti-diagonals
// in order reproduces raster-order Gauss-Seidel exactly.
//
// Mapping: rows are taken 32 at a time (a strip), lane j owns sweep-ordered
// row r' = 32k + j and marches along sweep-ordered column c' = t - j at step
// t.  At step t:
//   upwind-x   (r',   c'-1)  = this lane's own result of step t-1 (register)
//   upwind-y   (r'-1, c')    = lane j-1's result of step t-1   (__shfl_up)
//   downwind-x (r',   c'+1)  = this lane's prefetch, loaded in step t
//   downwind-y (r'+1, c')    = lane j+1's prefetch of step t  (__shfl_down)
// Lane 0 streams its upwind row from memory (previous strip, final for this
// sweep); the strip's last lane streams its downwind row (next strip, still
// old).  Every access is row-contiguous per lane and issued one step before
// its use.
#pragma once
#include "common.cuh"

namespace sa {

constexpr unsigned FULL_MASK = 0xffffffffu;

template <class V, class X>
struct Nb {
    bool has;
    V v;
    X x;
};

// Skipping unchanged cells.  A cell update is a function of the four
// neighbour values and the cell's own data only (the forward keeps
// min(current, candidates), the adjoint recomputes from its neighbours), so a
// cell none of whose neighbours changed since its last update would come out
// bit-identical: the sweep skips it.  This is exact -- fields, iteration
// counts and convergence sums are the same as updating every cell.
// Per cell a flag byte records
//   bit 0: a neighbour changed after the cell's last visit (update it next),
//   bit 1: the cell's value changed at its last visit.
// At its visit a cell is dirty if bit 0 is set or its left or upper
// neighbour (visited just before it in this sweep) changed.  The flags of a
// visited cell are written one step later, when its right neighbour (this
// lane) and lower neighbour (next lane) have been visited.  The strip's first
// lane reads bit 1 of the row above (previous strip) and sets bit 0 there when
// it changes.  A warp step whose 32 cells are all clean skips the update math.
// All flags start at 1 (every cell is updated at its first visit).
//
// P must provide: types V (field value), X (neighbour aux), Cell {V v; X x;
//   unsigned fl;}, nrows(), ncols(), row(rp, yd), col(cp, xd),
//   begin_row(iy, active), load(iy, ix, last) -> Cell, load_nb(iy, ix) -> Cell,
//   update(cur, iy, ix, xm, xp, ym, yp) -> V, account(cur, v, l1, linf)
//   (last sweep of an iteration), store(iy, ix, v, write_v, write_start),
//   store_flag(iy, ix, f).
template <class V>
__device__ __forceinline__ bool same_bits(V a, V b);
template <>
__device__ __forceinline__ bool same_bits<float>(float a, float b) {
    return __float_as_uint(a) == __float_as_uint(b);
}
template <>
__device__ __forceinline__ bool same_bits<double>(double a, double b) {
    return __double_as_longlong(a) == __double_as_longlong(b);
}

// One step of the march.  cur = column c, nx1 = column c+1, ld = target of the
// load of column c+1+LEAD.  Loads are issued LEAD steps before their first
// use (as downwind-x / downwind-y neighbour) and buffer roles rotate
// statically (the caller unrolls by LEAD+2), so no register copy ever waits
// on a load in flight.  bal = ballot of "changed" of the previous step,
// pfl = flags of this lane's previous cell.
template <int LEAD, class P, class Cell, class V, class X>
__device__ __forceinline__ void systolic_step(P& p, const int t, const int lane, const int NR,
                                              const int NC, const int rp, const bool act,
                                              const int iy, const bool edge_up,
                                              const bool edge_dn, const int iy_up,
                                              const int iy_dn, const int nr_strip, const int xd,
                                              const int yd, const bool last, Cell& cur,
                                              Cell& nx1, Cell& ld, Cell& ucur, Cell& uld,
                                              Cell& dcur, Cell& dld, V& prev_v, X& prev_x,
                                              unsigned& bal, unsigned& pfl, double& l1,
                                              double& linf) {
    const int c = t - lane;
    const bool valid = act && c >= 0 && c < NC;
    const int c2 = c + 1 + LEAD;
    if (act && c2 >= 0 && c2 < NC) {
        const int ix2 = p.col(c2, xd);
        ld = p.load(iy, ix2, last);
        if (edge_up) uld = p.load_nb(iy_up, ix2);
        if (edge_dn) dld = p.load_nb(iy_dn, ix2);
    }
    V up_v = __shfl_up_sync(FULL_MASK, prev_v, 1);
    X up_x = __shfl_up_sync(FULL_MASK, prev_x, 1);
    V dn_v = __shfl_down_sync(FULL_MASK, nx1.v, 1);
    X dn_x = __shfl_down_sync(FULL_MASK, nx1.x, 1);
    // left neighbour changed: own bit of the last ballot; upper: lane-1's bit
    // (the strip's first lane reads the row above)
    unsigned up_chg = lane > 0 ? (bal >> (lane - 1)) & 1u : 0u;
    if (edge_up) up_chg = (ucur.fl >> 1) & 1u;
    const bool dirty = valid && (((cur.fl | (bal >> lane) | up_chg) & 1u) != 0u);
    const bool work = __any_sync(FULL_MASK, dirty);
    bool chg = false;
    int ix = 0;
    if (valid) {
        ix = p.col(c, xd);
        const bool has_up = rp > 0;
        const bool has_dn = rp + 1 < NR;
        if (edge_up) {
            up_v = ucur.v;
            up_x = ucur.x;
        }
        if (edge_dn) {
            dn_v = dcur.v;
            dn_x = dcur.x;
        }
        V nv = cur.v;
        if (work) {
            const Nb<V, X> upw_x{c > 0, prev_v, prev_x};
            const Nb<V, X> dnw_x{c + 1 < NC, nx1.v, nx1.x};
            const Nb<V, X> upw_y{has_up, up_v, up_x};
            const Nb<V, X> dnw_y{has_dn, dn_v, dn_x};
            nv = p.update(cur, iy, ix, xd > 0 ? upw_x : dnw_x, xd > 0 ? dnw_x : upw_x,
                          yd > 0 ? upw_y : dnw_y, yd > 0 ? dnw_y : upw_y);
        }
        chg = !same_bits(nv, cur.v);
        bool wst = false;
        if (last) {
            p.account(cur, nv, l1, linf);
            wst = !same_bits(nv, cur.vs);
        }
        if (chg || wst) p.store(iy, ix, nv, chg, wst);
        prev_v = nv;
        prev_x = cur.x;
    }
    const unsigned nbal = __ballot_sync(FULL_MASK, chg);
    // flags of the previous cell (r', c-1): changed at its visit; a later
    // neighbour (right = this cell, lower = lane+1's cell of this step) changed
    if (act && c >= 1 && c <= NC) {
        const unsigned lower = (lane + 1 < nr_strip) ? (nbal >> (lane + 1)) & 1u : 0u;
        const unsigned f = (((bal >> lane) & 1u) << 1) | ((nbal >> lane) & 1u) | lower;
        if (f != pfl) p.store_flag(iy, p.col(c - 1, xd), f);
    }
    if (edge_up && chg) p.store_flag(iy_up, ix, ucur.fl | 1u);
    if (valid) pfl = cur.fl;
    bal = nbal;
}

// P::kLead = how many steps ahead a lane loads its row (1 for the long
// forward update, more for the short adjoint update).
template <class P>
__device__ __forceinline__ void systolic_sweep(P& p, const int xd, const int yd, const bool last,
                                               double& l1, double& linf) {
    using V = typename P::V;
    using X = typename P::X;
    using Cell = typename P::Cell;
    constexpr int LEAD = P::kLead;
    constexpr int NB = LEAD + 2;
    const int lane = threadIdx.x & 31;
    const int NR = p.nrows();
    const int NC = p.ncols();
    for (int k0 = 0; k0 < NR; k0 += 32) {
        const int rp = k0 + lane;
        const bool act = rp < NR;
        const int nr_strip = min(32, NR - k0);
        const int iy = act ? p.row(rp, yd) : 0;
        // strip-edge lanes also stream the neighbouring row of the adjacent
        // strip, with the same lead as their own row
        const bool edge_up = act && lane == 0 && rp > 0;
        const bool edge_dn = act && lane == nr_strip - 1 && rp + 1 < NR;
        const int iy_up = edge_up ? p.row(rp - 1, yd) : 0;
        const int iy_dn = edge_dn ? p.row(rp + 1, yd) : 0;
        p.begin_row(iy, act);
        Cell buf[NB], ub[NB], db[NB];
        // columns c .. c+LEAD of step 0 (what earlier steps would have loaded)
#pragma unroll
        for (int q = 0; q < NB; q++) {
            buf[q] = Cell{};
            ub[q] = Cell{};
            db[q] = Cell{};
            const int cq = q - lane;
            if (q <= LEAD && act && cq >= 0 && cq < NC) {
                const int ixq = p.col(cq, xd);
                buf[q] = p.load(iy, ixq, last);
                if (edge_up) ub[q] = p.load_nb(iy_up, ixq);
                if (edge_dn) db[q] = p.load_nb(iy_dn, ixq);
            }
        }
        V prev_v = V(0);
        X prev_x = X(0);
        unsigned bal = 0u, pfl = 0u;
        // one step more than the march: the last cell's flags are written
        // one step after its visit
        const int nsteps = NC + nr_strip;
        for (int t = 0; t < nsteps; t += NB) {
#pragma unroll
            for (int i = 0; i < NB; i++) {
                if (t + i < nsteps)
                    systolic_step<LEAD>(p, t + i, lane, NR, NC, rp, act, iy, edge_up, edge_dn,
                                        iy_up, iy_dn, nr_strip, xd, yd, last, buf[i % NB],
                                        buf[(i + 1) % NB], buf[(i + 1 + LEAD) % NB], ub[i % NB],
                                        ub[(i + 1 + LEAD) % NB], db[i % NB],
                                        db[(i + 1 + LEAD) % NB], prev_v, prev_x, bal, pfl, l1,
                                        linf);
            }
        }
        __syncwarp();
    }
}

// The four sweep directions of src/eikonal_solver.cpp:137-140 (and :466-469).
__device__ __forceinline__ int sweep_xd(int s) { return s < 2 ? 1 : -1; }
__device__ __forceinline__ int sweep_yd(int s) { return (s & 1) ? -1 : 1; }

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
}

}  // namespace sa
