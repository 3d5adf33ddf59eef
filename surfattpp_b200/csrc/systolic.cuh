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
//   unsigned fl;}, kLead, nrows(), ncols(), stride() (row pitch), row(rp, yd),
//   col(cp, xd) (sweep-ordered -> grid index), begin_row(iy, active),
//   load(k, last) -> Cell and load_nb(k) -> Cell (v, x, fl) at grid offset k,
//   update(cur, ix, xm, xp, ym, yp, xd, yd) -> V with xm / ym the upwind and
//   xp / yp the downwind neighbours in sweep order, account(cur, v, l1, linf)
//   (last sweep of an iteration), store(k, v, write_v, write_start),
//   store_flag(k, f), cp_of(ix, xd) (grid x -> sweep-ordered column, the
//   inverse of col), rng and crng (per-row x ranges of flag bit 0 and of
//   cells changed in the current iteration, see below).
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

// Per-lane state of one strip's march.
template <class V, class X>
struct March {
    int lane, NC, ioff, eoff, nr_strip, xd, yd;
    bool act, has_up, has_dn, eup, edn, last;
    V prev_v;           // this lane's previous result (upwind-x of its next cell)
    X prev_x;
    unsigned bal;       // ballot of "changed" of the previous step
    unsigned pfl;       // flags of this lane's previous cell
    int rmin, rmax;     // grid x range of this row's cells left with bit 0 set
    int umin, umax;     // lane 0: grid x where its row changed (bit 0 set above)
    int cmin, cmax;     // grid x range of this row's cells changed in this march
    int uf, ul;         // sweep columns where the row above changed in this sweep
    int lf, ll;         // sweep columns where the strip's last row changed
};

// One step of the march.  cur = column c, nx1 = column c+1, ld = target of the
// load of column c+1+LEAD.  Loads are issued LEAD steps before their first
// use (as downwind-x / downwind-y neighbour); the caller either unrolls by
// LEAD+2 and rotates the buffer roles statically, so no register copy ever
// waits on a load in flight, or (LEAD 1, long updates) runs one copy of the
// step and moves the buffers down after it.  Cells are addressed by their
// grid offset: ioff = this lane's row, eoff = the seam row streamed by the
// strip's first lane (eup, the row above) or last lane (edn, the row below);
// no lane does both, since a strip with one row is the grid's last.
template <int LEAD, class P, class Cell, class V, class X>
__device__ __forceinline__ void systolic_step(P& p, March<V, X>& L, const int t, Cell& cur,
                                              Cell& nx1, Cell& ld, Cell& ecur, Cell& eld,
                                              double& l1, double& linf) {
    const int lane = L.lane, NC = L.NC, xd = L.xd;
    const int c = t - lane;
    const bool valid = L.act && (unsigned)c < (unsigned)NC;
    const int c2 = c + 1 + LEAD;
    if (L.act && (unsigned)c2 < (unsigned)NC) {
        const int ix2 = p.col(c2, xd);
        ld = p.load(L.ioff + ix2, L.last);
        if (L.eup || L.edn) eld = p.load_nb(L.eoff + ix2);
    }
    V up_v = __shfl_up_sync(FULL_MASK, L.prev_v, 1);
    X up_x = __shfl_up_sync(FULL_MASK, L.prev_x, 1);
    V dn_v = __shfl_down_sync(FULL_MASK, nx1.v, 1);
    X dn_x = __shfl_down_sync(FULL_MASK, nx1.x, 1);
    if (L.eup) {
        up_v = ecur.v;
        up_x = ecur.x;
    }
    if (L.edn) {
        dn_v = ecur.v;
        dn_x = ecur.x;
    }
    bool work = true;
    if constexpr (P::kFlags) {
        // left neighbour changed: own bit of the last ballot; upper: lane-1's
        // bit (the strip's first lane reads bit 1 of the row above, current
        // only where that row changed in this sweep)
        unsigned up_chg = lane > 0 ? (L.bal >> (lane - 1)) & 1u : 0u;
        if (L.eup) up_chg = (c >= L.uf && c <= L.ul) ? (ecur.fl >> 1) & 1u : 0u;
        const bool dirty = valid && (((cur.fl | (L.bal >> lane) | up_chg) & 1u) != 0u);
        work = __any_sync(FULL_MASK, dirty);
    }
    bool chg = false;
    int ix = 0;
    if (valid) {
        ix = p.col(c, xd);
        V nv = cur.v;
        if (work)
            nv = p.update(cur, ix, Nb<V, X>{c > 0, L.prev_v, L.prev_x},
                          Nb<V, X>{c + 1 < NC, nx1.v, nx1.x}, Nb<V, X>{L.has_up, up_v, up_x},
                          Nb<V, X>{L.has_dn, dn_v, dn_x}, xd, L.yd);
        chg = !same_bits(nv, cur.v);
        bool wst = false;
        if (L.last) {
            p.account(cur, nv, l1, linf);
            wst = !same_bits(nv, cur.vs);
        }
        if (chg || wst) p.store(L.ioff + ix, nv, chg, wst);
        if (chg) {
            L.cmin = min(L.cmin, ix);
            L.cmax = max(L.cmax, ix);
        }
        L.prev_v = nv;
        L.prev_x = cur.x;
    }
    const unsigned nbal = __ballot_sync(FULL_MASK, chg);
    // flags of the previous cell (r', c-1): changed at its visit; a later
    // neighbour (right = this cell, lower = lane+1's cell of this step) changed
    if constexpr (P::kFlags) {
        if (L.act && c >= 1 && c <= NC) {
            const int ixp = p.col(c - 1, xd);
            const unsigned lower = (lane + 1 < L.nr_strip) ? (nbal >> (lane + 1)) & 1u : 0u;
            const unsigned f = (((L.bal >> lane) & 1u) << 1) | ((nbal >> lane) & 1u) | lower;
            if (f != L.pfl) p.store_flag(L.ioff + ixp, f);
            if (f & 1u) {
                L.rmin = min(L.rmin, ixp);
                L.rmax = max(L.rmax, ixp);
            }
        }
        if (L.eup && chg) {
            p.store_flag(L.eoff + ix, ecur.fl | 1u);
            L.umin = min(L.umin, ix);
            L.umax = max(L.umax, ix);
        }
        if (valid) L.pfl = cur.fl;
    }
    if ((nbal >> (L.nr_strip - 1)) & 1u) {
        const int cl = t - (L.nr_strip - 1);
        L.lf = min(L.lf, cl);
        L.ll = max(L.ll, cl);
    }
    L.bal = nbal;
}

// Marching only where something can change.  Per row the policy keeps the
// grid x range of its cells with flag bit 0 set (p.rng[iy], empty when
// x > y).  A strip's cells can only change from column `first` on: the
// first column of its rows' ranges, or where the row above changed in this
// sweep.  Before it every cell is clean and stays so, so the march starts
// there: each lane takes its previous cell (value, aux, flags) from memory
// and the pipeline is filled from that column.  After `lastd` (the last such
// column) and one step in which no cell changed, nothing can change any
// more: the march stops.  A strip with nothing to do is not marched.
// The last sweep of an iteration also visits every cell that changed since
// the iteration began (p.crng[iy], the x range of such cells per row): only
// those can add to the convergence sums or differ from the
// start-of-iteration copy; every other cell adds an exact zero.  All of
// this is exact: the cells not visited are exactly those the full march
// would have left bit-identical and whose sums terms are zero.
//
// Without flags (P::kFlags false: short updates, where the per-cell
// bookkeeping costs more than the updates it saves) every cell of the march
// is updated, and the ranges come from changes instead: a cell can only
// change in the next sweep if one of its four neighbours changed in this one
// (every cell that could change in this sweep was visited in it), so the
// next sweep's range of row r is the union of this sweep's changed ranges of
// rows r-1, r, r+1 widened by one column (p.rng2, swapped in at the end of
// the sweep).
//
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
    const int S = p.stride();
    int uf = NC, ul = -1;   // changes of the row above the current strip
    for (int k0 = 0; k0 < NR; k0 += 32) {
        const int rp = k0 + lane;
        const bool act = rp < NR;
        const int nr_strip = min(32, NR - k0);
        const int iy = act ? p.row(rp, yd) : 0;
        // columns (sweep order) this strip's march must cover
        int fc = NC, lc = -1;
        if (act) {
            int2 r = p.rng[iy];
            if (last) {
                const int2 q = p.crng[iy];
                r.x = min(r.x, q.x);
                r.y = max(r.y, q.y);
            }
            if (r.x <= r.y) {
                const int a = p.cp_of(r.x, xd), b = p.cp_of(r.y, xd);
                fc = min(a, b);
                lc = max(a, b);
            }
        }
        const int first = min(__reduce_min_sync(FULL_MASK, fc), uf);
        const int lastd = max(__reduce_max_sync(FULL_MASK, lc), ul);
        if (first >= NC) {   // no cell of the strip can change
            uf = NC;
            ul = -1;
            continue;
        }
        March<V, X> L;
        L.lane = lane;
        L.NC = NC;
        L.xd = xd;
        L.yd = yd;
        L.last = last;
        L.act = act;
        L.nr_strip = nr_strip;
        L.ioff = iy * S;
        L.has_up = act && rp > 0;
        L.has_dn = act && rp + 1 < NR;
        // strip-edge lanes also stream the neighbouring row of the adjacent
        // strip, with the same lead as their own row
        L.eup = lane == 0 && L.has_up;
        L.edn = lane == nr_strip - 1 && L.has_dn;
        const int iy_up = L.eup ? p.row(rp - 1, yd) : 0;
        L.eoff = L.eup ? iy_up * S : (L.edn ? p.row(rp + 1, yd) * S : 0);
        L.uf = uf;
        L.ul = ul;
        L.lf = NC;
        L.ll = -1;
        L.rmin = 0x7fffffff;
        L.rmax = -1;
        L.umin = 0x7fffffff;
        L.umax = -1;
        L.cmin = 0x7fffffff;
        L.cmax = -1;
        L.bal = 0u;
        L.pfl = 0u;
        L.prev_v = V(0);
        L.prev_x = X(0);
        p.begin_row(iy, act);
        // this lane's first column and the cell before it
        const int c0 = first - lane;
        if (act && c0 >= 1) {
            const Cell q = p.load_nb(L.ioff + p.col(c0 - 1, xd));
            L.prev_v = q.v;
            L.prev_x = q.x;
            L.pfl = q.fl;
        }
        Cell buf[NB], eb[NB];
        // columns c0 .. c0+LEAD (what earlier steps would have loaded)
#pragma unroll
        for (int q = 0; q < NB; q++) {
            buf[q] = Cell{};
            eb[q] = Cell{};
            const int cq = c0 + q;
            if (q <= LEAD && act && cq >= 0 && cq < NC) {
                const int ixq = p.col(cq, xd);
                buf[q] = p.load(L.ioff + ixq, last);
                if (L.eup || L.edn) eb[q] = p.load_nb(L.eoff + ixq);
            }
        }
        // one step more than the march: the last cell's flags are written
        // one step after its visit
        const int nsteps = NC + nr_strip;
        if constexpr (P::kRolled && LEAD == 1) {
            // one copy of the step (long updates: instruction-cache footprint
            // over register moves); the load of this step lands in `ld` and
            // moves down the buffer at the end of the step
            Cell cur = buf[0], nx1 = buf[1], ecur = eb[0], enx1 = eb[1];
            for (int t = first; t < nsteps; t++) {
                Cell ld = cur, eld = ecur;
                systolic_step<LEAD>(p, L, t, cur, nx1, ld, ecur, eld, l1, linf);
                cur = nx1;
                nx1 = ld;
                ecur = enx1;
                enx1 = eld;
                if (t - 31 > lastd && L.bal == 0u) break;
            }
        } else {
            for (int t = first; t < nsteps; t += NB) {
#pragma unroll
                for (int i = 0; i < NB; i++) {
                    if (t + i < nsteps)
                        systolic_step<LEAD>(p, L, t + i, buf[i % NB], buf[(i + 1) % NB],
                                            buf[(i + 1 + LEAD) % NB], eb[i % NB],
                                            eb[(i + 1 + LEAD) % NB], l1, linf);
                }
                if (t + NB - 1 - 31 > lastd && L.bal == 0u) break;
            }
        }
        if constexpr (!P::kFlags) {
            // next sweep's ranges: this row's changes widened by a column, in
            // this row and the rows above and below
            const bool any = L.cmin <= L.cmax;
            const int lo = any ? max(L.cmin - 1, p.col(0, 1)) : 0x7fffffff;
            const int hi = any ? min(L.cmax + 1, p.col(NC - 1, 1)) : -1;
            int nlo = lo, nhi = hi;
            const int alo = __shfl_up_sync(FULL_MASK, lo, 1);
            const int ahi = __shfl_up_sync(FULL_MASK, hi, 1);
            const int blo = __shfl_down_sync(FULL_MASK, lo, 1);
            const int bhi = __shfl_down_sync(FULL_MASK, hi, 1);
            if (lane > 0) {
                nlo = min(nlo, alo);
                nhi = max(nhi, ahi);
            }
            if (lane < 31) {
                nlo = min(nlo, blo);
                nhi = max(nhi, bhi);
            }
            if (act && nlo <= nhi) {
                int2 r = p.rng2[iy];
                r.x = min(r.x, nlo);
                r.y = max(r.y, nhi);
                p.rng2[iy] = r;
            }
            __syncwarp();
            // the rows outside the strip
            if (any && (L.eup || L.edn)) {
                const int iy_o = L.eup ? iy_up : p.row(rp + 1, yd);
                int2 r = p.rng2[iy_o];
                r.x = min(r.x, lo);
                r.y = max(r.y, hi);
                p.rng2[iy_o] = r;
            }
        }
        // every cell of the row that had bit 0 set was visited: the range is
        // replaced; lane 0 then adds where it set bit 0 in the row above.
        // Cells changed since the iteration began: added to, or (after the
        // last sweep, whose copy makes start == current) cleared.
        if (act) {
            if constexpr (P::kFlags) p.rng[iy] = make_int2(L.rmin, L.rmax);
            if (last) {
                p.crng[iy] = make_int2(0x7fffffff, -1);
            } else if (L.cmin <= L.cmax) {
                int2 q = p.crng[iy];
                q.x = min(q.x, L.cmin);
                q.y = max(q.y, L.cmax);
                p.crng[iy] = q;
            }
        }
        __syncwarp();
        if (P::kFlags && L.eup && L.umin <= L.umax) {
            int2 r = p.rng[iy_up];
            r.x = min(r.x, L.umin);
            r.y = max(r.y, L.umax);
            p.rng[iy_up] = r;
        }
        uf = L.lf;
        ul = L.ll;
        __syncwarp();
    }
    if constexpr (!P::kFlags) {
        int2* nxt = p.rng2;
        p.rng2 = p.rng;
        p.rng = nxt;
        for (int iy = lane; iy < p.ny; iy += 32) p.rng2[iy] = make_int2(0x7fffffff, -1);
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
