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

// A team of warps of one block marching one solve (cooperative sweeps).
// Strip j of a sweep (in sweep order) is marched by member j % W, each strip
// a fixed lag behind the one before it: a strip's first lane streams the row
// above from memory, so at its step t it needs the previous strip's last row
// finished up to column t + 1 + lead.  Every member publishes, in its word,
// the strip it marches and the last column its last row has finished (or
// that the strip is done: its stores, its range updates and its strip
// record are then visible); a member waits on the word of the strip before
// its own.  A strip is finished only after the strip before it, so the last
// strip of a sweep being done means the whole sweep is.  Cells are updated
// exactly as by one warp (the same neighbour values reach every update); a
// member that cannot yet know where the previous strip's last row changed
// starts its march at the previous strip's first column, and marching more
// cells than needed changes nothing (an update whose inputs did not change
// reproduces the cell).  Every wait is bounded: when it gives up, the team's
// error flag is set and the march goes on without it.
struct Team {
    int W;                       // members (1: the warp alone)
    int r;                       // this warp's role
    unsigned long long* word;    // [W] (shared): strip id << 32 | (column + 1)
    int4* sinfo;                 // per solve [strips]: {first, lf, ll, -} of strip j
    double* sums;                // per solve [strips][32]: last-sweep L1 partials
    int* err;                    // set when a wait gave up
};
constexpr int kStripDone = 0x7ffffff0;          // column value: strip finished
constexpr unsigned kTeamEnd = 0xffffffffu;       // strip id: member finished its sweeps
constexpr long long kTeamWaitNs = 2000000000ll;  // a wait gives up after 2 s

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.cta.shared.u64 %0, [%1];"
                 : "=l"(v)
                 : "r"((unsigned)__cvta_generic_to_shared(p))
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.cta.shared.u64 [%0], %1;"
                 :
                 : "r"((unsigned)__cvta_generic_to_shared(p)), "l"(v)
                 : "memory");
}
__device__ __forceinline__ long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return (long long)t;
}
__device__ __forceinline__ unsigned long long team_word(unsigned id, int col) {
    return ((unsigned long long)id << 32) | (unsigned)(col + 1);
}

// Waits (all lanes) until strip `id`, marched by member `role`, has its last
// row finished up to column c or is done; returns the column reached
// (kStripDone when the strip is finished, or when the wait gave up).
__device__ __forceinline__ int team_wait(const Team& T, int role, unsigned id, int c) {
    long long t0 = 0;
    for (int spin = 0;; spin++) {
        // after a wait of the block gave up, none waits any more
        if (__shfl_sync(FULL_MASK, *(volatile int*)T.err, 0) != 0) return kStripDone;
        // every lane acquires; lane 0's value decides, so the warp stays converged
        const unsigned long long w =
            __shfl_sync(FULL_MASK, ld_acquire_u64(T.word + role), 0);
        const unsigned wid = (unsigned)(w >> 32);
        const int col = (int)(unsigned)(w & 0xffffffffu) - 1;
        if (wid > id) return kStripDone;   // the member moved on: strip done
        if (wid == id && col >= c) return col;
        const long long now = __shfl_sync(FULL_MASK, global_ns(), 0);
        if (spin == 0) {
            t0 = now;
        } else if (now - t0 > kTeamWaitNs) {
            if ((threadIdx.x & 31) == 0) atomicExch(T.err, 1);
            return kStripDone;
        }
        if (spin >= 16) __nanosleep(32);
    }
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
//
// P::kCoop policies (the FP32 sweeps) accumulate the last sweep's L1 sum per
// strip and add the strip sums in strip order, so that a team (`tm`, `sweep`
// = 0..3 within the iteration) and a warp alone round it identically.
template <class P>
__device__ __forceinline__ void systolic_sweep(P& p, const int xd, const int yd, const bool last,
                                               double& l1, double& linf,
                                               const Team* tm = nullptr, const int sweep = 0) {
    using V = typename P::V;
    using X = typename P::X;
    using Cell = typename P::Cell;
    constexpr int LEAD = P::kLead;
    constexpr int NB = LEAD + 2;
    const int lane = threadIdx.x & 31;
    const int NR = p.nrows();
    const int NC = p.ncols();
    const int S = p.stride();
    const int nstrip = (NR + 31) >> 5;
    const bool coop = P::kCoop && tm != nullptr && tm->W > 1;
    const int W = coop ? tm->W : 1;
    const int me = coop ? tm->r : 0;
    const unsigned id0 = 1u + (unsigned)sweep * (unsigned)nstrip;   // strip id of strip 0
    if (coop && me == 0) {
        // strip 0 follows the previous sweep's last strip; once that one is
        // done the whole sweep is, and next sweep's ranges can be cleared
        if (sweep > 0 && (nstrip - 1) % W != 0) team_wait(*tm, (nstrip - 1) % W, id0 - 1, kStripDone);
        if constexpr (!P::kFlags)
            for (int iy = lane; iy < p.ny; iy += 32) p.rng2[iy] = make_int2(0x7fffffff, -1);
        __threadfence();
        __syncwarp();
    }
    int uf = NC, ul = -1;   // changes of the row above the current strip
    for (int j = me; j < nstrip; j += W) {
        const int k0 = j * 32;
        const unsigned id = id0 + (unsigned)j;
        const int rp = k0 + lane;
        const bool act = rp < NR;
        const int nr_strip = min(32, NR - k0);
        const int iy = act ? p.row(rp, yd) : 0;
        // team: nothing of the strip is read before the strip ahead of it
        // has started -- then the previous sweep, whose strips wrote this
        // strip's ranges and rows in the reversed order, is complete
        const int prole = (coop && j > 0) ? (j - 1) % W : -1;
        int avail = kStripDone;
        if (prole >= 0) avail = team_wait(*tm, prole, id - 1, -1);
        // columns (sweep order) this strip's march must cover
        int fc = NC, lc = -1;
        if (act) {
            // (a team merges the ranges with atomics, performed in L2: read
            // them from there, not from a line this SM's L1 may hold)
            int2 r = coop ? __ldcg(p.rng + iy) : p.rng[iy];
            if (last) {
                const int2 q = coop ? __ldcg(p.crng + iy) : p.crng[iy];
                r.x = min(r.x, q.x);
                r.y = max(r.y, q.y);
            }
            if (r.x <= r.y) {
                const int a = p.cp_of(r.x, xd), b = p.cp_of(r.y, xd);
                fc = min(a, b);
                lc = max(a, b);
            }
        }
        const int fcm = __reduce_min_sync(FULL_MASK, fc);
        const int lcm = __reduce_max_sync(FULL_MASK, lc);
        // team: the strip before this one (its member, and how far its last
        // row is).  uf / ul are final once it is done; before that, once its
        // last row has passed column fcm - 1, the first column where that row
        // changed (kept current in its record) decides min(fcm, uf) exactly,
        // and ul stays unknown (no early stop until it is done)
        bool known = true;
        if (prole >= 0) {
            const int want = fcm < NC ? fcm - 1 : kStripDone;
            if (avail < want) avail = team_wait(*tm, prole, id - 1, want);
            const int4 q = tm->sinfo[j - 1];
            uf = q.y;
            ul = q.z;
            if (avail != kStripDone) {
                known = false;
                ul = -1;
            }
        }
        const int first = min(fcm, uf);
        int lastd = max(lcm, ul);
        if (first >= NC) {   // no cell of the strip can change
            if (coop) {
                // (one lane, the strip's last, writes its record and word)
                if (last) tm->sums[j * 32 + lane] = 0.0;
                __threadfence();
                __syncwarp();
                if (lane == nr_strip - 1) {
                    tm->sinfo[j] = make_int4(NC, NC, -1, 0);
                    st_release_u64(tm->word + me, team_word(id, kStripDone));
                }
            }
            uf = NC;
            ul = -1;
            continue;
        }
        // Progress is the last column the strip's last lane has visited (not
        // merely one its row cannot change at): up to there that lane has also
        // read the next strip's first row, which the next strip may then
        // overwrite.
        if (coop) {
            if (lane == nr_strip - 1) {
                tm->sinfo[j] = make_int4(first, NC, -1, 0);
                st_release_u64(tm->word + me, team_word(id, -1));
            }
        }
        // the next column the first lane streams from the row above must be
        // finished by the strip before (coop only); kStripDone: wait until
        // that strip is done
        auto need = [&](int c) {
            if (known || c <= avail) return;
            if (c < kStripDone) {
                if (avail >= NC - 1) return;
                c = min(c, NC - 1);
            }
            avail = team_wait(*tm, prole, id - 1, c);
            if (avail == kStripDone) {
                known = true;
                ul = tm->sinfo[j - 1].z;
                lastd = max(lastd, ul);
            }
        };
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
        // the last sweep's L1 sum of this strip (kCoop) or the running sum
        double l1s = 0.0;
        double& l1r = P::kCoop ? l1s : l1;
        // this lane's first column and the cell before it
        const int c0 = first - lane;
        if (act && c0 >= 1) {
            const Cell q = p.load_nb(L.ioff + p.col(c0 - 1, xd));
            L.prev_v = q.v;
            L.prev_x = q.x;
            L.pfl = q.fl;
        }
        need(first + LEAD);
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
        const bool pub = coop && lane == nr_strip - 1;   // publishes the last row's progress
        if constexpr (P::kRolled && LEAD == 1) {
            // one copy of the step (long updates: instruction-cache footprint
            // over register moves); the load of this step lands in `ld` and
            // moves down the buffer at the end of the step
            Cell cur = buf[0], nx1 = buf[1], ecur = eb[0], enx1 = eb[1];
            for (int t = first; t < nsteps; t++) {
                if (coop) need(t + 1 + LEAD);
                Cell ld = cur, eld = ecur;
                systolic_step<LEAD>(p, L, t, cur, nx1, ld, ecur, eld, l1r, linf);
                cur = nx1;
                nx1 = ld;
                ecur = enx1;
                enx1 = eld;
                if (pub && (t & 7) == 7) {
                    tm->sinfo[j].y = L.lf;
                    st_release_u64(tm->word + me, team_word(id, min(max(t - lane, -1), NC - 1)));
                }
                if (known && t - 31 > lastd && L.bal == 0u) break;
            }
        } else {
            for (int t = first; t < nsteps; t += NB) {
                if (coop) need(t + NB + LEAD);
#pragma unroll
                for (int i = 0; i < NB; i++) {
                    if (t + i < nsteps)
                        systolic_step<LEAD>(p, L, t + i, buf[i % NB], buf[(i + 1) % NB],
                                            buf[(i + 1 + LEAD) % NB], eb[i % NB],
                                            eb[(i + 1 + LEAD) % NB], l1r, linf);
                }
                if (pub) {
                    tm->sinfo[j].y = L.lf;
                    st_release_u64(tm->word + me,
                                   team_word(id, min(max(t + NB - 1 - lane, -1), NC - 1)));
                }
                if (known && t + NB - 1 - 31 > lastd && L.bal == 0u) break;
            }
        }
        if constexpr (!P::kFlags) {
            // next sweep's ranges: this row's changes widened by a column, in
            // this row and the rows above and below (a team's neighbouring
            // strips merge into the same rows: atomics)
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
            auto merge = [&](int row, int a, int b) {
                if (coop) {
                    int* q = reinterpret_cast<int*>(p.rng2 + row);
                    atomicMin(q, a);
                    atomicMax(q + 1, b);
                } else {
                    int2 r = p.rng2[row];
                    r.x = min(r.x, a);
                    r.y = max(r.y, b);
                    p.rng2[row] = r;
                }
            };
            if (act && nlo <= nhi) merge(iy, nlo, nhi);
            __syncwarp();
            // the rows outside the strip
            if (any && (L.eup || L.edn)) merge(L.eup ? iy_up : p.row(rp + 1, yd), lo, hi);
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
                int2 q = coop ? __ldcg(p.crng + iy) : p.crng[iy];
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
        if constexpr (P::kCoop) {
            if (!coop) l1 += l1s;
            else if (last) tm->sums[j * 32 + lane] = l1s;
        }
        if (coop) {
            // finished after the strip before it (then ul is final), with its
            // stores, range updates and record visible
            need(kStripDone);
            __threadfence();
            __syncwarp();
            if (lane == nr_strip - 1) {
                tm->sinfo[j].y = L.lf;
                tm->sinfo[j].z = L.ll;
                st_release_u64(tm->word + me, team_word(id, kStripDone));
            }
        }
        uf = L.lf;
        ul = L.ll;
        __syncwarp();
    }
    if constexpr (!P::kFlags) {
        int2* nxt = p.rng2;
        p.rng2 = p.rng;
        p.rng = nxt;
        // (a team clears them at the next sweep's start, after this sweep)
        if (!coop) {
            for (int iy = lane; iy < p.ny; iy += 32) p.rng2[iy] = make_int2(0x7fffffff, -1);
            __syncwarp();
        }
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
