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
// Lane 0 reads its upwind row from memory (previous strip, final for this
// sweep); the strip's last lane reads its downwind row from memory (next
// strip, still old).  Every access is row-contiguous per lane.
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

// P must provide: types V (field value), X (neighbour aux), Cell {V v; X x;};
//   nrows(), ncols(), row(rp, yd), col(cp, xd), begin_row(iy, active),
//   load(iy, ix, last) -> Cell, load_nb(iy, ix) -> Cell,
//   update(cur, iy, ix, xm, xp, ym, yp, last, l1, linf) -> V,
//   store(iy, ix, v, last).
template <class P>
__device__ __forceinline__ void systolic_sweep(P& p, const int xd, const int yd, const bool last,
                                               double& l1, double& linf) {
    using V = typename P::V;
    using X = typename P::X;
    using Cell = typename P::Cell;
    const int lane = threadIdx.x & 31;
    const int NR = p.nrows();
    const int NC = p.ncols();
    for (int k0 = 0; k0 < NR; k0 += 32) {
        const int rp = k0 + lane;
        const bool act = rp < NR;
        const int nr_strip = min(32, NR - k0);
        const int iy = act ? p.row(rp, yd) : 0;
        p.begin_row(iy, act);
        Cell cur{}, nxt{};
        if (act && lane == 0) cur = p.load(iy, p.col(0, xd), last);
        V prev_v = V(0);
        X prev_x = X(0);
        const int nsteps = NC + nr_strip - 1;
        for (int t = 0; t < nsteps; ++t) {
            const int c = t - lane;
            const bool valid = act && c >= 0 && c < NC;
            const int cn = c + 1;
            if (act && cn >= 0 && cn < NC) nxt = p.load(iy, p.col(cn, xd), last);
            V up_v = __shfl_up_sync(FULL_MASK, prev_v, 1);
            X up_x = __shfl_up_sync(FULL_MASK, prev_x, 1);
            V dn_v = __shfl_down_sync(FULL_MASK, nxt.v, 1);
            X dn_x = __shfl_down_sync(FULL_MASK, nxt.x, 1);
            if (valid) {
                const int ix = p.col(c, xd);
                const bool has_up = rp > 0;
                const bool has_dn = rp + 1 < NR;
                if (lane == 0 && has_up) {
                    const Cell nb = p.load_nb(p.row(rp - 1, yd), ix);
                    up_v = nb.v;
                    up_x = nb.x;
                }
                if (lane == nr_strip - 1 && has_dn) {
                    const Cell nb = p.load_nb(p.row(rp + 1, yd), ix);
                    dn_v = nb.v;
                    dn_x = nb.x;
                }
                const Nb<V, X> upw_x{c > 0, prev_v, prev_x};
                const Nb<V, X> dnw_x{c + 1 < NC, nxt.v, nxt.x};
                const Nb<V, X> upw_y{has_up, up_v, up_x};
                const Nb<V, X> dnw_y{has_dn, dn_v, dn_x};
                const V nv = p.update(cur, iy, ix,
                                      xd > 0 ? upw_x : dnw_x, xd > 0 ? dnw_x : upw_x,
                                      yd > 0 ? upw_y : dnw_y, yd > 0 ? dnw_y : upw_y,
                                      last, l1, linf);
                p.store(iy, ix, nv, last);
                prev_v = nv;
                prev_x = cur.x;
            }
            cur = nxt;
        }
        __syncwarp();
    }
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
}

}  // namespace sa
