// Per-event helpers shared by the FP64 and FP32 batch kernels: source
// bookkeeping, receiver interpolation, adjoint source spreading, adjoint
// face-flux coefficients, the source mask and the kernel accumulation.
// All arithmetic here is FP64 and follows the reference's association.
#pragma once
#include "common.cuh"
#include "systolic.cuh"

namespace sa {

// include/utils.h:28-36
__device__ __forceinline__ double bilinear64(const double* M, int nx, int idx0, int idy0,
                                             double r1, double r2) {
    return (1 - r1) * (1 - r2) * M[(size_t)idy0 * nx + idx0]
         + (1 - r1) * r2 * M[(size_t)(idy0 + 1) * nx + idx0]
         + r1 * (1 - r2) * M[(size_t)idy0 * nx + idx0 + 1]
         + r1 * r2 * M[(size_t)(idy0 + 1) * nx + idx0 + 1];
}

struct SrcInfo {
    double x0, y0;        // radians
    int idx0, idy0;       // source cell (clamped)
    double r1, r2;        // fractional offsets (src/eikonal_solver.cpp:71-77)
    int fix_x0, fix_x1;   // columns with |(xx - x0)/dx| <= 1 (empty if fix_x0 > fix_x1)
};

// src/eikonal_solver.cpp:71-77 and the near-source test of :119-120.
__device__ inline SrcInfo source_info(const Grid& g, double evlo, double evla) {
    SrcInfo s;
    s.x0 = evlo * DEG2RAD;
    s.y0 = evla * DEG2RAD;
    const double fx = floor((s.x0 - g.xx[0]) / g.dx);
    const double fy = floor((s.y0 - g.yy[0]) / g.dy);
    int idx0 = (int)fmax(-4.0, fmin((double)g.nx + 4.0, fx));
    int idy0 = (int)fmax(-4.0, fmin((double)g.ny + 4.0, fy));
    const int cx = idx0;
    idx0 = max(0, min(idx0, g.nx - 2));
    idy0 = max(0, min(idy0, g.ny - 2));
    s.idx0 = idx0;
    s.idy0 = idy0;
    s.r1 = fmin(1.0, (s.x0 - g.xx[idx0]) / g.dx);
    s.r2 = fmin(1.0, (s.y0 - g.yy[idy0]) / g.dy);
    s.fix_x0 = 1 << 30;
    s.fix_x1 = -1;
    for (int ix = max(0, cx - 3); ix <= min(g.nx - 1, cx + 4); ix++) {
        if (fabs((g.xx[ix] - s.x0) / g.dx) <= 1.0) {
            s.fix_x0 = min(s.fix_x0, ix);
            s.fix_x1 = max(s.fix_x1, ix);
        }
    }
    return s;
}

// include/utils.h:358-409 (one query point).
// The cell and bilinear weights interp2d uses for one point (row-major
// offsets k[4] of (i, j), (i+1, j), (i, j+1), (i+1, j+1)); false outside.
__device__ inline bool interp2d_weights(const double* xg, int nx, const double* yg, int ny,
                                        double qx, double qy, size_t* k, double* w) {
    if (qx < xg[0] || qx > xg[nx - 1] || qy < yg[0] || qy > yg[ny - 1]) return false;
    int lo = 0, hi = nx;   // lower_bound
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (xg[mid] < qx) lo = mid + 1;
        else hi = mid;
    }
    int i = lo;
    if (i == nx) --i;
    if (i > 0 && xg[i] > qx) --i;
    i = max(0, min(i, nx - 2));
    lo = 0;
    hi = ny;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (yg[mid] < qy) lo = mid + 1;
        else hi = mid;
    }
    int j = lo;
    if (j == ny) --j;
    if (j > 0 && yg[j] > qy) --j;
    j = max(0, min(j, ny - 2));
    const double x1 = xg[i], x2 = xg[i + 1];
    const double y1 = yg[j], y2 = yg[j + 1];
    const double tx = (qx - x1) / (x2 - x1);
    const double ty = (qy - y1) / (y2 - y1);
    k[0] = (size_t)j * nx + i;
    k[1] = (size_t)j * nx + i + 1;
    k[2] = (size_t)(j + 1) * nx + i;
    k[3] = (size_t)(j + 1) * nx + i + 1;
    w[0] = (1 - tx) * (1 - ty);
    w[1] = (tx) * (1 - ty);
    w[2] = (1 - tx) * (ty);
    w[3] = (tx) * (ty);
    return true;
}

__device__ inline double interp2d_pt(const double* xg, int nx, const double* yg, int ny,
                                     const double* z, double qx, double qy) {
    size_t k[4];
    double w[4];
    if (!interp2d_weights(xg, nx, yg, ny, qx, qy, k, w))
        return __longlong_as_double(0x7ff8000000000000ll);
    return w[0] * z[k[0]] + w[1] * z[k[1]] + w[2] * z[k[2]] + w[3] * z[k[3]];
}

// Bilinear spreading of adjoint sources normalised by the cell area
// (src/eikonal_solver.cpp:354-375).  Called by one lane, receivers in order.
// With zero_out, writes 0 to the same cells instead (scratch cleanup).
__device__ inline void spread_delta(const Grid& g, const Events& ev, int r0, int nr,
                                    const double* sadj, double* delta, bool zero_out) {
    const int nx = g.nx, ny = g.ny;
    for (int ir = 0; ir < nr; ir++) {
        const int st = ev.rec_idx[r0 + ir];
        const double xrec = ev.stlo[st] * DEG2RAD;
        const double yrec = ev.stla[st] * DEG2RAD;
        const double fx = floor((xrec - g.xx[0]) / g.dx);
        const double fy = floor((yrec - g.yy[0]) / g.dy);
        int idx0 = (int)fmax(-4.0, fmin((double)nx + 4.0, fx));
        int idy0 = (int)fmax(-4.0, fmin((double)ny + 4.0, fy));
        idx0 = max(0, min(idx0, nx - 2));
        idy0 = max(0, min(idy0, ny - 2));
        const size_t k00 = (size_t)idy0 * nx + idx0;
        if (zero_out) {
            delta[k00] = 0.0;
            delta[k00 + nx] = 0.0;
            delta[k00 + 1] = 0.0;
            delta[k00 + nx + 1] = 0.0;
            continue;
        }
        const double r1 = fmin(1.0, (xrec - g.xx[idx0]) / g.dx);
        const double r2 = fmin(1.0, (yrec - g.yy[idy0]) / g.dy);
        const double area = g.dx * R_EARTH * ev.cos_stla[st] * g.dy * R_EARTH;
        const double w = sadj[ir] / area;
        delta[k00] += w * (1 - r1) * (1 - r2);
        delta[k00 + nx] += w * (1 - r1) * r2;
        delta[k00 + 1] += w * r1 * (1 - r2);
        delta[k00 + nx + 1] += w * r1 * r2;
    }
}

// Face fluxes of src/eikonal_solver.cpp:404-441 for one cell.
// A(ix,iy) = a1 at ix in [1,nx-1] (interior iy); B(ix,iy) = b1 at iy in [1,ny-1].
__device__ __forceinline__ double face_a1(const double* T, const double* a, const double* c,
                                          int nx, int ix, int iy, double dx, double dy) {
    const size_t k = (size_t)iy * nx + ix;
    return -(T[k] - T[k - 1]) / dx * (a[k] + a[k - 1]) / 2.0
         + (T[k + nx] - T[k - nx] + T[k - 1 + nx] - T[k - 1 - nx]) / (4.0 * dy)
           * (c[k] + c[k - 1]) / 2.0;
}
__device__ __forceinline__ double face_b1(const double* T, const double* b, const double* c,
                                          int nx, int ix, int iy, double dx, double dy) {
    const size_t k = (size_t)iy * nx + ix;
    return -(T[k] - T[k - nx]) / dy * (b[k] + b[k - nx]) / 2.0
         + (T[k + 1] - T[k - 1] + T[k + 1 - nx] - T[k - 1 - nx]) / (4.0 * dx)
           * (c[k] + c[k - nx]) / 2.0;
}

// Same, isotropic metric (a per row, c = +0.0 everywhere, b constant).
__device__ __forceinline__ double face_a1_iso(const double* T, double arow, int nx, int ix,
                                              int iy, double dx, double dy) {
    const size_t k = (size_t)iy * nx + ix;
    const double c0 = 0.0;
    return -(T[k] - T[k - 1]) / dx * (arow + arow) / 2.0
         + (T[k + nx] - T[k - nx] + T[k - 1 + nx] - T[k - 1 - nx]) / (4.0 * dy) * (c0 + c0) / 2.0;
}
__device__ __forceinline__ double face_b1_iso(const double* T, double brow_here,
                                              double brow_below, int nx, int ix, int iy,
                                              double dx, double dy) {
    const size_t k = (size_t)iy * nx + ix;
    const double c0 = 0.0;
    return -(T[k] - T[k - nx]) / dy * (brow_here + brow_below) / 2.0
         + (T[k + 1] - T[k - 1] + T[k + 1 - nx] - T[k - 1 - nx]) / (4.0 * dx) * (c0 + c0) / 2.0;
}

// Index range zeroed by eikonal::mask_uniform_grid (src/eikonal_solver.cpp:514-536),
// computed on the degree grid.
struct MaskBox {
    int ix_lo, ix_hi, iy_lo, iy_hi;
};
__device__ inline MaskBox mask_box(const Grid& g, double x0, double y0) {
    const int nx = g.nx, ny = g.ny;
    const double dx = g.xx_deg[1] - g.xx_deg[0];
    const double dy = g.yy_deg[1] - g.yy_deg[0];
    auto clampi = [](double v) { return (int)fmax(-1e9, fmin(1e9, v)); };
    MaskBox m;
    m.ix_lo = max(0, clampi(floor((x0 - 1.5 * dx - g.xx_deg[0]) / dx)) + 1);
    m.ix_hi = min(nx - 1, clampi(ceil((x0 + 1.5 * dx - g.xx_deg[0]) / dx)) - 1);
    m.iy_lo = max(0, clampi(floor((y0 - 1.5 * dy - g.yy_deg[0]) / dy)) + 1);
    m.iy_hi = min(ny - 1, clampi(ceil((y0 + 1.5 * dy - g.yy_deg[0]) / dy)) - 1);
    return m;
}

// Per-lane walk over the cells of an nx-wide plane of n cells in warp
// stride: f(k, ix, iy) at k = lane, lane + 32, ...  The column and row are
// carried along instead of divided out of k (a 64-bit division per cell).
template <class F>
__device__ __forceinline__ void for_cells(int nx, size_t n, int lane, F&& f) {
    int ix = lane % nx, iy = lane / nx;
    for (size_t k = lane; k < n; k += 32) {
        f(k, ix, iy);
        ix += 32;
        while (ix >= nx) {
            ix -= nx;
            iy++;
        }
    }
}

__device__ __forceinline__ unsigned int warp_next_event(unsigned int* queue) {
    unsigned int e = 0;
    if ((threadIdx.x & 31) == 0) e = atomicAdd(queue, 1u);
    return __shfl_sync(FULL_MASK, e, 0);
}

}  // namespace sa
