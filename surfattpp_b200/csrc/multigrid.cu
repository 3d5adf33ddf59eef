// Multigrid kernel smoothing (the reference's smooth_method 1):
// PostProc::InvGrid::init / fwd2inv / inv2fwd (src/postproc.cpp:160-386)
// and PostProc::smooth (:465-480).
//
// nset staggered coarse grids of (n_inv + 2) nodes per axis; the field is
// projected onto them (fwd2inv) and interpolated back (inv2fwd), averaged
// over the sets.  Kept as the reference computes it:
//   * fwd2inv adds each fine node to ONE coarse node, the corner n = 7
//     (idx+1, idy, idz+1) with weight wx (1 - wy) wz: its accumulation sits
//     after the corner loop;
//   * the coarse index uses the inner counts n_inv_J, n_inv_K as strides
//     (I2V_INV_GRIDS, include/postproc.h:53-55), so distinct corners share
//     entries.
// Exactness: the reference sums fwd2inv's contributions in (set, ix, iy, iz)
// order.  At set-up every contribution's coarse entry is computed and a
// stable sort groups them by entry with that order kept; a smoothing call
// then sums each entry's segment in order (one thread per coarse entry) and
// interpolates per fine node over the sets in order, all with -fmad=false,
// so the result equals a CPU evaluation bit for bit.
#include <cub/cub.cuh>

#include <vector>

#include "launch.h"
#include "surfatt_gpu.h"

namespace sa {
namespace {

// per-axis tables of one set: the coarse cell of each fine node and its weight
struct Axis {
    const int* cell;      // [nset][n]
    const double* w;      // [nset][n]
};

struct MG {
    int nx, ny, nz, nI, nJ, nK, nset;
    Axis ax, ay, az;
    __device__ int idx(int A, int B, int C, int D) const {
        return A * nK * nJ * nset + B * nK * nset + C * nset + D;
    }
};

// entry of contribution e = ((ig * nx + i) * ny + j) * nz + k (n = 7 corner)
__global__ void mg_entry_kernel(MG g, size_t ncontrib, unsigned* key, unsigned* val) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ncontrib;
         e += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(e % g.nz);
        const int j = (int)((e / g.nz) % g.ny);
        const int i = (int)((e / ((size_t)g.nz * g.ny)) % g.nx);
        const int ig = (int)(e / ((size_t)g.nz * g.ny * g.nx));
        const int ix = g.ax.cell[(size_t)ig * g.nx + i];
        const int iy = g.ay.cell[(size_t)ig * g.ny + j];
        const int iz = g.az.cell[(size_t)ig * g.nz + k];
        key[e] = (unsigned)g.idx(ix + 1, iy, iz + 1, ig);
        val[e] = (unsigned)e;
    }
}

// fwd2inv: per coarse entry, its contributions in the reference's order
__global__ void mg_project_kernel(MG g, int ngrid, const int* __restrict__ seg,
                                  const unsigned* __restrict__ order,
                                  const double* __restrict__ buf, double* arr) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= ngrid) return;
    double tmp = 0.0, weight = 0.0;
    for (int p = seg[m]; p < seg[m + 1]; p++) {
        const size_t e = order[p];
        const int k = (int)(e % g.nz);
        const int j = (int)((e / g.nz) % g.ny);
        const int i = (int)((e / ((size_t)g.nz * g.ny)) % g.nx);
        const int ig = (int)(e / ((size_t)g.nz * g.ny * g.nx));
        const double wx = g.ax.w[(size_t)ig * g.nx + i];
        const double wy = g.ay.w[(size_t)ig * g.ny + j];
        const double wz = g.az.w[(size_t)ig * g.nz + k];
        const double wt = wx * (1.0 - wy) * wz;
        weight += wt;
        tmp += wt * buf[((size_t)i * g.ny + j) * g.nz + k];
    }
    arr[m] = weight > 0.0 ? tmp / weight : 0.0;
}

// inv2fwd: per fine node, the 8 corners of each set, sets in order
__global__ void mg_interp_kernel(MG g, const double* __restrict__ arr, double* out) {
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % g.nz);
        const int j = (int)((t / g.nz) % g.ny);
        const int i = (int)(t / ((size_t)g.nz * g.ny));
        double acc = 0.0;
        for (int ig = 0; ig < g.nset; ig++) {
            const int ix = g.ax.cell[(size_t)ig * g.nx + i];
            const int iy = g.ay.cell[(size_t)ig * g.ny + j];
            const int iz = g.az.cell[(size_t)ig * g.nz + k];
            const double wx = g.ax.w[(size_t)ig * g.nx + i];
            const double wy = g.ay.w[(size_t)ig * g.ny + j];
            const double wz = g.az.w[(size_t)ig * g.nz + k];
            const double w[8] = {(1.0 - wx) * (1.0 - wy) * (1.0 - wz), (1.0 - wx) * wy * (1.0 - wz),
                                 wx * wy * (1.0 - wz),                 wx * (1.0 - wy) * (1.0 - wz),
                                 (1.0 - wx) * (1.0 - wy) * wz,         (1.0 - wx) * wy * wz,
                                 wx * wy * wz,                         wx * (1.0 - wy) * wz};
            const int m[8] = {g.idx(ix, iy, iz, ig),         g.idx(ix, iy + 1, iz, ig),
                              g.idx(ix + 1, iy + 1, iz, ig), g.idx(ix + 1, iy, iz, ig),
                              g.idx(ix, iy, iz + 1, ig),     g.idx(ix, iy + 1, iz + 1, ig),
                              g.idx(ix + 1, iy + 1, iz + 1, ig), g.idx(ix + 1, iy, iz + 1, ig)};
            double val = 0.0;
            for (int c = 0; c < 8; c++) val += w[c] * arr[m[c]];
            acc += val;
        }
        out[t] = acc / (double)g.nset;
    }
}

unsigned grid_blocks(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

// include/utils.h:39-60
int locate_bissection(const double* v, int n, double x) {
    int low = 0, high = n - 1;
    if (x < v[0] || x > v[n - 1]) return -1;
    while (high - low > 1) {
        const int mid = (high + low) / 2;
        if (v[mid] > x) high = mid;
        else low = mid;
    }
    if (x == v[0]) return 0;
    if (x == v[n - 1]) return n - 2;
    return low;
}

// InvGrid::init for one axis (src/postproc.cpp:160-207): coarse nodes of
// every set, then each fine node's cell and weight in each set; false when a
// fine node falls outside (the reference aborts)
bool axis_tables(const double* g, int n, int ninner, int nset, std::vector<int>& cell,
                 std::vector<double>& w) {
    const int m = ninner + 2;
    const double g0 = g[0], g1 = g[n - 1];
    const double d = (g1 - g0) / ninner;
    const double add = d / nset;
    std::vector<double> c(m);
    cell.assign((size_t)nset * n, 0);
    w.assign((size_t)nset * n, 0.0);
    for (int is = 0; is < nset; ++is) {
        c[0] = g0 - add;
        c[m - 1] = g1 + add;
        for (int j = 1; j < m - 1; ++j) c[j] = (g0 + (j - 1) * d) + is * add;
        for (int i = 0; i < n; ++i) {
            const int id = locate_bissection(c.data(), m, g[i]);
            if (id < 0) return false;
            cell[(size_t)is * n + i] = id;
            w[(size_t)is * n + i] = (g[i] - c[id]) / (c[id + 1] - c[id]);
        }
    }
    return true;
}

}  // namespace
}  // namespace sa

using namespace sa;

struct sa_multigrid {
    int device = 0;
    MG g{};
    int ngrid = 0;
    int *cell = nullptr, *seg = nullptr;
    double *w = nullptr, *arr = nullptr;
    unsigned* order = nullptr;
    ~sa_multigrid() {
        cudaFree(cell);
        cudaFree(seg);
        cudaFree(w);
        cudaFree(arr);
        cudaFree(order);
    }
};

extern "C" int sa_multigrid_create(int device, int nx, int ny, int nz, const double* x,
                                   const double* y, const double* z, const int* n_inv, int nset,
                                   sa_multigrid** out) {
    if (!out || !x || !y || !z || !n_inv || nx < 2 || ny < 2 || nz < 2 || nset < 1 ||
        n_inv[0] < 1 || n_inv[1] < 1 || n_inv[2] < 1)
        return SA_ERR_ARG;
    *out = nullptr;
    const size_t ngrid = (size_t)(n_inv[0] + 2) * (n_inv[1] + 2) * (n_inv[2] + 2) * nset;
    const size_t ncontrib = (size_t)nset * nx * ny * nz;
    if (ngrid >= (1u << 31) || ncontrib >= (1u << 31)) return SA_ERR_ARG;
    std::vector<int> cx, cy, cz;
    std::vector<double> wx, wy, wz;
    if (!axis_tables(x, nx, n_inv[0], nset, cx, wx) || !axis_tables(y, ny, n_inv[1], nset, cy, wy) ||
        !axis_tables(z, nz, n_inv[2], nset, cz, wz))
        return SA_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return SA_ERR_CUDA;
    sa_multigrid* M = new sa_multigrid();
    M->device = device;
    M->ngrid = (int)ngrid;
    const size_t na = (size_t)nset * (nx + ny + nz);
    cudaError_t e = cudaMalloc(&M->cell, na * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&M->w, na * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&M->arr, ngrid * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&M->seg, (ngrid + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&M->order, ncontrib * sizeof(unsigned));
    std::vector<int> call(cx);
    call.insert(call.end(), cy.begin(), cy.end());
    call.insert(call.end(), cz.begin(), cz.end());
    std::vector<double> wall(wx);
    wall.insert(wall.end(), wy.begin(), wy.end());
    wall.insert(wall.end(), wz.begin(), wz.end());
    if (e == cudaSuccess) e = cudaMemcpy(M->cell, call.data(), na * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(M->w, wall.data(), na * sizeof(double), cudaMemcpyHostToDevice);
    MG& g = M->g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.nI = n_inv[0];
    g.nJ = n_inv[1];
    g.nK = n_inv[2];
    g.nset = nset;
    g.ax = {M->cell, M->w};
    g.ay = {M->cell + (size_t)nset * nx, M->w + (size_t)nset * nx};
    g.az = {M->cell + (size_t)nset * (nx + ny), M->w + (size_t)nset * (nx + ny)};
    // group the contributions by coarse entry, keeping their order (stable sort)
    unsigned *key = nullptr, *key2 = nullptr, *val = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    if (e == cudaSuccess) e = cudaMalloc(&key, ncontrib * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&key2, ncontrib * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&val, ncontrib * sizeof(unsigned));
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key2, val, M->order,
                                            (int)ncontrib);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 1));
    if (e == cudaSuccess) {
        mg_entry_kernel<<<grid_blocks(ncontrib), 256>>>(g, ncontrib, key, val);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key2, val, M->order,
                                            (int)ncontrib);
    std::vector<unsigned> keys(ncontrib);
    if (e == cudaSuccess)
        e = cudaMemcpy(keys.data(), key2, ncontrib * sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) {   // segment offsets of the sorted keys
        std::vector<int> seg(ngrid + 1, 0);
        for (size_t p = 0; p < ncontrib; p++) seg[keys[p] + 1]++;
        for (size_t m = 0; m < ngrid; m++) seg[m + 1] += seg[m];
        e = cudaMemcpy(M->seg, seg.data(), (ngrid + 1) * sizeof(int), cudaMemcpyHostToDevice);
    }
    cudaFree(key);
    cudaFree(key2);
    cudaFree(val);
    cudaFree(tmp);
    if (e != cudaSuccess) {
        delete M;
        return e == cudaErrorMemoryAllocation ? SA_ERR_NOMEM : SA_ERR_CUDA;
    }
    *out = M;
    return SA_OK;
}

extern "C" void sa_multigrid_destroy(sa_multigrid* M) {
    if (!M) return;
    cudaSetDevice(M->device);
    delete M;
}

extern "C" int sa_multigrid_smooth(sa_multigrid* M, const double* field, double* out,
                                   void* stream) {
    if (!M || !field || !out || field == out) return SA_ERR_ARG;
    if (cudaSetDevice(M->device) != cudaSuccess) return SA_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    mg_project_kernel<<<(M->ngrid + 127) / 128, 128, 0, st>>>(M->g, M->ngrid, M->seg, M->order,
                                                               field, M->arr);
    const size_t n = (size_t)M->g.nx * M->g.ny * M->g.nz;
    mg_interp_kernel<<<grid_blocks(n), 256, 0, st>>>(M->g, M->arr, out);
    return cudaGetLastError() == cudaSuccess ? SA_OK : SA_ERR_CUDA;
}
