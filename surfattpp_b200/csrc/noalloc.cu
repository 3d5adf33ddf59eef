// Allocation-free forward travel-time solve.
//
// Some callers cannot allocate device memory at the time they call us: code
// that runs inside another framework's memory pool or allocator callback,
// real-time or embedded hosts that forbid cudaMalloc after start-up, and
// hosts whose device memory is fully reserved up front.  For them,
// sa_eik_fwd_field_noalloc solves one eikonal::FSM_UW_PS_lonlat_2d problem
// with every intermediate (grid tables, metric and geometry planes, the grid
// spacing, the warp's sweep scratch and the work counter) in the file-scope
// device array below.  The caller passes device inputs and outputs only, and
// the call neither allocates nor synchronises: all of it is enqueued on the
// caller's stream.
//
// Limits and sharing:
//   * the array is NOALLOC_BYTES (64 MiB) and every GPU that loads the
//     library holds it until the process exits;
//   * a grid needs 145 bytes per cell (56 in the metric and geometry planes,
//     89 in the sweep scratch), so nx*ny is limited to about 462,000 cells
//     (680 x 680 fits, 690 x 690 does not); larger grids are rejected with
//     SA_ERR_ARG and a message on stderr;
//   * every call shares the array and it keeps the last call's contents, so
//     calls that overlap on the GPU (different streams or host threads at the
//     same time) race: serialise them;
//   * the first call in each context looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture (and again after a device reset).
//
// Compiled with -fmad=false: the grid, metric and geometry planes round as
// the plan path's host arithmetic does, with correctly rounded sin and cos.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "batch.cuh"
#include "crmath.cuh"
#include "launch.h"
#include "surfatt_gpu.h"

namespace sa {
namespace {

constexpr size_t NOALLOC_BYTES = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Offsets of the pieces inside g_noalloc_scratch for an nx x ny grid.
// The forward solve (MODE_FWD) reads no adjoint metric planes, so none are
// reserved.
struct NoAllocLayout {
    size_t xx, yy, cosy, siny, dxdy, mt, G, Gx, Gy;
    size_t ev_src, ev_iper, ev_evlo, ev_evla, ev_ptr, queue, slot, total;
    size_t slot_bytes;
};

NoAllocLayout noalloc_layout(int nx, int ny) {
    NoAllocLayout L{};
    const size_t n = (size_t)nx * ny;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o += align_up(bytes, 256);
        return at;
    };
    L.xx = take(nx * sizeof(double));
    L.yy = take(ny * sizeof(double));
    L.cosy = take(ny * sizeof(double));
    L.siny = take(ny * sizeof(double));
    L.dxdy = take(2 * sizeof(double));
    L.mt = take(4 * n * sizeof(double));
    L.G = take(n * sizeof(double));
    L.Gx = take(n * sizeof(double));
    L.Gy = take(n * sizeof(double));
    L.ev_src = take(sizeof(int));
    L.ev_iper = take(sizeof(int));
    L.ev_evlo = take(sizeof(double));
    L.ev_evla = take(sizeof(double));
    L.ev_ptr = take(2 * sizeof(int));
    L.queue = take(sizeof(unsigned int));
    L.slot_bytes = slot_layout<double>(nx, ny, 1).total;
    L.slot = take(L.slot_bytes);
    L.total = o;
    return L;
}

// Builds everything the batch kernel reads besides the caller's arrays:
// radian grids and their spacing dx = xx(1) - xx(0), dy = yy(1) - yy(0), row
// trigonometry, the forward metric planes from spha, sphb, sphc
// (src/eikonal_solver.cpp:55-65), the great-circle geometry of the one
// source (:96-116; correctly rounded sin / cos, CUDA's acos) and a one-event
// list; zeroes the work counter.
__global__ void noalloc_prep_kernel(int nx, int ny, const double* __restrict__ xx_deg,
                                    const double* __restrict__ yy_deg,
                                    const double* __restrict__ spha,
                                    const double* __restrict__ sphb,
                                    const double* __restrict__ sphc, double x0_deg, double y0_deg,
                                    unsigned char* base, NoAllocLayout L) {
    double* xx = reinterpret_cast<double*>(base + L.xx);
    double* yy = reinterpret_cast<double*>(base + L.yy);
    double* cosy = reinterpret_cast<double*>(base + L.cosy);
    double* siny = reinterpret_cast<double*>(base + L.siny);
    double* mt = reinterpret_cast<double*>(base + L.mt);
    double* G = reinterpret_cast<double*>(base + L.G);
    double* Gx = reinterpret_cast<double*>(base + L.Gx);
    double* Gy = reinterpret_cast<double*>(base + L.Gy);
    const size_t n = (size_t)nx * ny;
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t nth = (size_t)gridDim.x * blockDim.x;
    const double x0 = x0_deg * DEG2RAD, y0 = y0_deg * DEG2RAD;
    const double sy0 = cr::sin(y0), cy0 = cr::cos(y0);
    for (size_t i = tid; i < (size_t)nx; i += nth) xx[i] = xx_deg[i] * DEG2RAD;
    for (size_t i = tid; i < (size_t)ny; i += nth) {
        const double y = yy_deg[i] * DEG2RAD;
        yy[i] = y;
        cosy[i] = cr::cos(y);
        siny[i] = cr::sin(y);
    }
    for (size_t k = tid; k < n; k += nth) {
        const int iy = (int)(k / nx), ix = (int)(k % nx);
        const double y = yy_deg[iy] * DEG2RAD;
        const double cos_y = cr::cos(y), sin_y = cr::sin(y);
        const double cos2_y = cos_y * cos_y;
        const double R2 = R_EARTH * R_EARTH;
        mt[4 * k + 0] = spha[k] / (R2 * cos2_y);
        mt[4 * k + 1] = sphb[k] / R2;
        mt[4 * k + 2] = sphc[k] / (R_EARTH * R_EARTH * cos_y);
        mt[4 * k + 3] = 0.0;
        const double dlon = xx_deg[ix] * DEG2RAD - x0;
        const double cdl = cr::cos(dlon), sdl = cr::sin(dlon);
        const double tmp = sin_y * sy0 + cos_y * cy0 * cdl;
        const double tmp_c = fmax(-1.0, fmin(1.0, tmp));
        G[k] = acos(tmp_c) * R_EARTH;
        const double sin_d = sqrt(fmax(0.0, 1.0 - tmp_c * tmp_c));
        if (sin_d < 1e-14) {
            Gx[k] = 0.0;
            Gy[k] = 0.0;
        } else {
            Gx[k] = cos_y * cy0 * sdl / sin_d * R_EARTH;
            Gy[k] = -(cos_y * sy0 - sin_y * cy0 * cdl) / sin_d * R_EARTH;
        }
    }
    if (tid == 0) {
        double* dxdy = reinterpret_cast<double*>(base + L.dxdy);
        dxdy[0] = xx_deg[1] * DEG2RAD - xx_deg[0] * DEG2RAD;
        dxdy[1] = yy_deg[1] * DEG2RAD - yy_deg[0] * DEG2RAD;
        *reinterpret_cast<int*>(base + L.ev_src) = 0;
        *reinterpret_cast<int*>(base + L.ev_iper) = 0;
        *reinterpret_cast<double*>(base + L.ev_evlo) = x0_deg;
        *reinterpret_cast<double*>(base + L.ev_evla) = y0_deg;
        reinterpret_cast<int*>(base + L.ev_ptr)[0] = 0;
        reinterpret_cast<int*>(base + L.ev_ptr)[1] = 0;
        *reinterpret_cast<unsigned int*>(base + L.queue) = 0u;
    }
}

std::mutex g_sym_mutex;
unsigned char* g_sym_addr[64] = {};
void* g_sym_ctx[64] = {};

// The driver's cuCtxGetCurrent, through the runtime (no link to libcuda).
using CtxGetCurrentFn = int (*)(void**);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn f = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<CtxGetCurrentFn>(nullptr);
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    return f;
}

// Device address of g_noalloc_scratch in the current context, looked up on
// the first call in each context (a device reset makes a new context and a
// new module instance, so an address cached by device ordinal alone could
// be stale).
unsigned char* scratch_address(int device, cudaError_t* err) {
    *err = cudaSuccess;
    if (device < 0 || device >= 64) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    void* ctx = nullptr;
    if (CtxGetCurrentFn f = ctx_get_current()) f(&ctx);
    std::lock_guard<std::mutex> lock(g_sym_mutex);
    if (!g_sym_addr[device] || !ctx || ctx != g_sym_ctx[device]) {
        void* p = nullptr;
        *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (*err != cudaSuccess) return nullptr;
        g_sym_addr[device] = static_cast<unsigned char*>(p);
        g_sym_ctx[device] = ctx;
    }
    return g_sym_addr[device];
}

}  // namespace
}  // namespace sa

using namespace sa;

extern "C" int sa_eik_fwd_field_noalloc(int nx, int ny, const double* xx_deg,
                                        const double* yy_deg, const double* spha,
                                        const double* sphb, const double* sphc,
                                        const double* fun, double x0_deg, double y0_deg,
                                        double* T_out, int* niter, int* status, void* stream) {
    if (nx < 3 || ny < 3) {
        std::fprintf(stderr, "sa_eik_fwd_field_noalloc: grid must be at least 3x3\n");
        return SA_ERR_ARG;
    }
    if (!xx_deg || !yy_deg || !spha || !sphb || !sphc || !fun || !T_out) {
        std::fprintf(stderr, "sa_eik_fwd_field_noalloc: null input or output pointer\n");
        return SA_ERR_ARG;
    }
    const NoAllocLayout L = noalloc_layout(nx, ny);
    if (L.total > NOALLOC_BYTES) {
        std::fprintf(stderr,
                     "sa_eik_fwd_field_noalloc: %d x %d grid needs %zu bytes of scratch, more "
                     "than the fixed %zu-byte device array; use sa_eik_fwd_field\n",
                     nx, ny, L.total, NOALLOC_BYTES);
        return SA_ERR_ARG;
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return SA_ERR_CUDA;
    cudaError_t err;
    unsigned char* base = scratch_address(device, &err);
    if (!base) {
        std::fprintf(stderr, "sa_eik_fwd_field_noalloc: cudaGetSymbolAddress failed: %s\n",
                     cudaGetErrorString(err));
        return SA_ERR_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)nx * ny;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((n + threads - 1) / threads, 148 * 8);
    noalloc_prep_kernel<<<blocks, threads, 0, st>>>(nx, ny, xx_deg, yy_deg, spha, sphb, sphc,
                                                    x0_deg, y0_deg, base, L);
    if (cudaGetLastError() != cudaSuccess) return SA_ERR_CUDA;
    BatchDesc d{};
    d.g.nx = nx;
    d.g.ny = ny;
    d.g.xx_deg = xx_deg;
    d.g.yy_deg = yy_deg;
    d.g.xx = reinterpret_cast<const double*>(base + L.xx);
    d.g.yy = reinterpret_cast<const double*>(base + L.yy);
    d.g.cosy = reinterpret_cast<const double*>(base + L.cosy);
    d.g.siny = reinterpret_cast<const double*>(base + L.siny);
    // dx, dy: formed on the device by the prep kernel (dxdy plane)
    d.g.dx = 0.0;
    d.g.dy = 0.0;
    d.nper = 1;
    d.iso = 0;
    d.fun64 = fun;
    d.mt64 = reinterpret_cast<const double*>(base + L.mt);
    d.b_p64 = nullptr;   // adjoint planes: not read by MODE_FWD
    d.a_a64 = nullptr;
    d.c_a64 = nullptr;
    d.G64 = reinterpret_cast<const double*>(base + L.G);
    d.Gx64 = reinterpret_cast<const double*>(base + L.Gx);
    d.Gy64 = reinterpret_cast<const double*>(base + L.Gy);
    d.ev.ne = 1;
    d.ev.src = reinterpret_cast<const int*>(base + L.ev_src);
    d.ev.iper = reinterpret_cast<const int*>(base + L.ev_iper);
    d.ev.evlo = reinterpret_cast<const double*>(base + L.ev_evlo);
    d.ev.evla = reinterpret_cast<const double*>(base + L.ev_evla);
    d.ev.rec_ptr = reinterpret_cast<const int*>(base + L.ev_ptr);
    d.out.T_out = T_out;
    d.out.fwd_iters = niter;
    d.out.status = status;
    d.sc.nslots = 1;
    d.sc.slot_bytes = L.slot_bytes;
    d.sc.base = base + L.slot;
    d.sc.queue = reinterpret_cast<unsigned int*>(base + L.queue);
    d.maxr = 1;
    d.mode = MODE_FWD;
    if (launch_batch64_dev_spacing(d, reinterpret_cast<const double*>(base + L.dxdy), st) !=
        cudaSuccess)
        return SA_ERR_CUDA;
    return SA_OK;
}
