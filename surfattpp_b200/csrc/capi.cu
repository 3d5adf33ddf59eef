// C ABI of libsurfatt_gpu.so (declared in include/surfatt_gpu.h).
//
// Host-side work here is bookkeeping only: argument checks, unique-source
// grouping of the event list, C-library trigonometric row/column tables (so
// the device geometry matches a CPU evaluation bit for bit), uploads, and
// launching / graph-replaying the device pipeline.  No numerical path of the
// engine runs on the host.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <array>
#include <map>
#include <cstring>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "launch.h"
#include "surfatt_gpu.h"

using namespace sa;

struct sa_ctx;

namespace {

int fail(sa_ctx* ctx, int code, const std::string& msg);

#define SA_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? SA_ERR_NOMEM : SA_ERR_CUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));             \
    } while (0)

template <class T>
struct DArr {
    T* p = nullptr;
    size_t n = 0;
    ~DArr() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        if (count <= n && p) return cudaSuccess;
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
    cudaError_t upload(const T* h, size_t count, cudaStream_t st) {
        cudaError_t e = alloc(count);
        if (e != cudaSuccess) return e;
        if (count) e = cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st);
        return e;
    }
};

// Device copies of the per-layer flattening constants and of the period list,
// rebuilt when the depth grid or the periods change.
struct LayerConstCache {
    int nz = -1;
    std::vector<double> z;
    DArr<unsigned char> dev;
};
struct PeriodCache {
    std::vector<double> p;
    DArr<double> dev;
};
}  // namespace

struct sa_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    LayerConstCache lc;
    PeriodCache pc;
    DArr<double> red;   // reduction scratch of the optimizer entry points
    // launch configuration chosen by sa_plan_autotune per grid size:
    // (nx, ny, precision) -> (variant, active slots; 0 = all)
    std::map<std::array<int, 3>, std::array<int, 2>> tune;
};

namespace {
int fail(sa_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

struct GraphKey {
    const void* ptr[17];
    int calc_adj;
    bool operator==(const GraphKey& o) const {
        return calc_adj == o.calc_adj && std::memcmp(ptr, o.ptr, sizeof(ptr)) == 0;
    }
};

}  // namespace

struct sa_plan {
    sa_ctx* ctx = nullptr;
    int prec = SA_FP64;
    int nx = 0, ny = 0, nper = 0, ne = 0, nsta = 0, nsrc = 0, npair = 0;
    double dx = 0, dy = 0;
    DArr<double> xx_deg, yy_deg, xx, yy, cosy, siny, a_f_row64, a_a_row64;
    DArr<float> a_f_row32;
    DArr<double> evlo, evla, stlo, stla, cos_stla;
    DArr<int> iper, src, rec_ptr, rec_idx;
    DArr<double> G64, Gx64, Gy64;
    DArr<float> G32, Gx32, Gy32;
    DArr<double> fun64, inv3, mt64, b_p64, a_a64, c_a64;
    DArr<float> fun32, mt32;
    int maxr = 0;
    DArr<double> chi_ev;
    DArr<int> status_tmp, worst;
    DArr<unsigned char> scratch;
    DArr<unsigned int> queue;
    // cost-ordered work queue: events sorted by the previous evaluation's
    // sweep counts, longest first, so the persistent kernel's tail is short
    DArr<int> fit, ait, order, ord_idx;
    DArr<unsigned int> key_a, key_b;
    DArr<unsigned char> sort_tmp;
    size_t sort_bytes = 0;
    int nslots = 0;
    size_t slot_bytes = 0;
    int variant = 0;      // FP32 batch-kernel launch variant (batch.cuh)
    int active = 0;       // event slots in use (0 = all nslots)
    // deterministic accumulation (sa_plan_set_deterministic): events run in
    // chunks of `chunk`; each writes its contribution plane to `contrib`,
    // then the chunk is summed into adj_s in event order, per period
    // (per_ptr[(c * (nper + 1)) + ip] .. into per_ev)
    bool determ = false;
    int chunk = 0;
    DArr<double> contrib;
    DArr<int> iota, per_ptr, per_ev;
    double* dbg_T = nullptr;
    double* dbg_Ta = nullptr;
    double* kden_out = nullptr;   // is_kden accumulation target (sa_plan_kden_output)
    int discrete = 0;             // sa_plan_set_adjoint: 1 = exact discrete adjoint
    bool use_graph = true;
    bool have_graph = false;
    GraphKey key{};
    cudaGraphExec_t gexec = nullptr;
    bool timing = false;                    // events around the batch launch (no graph)
    cudaEvent_t tk0 = nullptr, tk1 = nullptr;
    ~sa_plan() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (tk0) cudaEventDestroy(tk0);
        if (tk1) cudaEventDestroy(tk1);
    }
};

extern "C" int sa_version(void) { return 100; }

extern "C" int sa_ctx_create(int device, sa_ctx** out) {
    if (!out) return SA_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return SA_ERR_CUDA;
    if (device < 0 || device >= ndev) return SA_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return SA_ERR_CUDA;
    sa_ctx* c = new sa_ctx();
    c->device = device;
    if (cudaStreamCreate(&c->stream) != cudaSuccess) {   // blocking: orders with the legacy stream
        delete c;
        return SA_ERR_CUDA;
    }
    *out = c;
    return SA_OK;
}

extern "C" void sa_ctx_destroy(sa_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

extern "C" const char* sa_ctx_error(const sa_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

// src/eikonal_solver.cpp:514-536
extern "C" int sa_mask_uniform_grid(int nx, int ny, const double* xx, const double* yy,
                                    double* table, double x0, double y0) {
    if (nx < 2 || ny < 2) return SA_OK;
    if (!xx || !yy || !table) return SA_ERR_ARG;
    const double dx = xx[1] - xx[0];
    const double dy = yy[1] - yy[0];
    const int ix_lo = std::max(0, static_cast<int>(std::floor((x0 - 1.5 * dx - xx[0]) / dx)) + 1);
    const int ix_hi = std::min(nx - 1, static_cast<int>(std::ceil((x0 + 1.5 * dx - xx[0]) / dx)) - 1);
    const int iy_lo = std::max(0, static_cast<int>(std::floor((y0 - 1.5 * dy - yy[0]) / dy)) + 1);
    const int iy_hi = std::min(ny - 1, static_cast<int>(std::ceil((y0 + 1.5 * dy - yy[0]) / dy)) - 1);
    if (ix_lo <= ix_hi && iy_lo <= iy_hi)
        for (int iy = iy_lo; iy <= iy_hi; iy++)
            for (int ix = ix_lo; ix <= ix_hi; ix++) table[ix + (size_t)nx * iy] = 0.0;
    return SA_OK;
}

namespace {

// Grid tables and (optionally) events/geometry of a plan.
int plan_grid(sa_plan* P, const double* xx_deg, const double* yy_deg) {
    sa_ctx* ctx = P->ctx;
    const int nx = P->nx, ny = P->ny;
    cudaStream_t st = ctx->stream;
    std::vector<double> xr(nx), yr(ny), cy(ny), sy(ny), af(ny), aa(ny);
    std::vector<float> af32(ny);
    const double R2 = R_EARTH * R_EARTH;
    for (int i = 0; i < nx; i++) xr[i] = xx_deg[i] * DEG2RAD;
    for (int i = 0; i < ny; i++) {
        yr[i] = yy_deg[i] * DEG2RAD;
        cy[i] = std::cos(yr[i]);
        sy[i] = std::sin(yr[i]);
        const double cos2_y = cy[i] * cy[i];
        af[i] = 1.0 / (R2 * cos2_y);            // src/eikonal_solver.cpp:61, spha = 1
        aa[i] = 1.0 / (R2 * cy[i] * cy[i]);     // src/eikonal_solver.cpp:385
        af32[i] = (float)af[i];
    }
    P->dx = xr[1] - xr[0];
    P->dy = yr[1] - yr[0];
    SA_CUDA(P->xx_deg.upload(xx_deg, nx, st));
    SA_CUDA(P->yy_deg.upload(yy_deg, ny, st));
    SA_CUDA(P->xx.upload(xr.data(), nx, st));
    SA_CUDA(P->yy.upload(yr.data(), ny, st));
    SA_CUDA(P->cosy.upload(cy.data(), ny, st));
    SA_CUDA(P->siny.upload(sy.data(), ny, st));
    SA_CUDA(P->a_f_row64.upload(af.data(), ny, st));
    SA_CUDA(P->a_a_row64.upload(aa.data(), ny, st));
    SA_CUDA(P->a_f_row32.upload(af32.data(), ny, st));
    SA_CUDA(cudaStreamSynchronize(st));
    return SA_OK;
}

int plan_events(sa_plan* P, int ne, const double* evlo, const double* evla, const int* iper,
                const int* rec_ptr, const int* rec_idx, int nsta, const double* stlo,
                const double* stla) {
    sa_ctx* ctx = P->ctx;
    cudaStream_t st = ctx->stream;
    const int nx = P->nx, ny = P->ny;
    const size_t n = (size_t)nx * ny;
    P->ne = ne;
    P->nsta = nsta;
    P->npair = ne > 0 ? rec_ptr[ne] : 0;
    if (ne > 0 && rec_ptr[0] != 0) return fail(ctx, SA_ERR_ARG, "rec_ptr[0] must be 0");
    for (int e = 0; e < ne; e++) {
        if (iper[e] < 0 || iper[e] >= P->nper) return fail(ctx, SA_ERR_ARG, "iper out of range");
        const int nr = rec_ptr[e + 1] - rec_ptr[e];
        if (nr < 0) return fail(ctx, SA_ERR_ARG, "rec_ptr must be non-decreasing");
        if ((size_t)nr > n) return fail(ctx, SA_ERR_ARG, "more receivers than grid cells");
        P->maxr = std::max(P->maxr, nr);
    }
    for (int i = 0; i < P->npair; i++)
        if (rec_idx[i] < 0 || rec_idx[i] >= nsta)
            return fail(ctx, SA_ERR_ARG, "rec_idx out of range");
    // unique sources (SrcRec groups events by source name; here by position)
    std::unordered_map<uint64_t, std::vector<int>> buckets;
    std::vector<int> src(ne);
    std::vector<double> ux, uy;
    for (int e = 0; e < ne; e++) {
        uint64_t a, b;
        std::memcpy(&a, &evlo[e], 8);
        std::memcpy(&b, &evla[e], 8);
        const uint64_t h = a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull);
        int found = -1;
        for (int s : buckets[h])
            if (ux[s] == evlo[e] && uy[s] == evla[e]) found = s;
        if (found < 0) {
            found = (int)ux.size();
            ux.push_back(evlo[e]);
            uy.push_back(evla[e]);
            buckets[h].push_back(found);
        }
        src[e] = found;
    }
    const int nsrc = (int)ux.size();
    P->nsrc = nsrc;
    std::vector<double> hxx(nx);
    SA_CUDA(cudaMemcpy(hxx.data(), P->xx.p, nx * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<double> sy0(std::max(nsrc, 1)), cy0(std::max(nsrc, 1));
    std::vector<double> cdl((size_t)std::max(nsrc, 1) * nx), sdl((size_t)std::max(nsrc, 1) * nx);
    for (int s = 0; s < nsrc; s++) {
        const double x0 = ux[s] * DEG2RAD, y0 = uy[s] * DEG2RAD;
        sy0[s] = std::sin(y0);
        cy0[s] = std::cos(y0);
        for (int ix = 0; ix < nx; ix++) {
            const double dlon = hxx[ix] - x0;
            cdl[(size_t)s * nx + ix] = std::cos(dlon);
            sdl[(size_t)s * nx + ix] = std::sin(dlon);
        }
    }
    std::vector<double> cst(std::max(nsta, 1));
    for (int i = 0; i < nsta; i++) cst[i] = std::cos(stla[i] * DEG2RAD);
    SA_CUDA(P->evlo.upload(evlo, ne, st));
    SA_CUDA(P->evla.upload(evla, ne, st));
    SA_CUDA(P->iper.upload(iper, ne, st));
    SA_CUDA(P->src.upload(src.data(), ne, st));
    SA_CUDA(P->rec_ptr.upload(rec_ptr, ne + 1, st));
    SA_CUDA(P->rec_idx.upload(rec_idx, P->npair, st));
    SA_CUDA(P->stlo.upload(stlo, nsta, st));
    SA_CUDA(P->stla.upload(stla, nsta, st));
    SA_CUDA(P->cos_stla.upload(cst.data(), nsta, st));
    DArr<double> d_sy0, d_cy0, d_cdl, d_sdl;
    SA_CUDA(d_sy0.upload(sy0.data(), nsrc, st));
    SA_CUDA(d_cy0.upload(cy0.data(), nsrc, st));
    SA_CUDA(d_cdl.upload(cdl.data(), (size_t)nsrc * nx, st));
    SA_CUDA(d_sdl.upload(sdl.data(), (size_t)nsrc * nx, st));
    const size_t ng = (size_t)std::max(nsrc, 1) * n;
    SA_CUDA(P->G64.alloc(ng));
    if (P->prec == SA_FP64) {
        // FP64 parity path: great-circle geometry from the C library's acos,
        // i.e. the very T0 a CPU evaluation of src/eikonal_solver.cpp:96-116
        // produces.  It depends on the stations only and is built once per
        // plan; T, residuals and adjoint fields are then bit-identical.
        SA_CUDA(P->Gx64.alloc(ng));
        SA_CUDA(P->Gy64.alloc(ng));
        std::vector<double> hG(ng), hGx(ng), hGy(ng), sy(ny), cy(ny);
        SA_CUDA(cudaMemcpy(sy.data(), P->siny.p, ny * sizeof(double), cudaMemcpyDeviceToHost));
        SA_CUDA(cudaMemcpy(cy.data(), P->cosy.p, ny * sizeof(double), cudaMemcpyDeviceToHost));
        const int nth = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), 64));
        std::vector<std::thread> pool;
        for (int t = 0; t < nth; t++)
            pool.emplace_back([&, t]() {
                for (int s = t; s < nsrc; s += nth)
                    for (int iy = 0; iy < ny; iy++)
                        for (int ix = 0; ix < nx; ix++) {
                            const size_t i = (size_t)s * n + (size_t)iy * nx + ix;
                            const double cdlv = cdl[(size_t)s * nx + ix];
                            const double sdlv = sdl[(size_t)s * nx + ix];
                            const double tmp = sy[iy] * sy0[s] + cy[iy] * cy0[s] * cdlv;
                            const double tmp_c = std::max(-1.0, std::min(1.0, tmp));
                            hG[i] = std::acos(tmp_c) * R_EARTH;
                            const double sin_d = std::sqrt(std::max(0.0, 1.0 - tmp_c * tmp_c));
                            if (sin_d < 1e-14) {
                                hGx[i] = 0.0;
                                hGy[i] = 0.0;
                            } else {
                                hGx[i] = cy[iy] * cy0[s] * sdlv / sin_d * R_EARTH;
                                hGy[i] = -(cy[iy] * sy0[s] - sy[iy] * cy0[s] * cdlv) / sin_d * R_EARTH;
                            }
                        }
            });
        for (auto& th : pool) th.join();
        if (nsrc) {
            SA_CUDA(cudaMemcpyAsync(P->G64.p, hG.data(), ng * sizeof(double), cudaMemcpyHostToDevice, st));
            SA_CUDA(cudaMemcpyAsync(P->Gx64.p, hGx.data(), ng * sizeof(double), cudaMemcpyHostToDevice, st));
            SA_CUDA(cudaMemcpyAsync(P->Gy64.p, hGy.data(), ng * sizeof(double), cudaMemcpyHostToDevice, st));
            SA_CUDA(cudaStreamSynchronize(st));
        }
    } else {
        SA_CUDA(P->G32.alloc(ng));
        SA_CUDA(P->Gx32.alloc(ng));
        SA_CUDA(P->Gy32.alloc(ng));
        if (nsrc)
            SA_CUDA(launch_geometry<float>(nx, ny, nsrc, P->siny.p, P->cosy.p, d_sy0.p, d_cy0.p,
                                           d_cdl.p, d_sdl.p, P->G32.p, P->Gx32.p, P->Gy32.p,
                                           P->G64.p, st));
    }
    SA_CUDA(P->chi_ev.alloc(std::max(ne, 1)));
    SA_CUDA(P->status_tmp.alloc(std::max(ne, 1)));
    SA_CUDA(P->worst.alloc(1));
    SA_CUDA(P->queue.alloc(1));
    {
        const size_t ne1 = (size_t)std::max(ne, 1);
        SA_CUDA(P->fit.alloc(ne1));
        SA_CUDA(P->ait.alloc(ne1));
        SA_CUDA(cudaMemsetAsync(P->fit.p, 0, ne1 * sizeof(int), st));
        SA_CUDA(cudaMemsetAsync(P->ait.p, 0, ne1 * sizeof(int), st));
        std::vector<int> iota(ne1);
        for (size_t i = 0; i < ne1; i++) iota[i] = (int)i;
        SA_CUDA(P->order.upload(iota.data(), ne1, st));
        SA_CUDA(P->ord_idx.alloc(ne1));
        SA_CUDA(P->key_a.alloc(ne1));
        SA_CUDA(P->key_b.alloc(ne1));
        P->sort_bytes = ne > 0 ? sort_events_temp_bytes(ne) : 0;
        SA_CUDA(P->sort_tmp.alloc(std::max<size_t>(P->sort_bytes, 1)));
    }
    // scratch slots: one per resident warp, bounded by events and free memory
    const int maxs = P->prec == SA_FP64 ? batch64_max_slots(ctx->device) : batch32_max_slots(ctx->device);
    P->slot_bytes = P->prec == SA_FP64 ? batch64_slot_bytes(nx, ny, P->maxr)
                                       : batch32_slot_bytes(nx, ny, P->maxr);
    size_t fr = 0, tot = 0;
    SA_CUDA(cudaMemGetInfo(&fr, &tot));
    const size_t budget = fr / 10 * 7;
    int ns = std::min(maxs, std::max(ne, 1));
    while (ns > 1 && (size_t)ns * P->slot_bytes > budget) ns--;
    P->nslots = ns;
    SA_CUDA(P->scratch.alloc((size_t)ns * P->slot_bytes));
    // the adjoint-source plane of every slot must start at zero
    SA_CUDA(cudaMemsetAsync(P->scratch.p, 0, (size_t)ns * P->slot_bytes, st));
    SA_CUDA(cudaStreamSynchronize(st));
    return SA_OK;
}

int plan_media(sa_plan* P, const double* svel, const double* m11, const double* m12,
               const double* m22, bool general, cudaStream_t st) {
    sa_ctx* ctx = P->ctx;
    const size_t np = (size_t)P->nx * P->ny * P->nper;
    SA_CUDA(P->fun64.alloc(np));
    SA_CUDA(P->inv3.alloc(np));
    if (general) {
        SA_CUDA(P->mt64.alloc(4 * np));
        SA_CUDA(P->b_p64.alloc(np));
        SA_CUDA(P->a_a64.alloc(np));
        SA_CUDA(P->c_a64.alloc(np));
    }
    SA_CUDA(launch_media64(P->nx, P->ny, P->nper, svel, general ? m11 : nullptr, m12, m22,
                           P->cosy.p, P->fun64.p, P->inv3.p, P->mt64.p, P->b_p64.p, P->a_a64.p,
                           P->c_a64.p, st));
    if (P->prec == SA_FP32) {
        SA_CUDA(P->fun32.alloc(np));
        if (general) SA_CUDA(P->mt32.alloc(4 * np));
        SA_CUDA(launch_media32(P->nx, P->ny, P->nper, P->fun64.p, general ? P->mt64.p : nullptr,
                               P->fun32.p, P->mt32.p, st));
    }
    return SA_OK;
}

BatchDesc plan_desc(sa_plan* P, bool general) {
    BatchDesc d{};
    d.g.nx = P->nx;
    d.g.ny = P->ny;
    d.g.xx_deg = P->xx_deg.p;
    d.g.yy_deg = P->yy_deg.p;
    d.g.xx = P->xx.p;
    d.g.yy = P->yy.p;
    d.g.cosy = P->cosy.p;
    d.g.siny = P->siny.p;
    d.g.dx = P->dx;
    d.g.dy = P->dy;
    d.nper = P->nper;
    d.iso = general ? 0 : 1;
    d.fun64 = P->fun64.p;
    d.inv3 = P->inv3.p;
    d.a_f_row64 = P->a_f_row64.p;
    d.a_a_row64 = P->a_a_row64.p;
    d.b_iso = 1.0 / (R_EARTH * R_EARTH);
    d.mt64 = P->mt64.p;
    d.b_p64 = P->b_p64.p;
    d.a_a64 = P->a_a64.p;
    d.c_a64 = P->c_a64.p;
    d.G64 = P->G64.p;
    d.Gx64 = P->Gx64.p;
    d.Gy64 = P->Gy64.p;
    d.fun32 = P->fun32.p;
    d.a_f_row32 = P->a_f_row32.p;
    d.b_iso32 = (float)d.b_iso;
    d.mt32 = P->mt32.p;
    d.G32 = P->G32.p;
    d.Gx32 = P->Gx32.p;
    d.Gy32 = P->Gy32.p;
    d.ev.ne = P->ne;
    d.ev.src = P->src.p;
    d.ev.iper = P->iper.p;
    d.ev.evlo = P->evlo.p;
    d.ev.evla = P->evla.p;
    d.ev.rec_ptr = P->rec_ptr.p;
    d.ev.rec_idx = P->rec_idx.p;
    d.ev.stlo = P->stlo.p;
    d.ev.stla = P->stla.p;
    d.ev.cos_stla = P->cos_stla.p;
    d.sc.nslots = (P->active > 0 && P->active < P->nslots) ? P->active : P->nslots;
    d.sc.nwarps = P->nslots;
    d.sc.slot_bytes = P->slot_bytes;
    d.variant = P->prec == SA_FP32 ? P->variant : 0;
    d.discrete = P->discrete;
    d.sc.base = P->scratch.p;
    d.sc.queue = P->queue.p;
    d.maxr = P->maxr;
    return d;
}

// Enqueue one evaluation (no synchronisation).
int plan_enqueue(sa_plan* P, const double* svel, const double* m11, const double* m12,
                 const double* m22, const double* tt_obs, const double* weight, int calc_adj,
                 double* syn, double* adj_s, double* chi, int* fwd_iters, int* adj_iters,
                 int* status, cudaStream_t st, const double* sadj = nullptr) {
    sa_ctx* ctx = P->ctx;
    const bool general = m11 != nullptr;
    int rc = plan_media(P, svel, m11, m12, m22, general, st);
    if (rc) return rc;
    BatchDesc d = plan_desc(P, general);
    d.ev.tt_obs = tt_obs;
    d.ev.weight = weight;
    d.ev.sadj = sadj;
    d.out.syn = syn;
    d.out.chi_ev = (calc_adj && chi && !sadj) ? P->chi_ev.p : nullptr;
    d.out.adj_s = calc_adj ? adj_s : nullptr;
    d.out.fwd_iters = P->fit.p;
    d.out.adj_iters = P->ait.p;
    d.sc.order = P->order.p;
    d.out.status = status ? status : P->status_tmp.p;
    d.out.T_out = P->dbg_T;
    d.out.Ta_out = P->dbg_Ta;
    d.out.kden_s = (calc_adj && !sadj) ? P->kden_out : nullptr;
    d.mode = calc_adj ? MODE_FWD_ADJ : MODE_FWD;
    SA_CUDA(cudaMemsetAsync(P->queue.p, 0, sizeof(unsigned int), st));
    if (calc_adj && adj_s)
        SA_CUDA(cudaMemsetAsync(adj_s, 0, (size_t)P->nx * P->ny * P->nper * sizeof(double), st));
    if (d.out.kden_s)
        SA_CUDA(cudaMemsetAsync(d.out.kden_s, 0,
                                (size_t)P->nx * P->ny * P->nper * sizeof(double), st));
    const bool determ = P->determ && calc_adj && adj_s && P->ne > 0;
    if (P->ne > 0) {
        if (P->timing) SA_CUDA(cudaEventRecord(P->tk0, st));
        if (!determ) {
            SA_CUDA(P->prec == SA_FP64 ? launch_batch64(d, st) : launch_batch32(d, st));
        } else {
            // chunks of events in event order; within a chunk the queue hands
            // them out in index order, and the ordered reduction adds their
            // planes to adj_s as the reference's event loop does
            const size_t n = (size_t)P->nx * P->ny;
            for (int e0 = 0, c = 0; e0 < P->ne; e0 += P->chunk, c++) {
                const int e1 = std::min(P->ne, e0 + P->chunk);
                BatchDesc dc = d;
                dc.ev.ne = e1 - e0;
                dc.sc.order = P->iota.p + e0;
                dc.out.contrib = P->contrib.p;
                dc.out.contrib_e0 = e0;
                if (e0 > 0) SA_CUDA(cudaMemsetAsync(P->queue.p, 0, sizeof(unsigned int), st));
                SA_CUDA(P->prec == SA_FP64 ? launch_batch64(dc, st) : launch_batch32(dc, st));
                SA_CUDA(launch_ordered_accumulate(n, P->nper, e0,
                                                  P->per_ptr.p + (size_t)c * (P->nper + 1),
                                                  P->per_ev.p, P->contrib.p, adj_s, st));
            }
        }
        if (P->timing) SA_CUDA(cudaEventRecord(P->tk1, st));
        if (calc_adj && chi && !sadj)
            SA_CUDA(determ ? launch_sum_events_ordered(P->ne, P->chi_ev.p, chi, st)
                           : launch_sum_events(P->ne, P->chi_ev.p, chi, st));
        SA_CUDA(launch_fold_status(P->ne, d.out.status, P->worst.p, st));
        const size_t ib = (size_t)P->ne * sizeof(int);
        if (fwd_iters)
            SA_CUDA(cudaMemcpyAsync(fwd_iters, P->fit.p, ib, cudaMemcpyDeviceToDevice, st));
        if (calc_adj && adj_iters)
            SA_CUDA(cudaMemcpyAsync(adj_iters, P->ait.p, ib, cudaMemcpyDeviceToDevice, st));
        SA_CUDA(launch_event_cost(P->ne, P->fit.p, P->ait.p, P->key_a.p, P->ord_idx.p, st));
        SA_CUDA(launch_sort_events(P->ne, P->key_a.p, P->key_b.p, P->ord_idx.p, P->order.p,
                                   P->sort_tmp.p, P->sort_bytes, st));
    } else {
        if (calc_adj && chi) SA_CUDA(cudaMemsetAsync(chi, 0, sizeof(double), st));
        SA_CUDA(cudaMemsetAsync(P->worst.p, 0, sizeof(int), st));
    }
    return SA_OK;
}

}  // namespace

extern "C" int sa_plan_create(sa_ctx* ctx, int precision, int nx, int ny, int nper,
                              const double* xx_deg, const double* yy_deg, int ne,
                              const double* evlo, const double* evla, const int* iper,
                              const int* rec_ptr, const int* rec_idx, int nsta,
                              const double* stlo, const double* stla, sa_plan** out) {
    if (!ctx || !out) return SA_ERR_ARG;
    *out = nullptr;
    if (precision != SA_FP64 && precision != SA_FP32) return fail(ctx, SA_ERR_ARG, "precision");
    if (nx < 3 || ny < 3) return fail(ctx, SA_ERR_ARG, "Grid must be at least 3x3");
    if (nper < 1 || ne < 0 || nsta < 0) return fail(ctx, SA_ERR_ARG, "nper/ne/nsta");
    if (!xx_deg || !yy_deg || (ne > 0 && (!evlo || !evla || !iper || !rec_ptr)))
        return fail(ctx, SA_ERR_ARG, "null input");
    SA_CUDA(cudaSetDevice(ctx->device));
    sa_plan* P = new sa_plan();
    P->ctx = ctx;
    P->prec = precision;
    P->nx = nx;
    P->ny = ny;
    P->nper = nper;
    int rc = plan_grid(P, xx_deg, yy_deg);
    if (!rc) rc = plan_events(P, ne, evlo, evla, iper, rec_ptr, rec_idx, nsta, stlo, stla);
    if (rc) {
        delete P;
        return rc;
    }
    // a configuration tuned earlier for this grid size
    const auto it = ctx->tune.find({nx, ny, precision});
    if (it != ctx->tune.end()) {
        P->variant = it->second[0];
        P->active = it->second[1];
    }
    *out = P;
    return SA_OK;
}

extern "C" void sa_plan_destroy(sa_plan* plan) { delete plan; }

// Launch-configuration autotuner.  Candidates: every FP32 launch variant
// (rolled / unrolled forward step x adjoint load lead 2 / 3 x tail teams off
// / on; FP64: the one kernel) x all or three quarters of the resident event
// slots, and with tail teams also a quarter (one solve per block).  Each
// candidate runs the plan's own evaluation twice, the second timed with
// CUDA events around the batch kernel; the fastest is kept for this plan and
// for plans of the same grid size created later on this context.  Results do
// not depend on the choice: the FP32 sweeps spell out every rounding, so all
// variants compute the same values (only the atomic accumulation order of
// adj_s varies).
extern "C" int sa_plan_autotune(sa_plan* P, const double* svel, const double* m11,
                                const double* m12, const double* m22, const double* tt_obs,
                                const double* weight, int calc_adj, double* adj_s,
                                float* ms_out, int* n_out, int* choice, void* stream) {
    if (!P) return SA_ERR_ARG;
    sa_ctx* ctx = P->ctx;
    if (!svel) return fail(ctx, SA_ERR_ARG, "svel is required");
    if ((m11 == nullptr) != (m22 == nullptr) || (m11 == nullptr) != (m12 == nullptr))
        return fail(ctx, SA_ERR_ARG, "m11, m12, m22 must be all set or all NULL");
    if (P->npair > 0 && (!tt_obs || !weight)) return fail(ctx, SA_ERR_ARG, "tt_obs/weight");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const int nvar = P->prec == SA_FP32 ? kBatchVariants : 1;
    // (variant, slots in use): all or three quarters; with tail teams also a
    // quarter (one solve per block, its three other warps as the team)
    std::vector<std::pair<int, int>> cand;
    for (int v = 0; v < nvar; v++) {
        cand.push_back({v, 0});
        cand.push_back({v, std::max(1, P->nslots * 3 / 4)});
        if (v & 4) cand.push_back({v, std::max(1, P->nslots / 4)});
    }
    const int ncand = (int)cand.size();
    const bool had_timing = P->timing;
    if (!P->tk0) {
        SA_CUDA(cudaEventCreate(&P->tk0));
        SA_CUDA(cudaEventCreate(&P->tk1));
    }
    P->timing = true;
    float best = 0.f;
    int best_c = 0;
    for (int c = 0; c < ncand; c++) {
        P->variant = cand[c].first;
        P->active = cand[c].second;
        float ms = 0.f;
        for (int rep = 0; rep < 2; rep++) {
            const int rc = plan_enqueue(P, svel, m11, m12, m22, tt_obs, weight, calc_adj,
                                        nullptr, adj_s, nullptr, nullptr, nullptr, nullptr, st);
            if (rc) {
                P->timing = had_timing;
                return rc;
            }
        }
        SA_CUDA(cudaEventSynchronize(P->tk1));
        SA_CUDA(cudaEventElapsedTime(&ms, P->tk0, P->tk1));
        if (ms_out && c < SA_TUNE_MAX_CANDIDATES) ms_out[c] = ms;
        if (c == 0 || ms < best) {
            best = ms;
            best_c = c;
        }
    }
    P->timing = had_timing;
    P->variant = cand[best_c].first;
    P->active = cand[best_c].second;
    P->have_graph = false;
    ctx->tune[{P->nx, P->ny, P->prec}] = {P->variant, P->active};
    if (n_out) *n_out = ncand;
    if (choice) *choice = best_c;
    return SA_OK;
}

extern "C" int sa_plan_set_tune(sa_plan* P, int variant, int active_slots) {
    if (!P) return SA_ERR_ARG;
    const int nvar = P->prec == SA_FP32 ? kBatchVariants : 1;
    if (variant < 0 || variant >= nvar || active_slots < 0)
        return fail(P->ctx, SA_ERR_ARG, "sa_plan_set_tune: variant or active_slots out of range");
    P->variant = variant;
    P->active = active_slots;
    P->have_graph = false;
    return SA_OK;
}

extern "C" int sa_plan_get_tune(sa_plan* P, int* variant, int* active_slots, int* nslots) {
    if (!P) return SA_ERR_ARG;
    if (variant) *variant = P->variant;
    if (active_slots) *active_slots = P->active > 0 ? std::min(P->active, P->nslots) : P->nslots;
    if (nslots) *nslots = P->nslots;
    return SA_OK;
}

extern "C" int sa_plan_kden_output(sa_plan* P, double* kden_s) {
    if (!P) return SA_ERR_ARG;
    P->kden_out = kden_s;
    return SA_OK;
}

extern "C" int sa_plan_set_deterministic(sa_plan* P, int enable, size_t max_bytes) {
    if (!P) return SA_ERR_ARG;
    sa_ctx* ctx = P->ctx;
    SA_CUDA(cudaSetDevice(ctx->device));
    P->have_graph = false;   // the evaluation's launches change
    if (!enable) {
        P->determ = false;
        P->contrib.release();
        return SA_OK;
    }
    const size_t n = (size_t)P->nx * P->ny;
    if (max_bytes == 0) {
        size_t fr = 0, tot = 0;
        SA_CUDA(cudaMemGetInfo(&fr, &tot));
        max_bytes = fr / 4;
    }
    const int ne = std::max(P->ne, 1);
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(ne, max_bytes / (n * 8)));
    std::vector<int> iper(ne, 0);
    if (P->ne > 0)
        SA_CUDA(cudaMemcpy(iper.data(), P->iper.p, P->ne * sizeof(int), cudaMemcpyDeviceToHost));
    const int nchunk = (P->ne + chunk - 1) / chunk;
    std::vector<int> iota(ne), ptr, ev;
    for (int e = 0; e < ne; e++) iota[e] = e;
    for (int c = 0; c < nchunk; c++) {
        const int e0 = c * chunk, e1 = std::min(P->ne, e0 + chunk);
        for (int ip = 0; ip < P->nper; ip++) {
            ptr.push_back((int)ev.size());
            for (int e = e0; e < e1; e++)
                if (iper[e] == ip) ev.push_back(e);
        }
        ptr.push_back((int)ev.size());
    }
    if (ptr.empty()) ptr.push_back(0);
    if (ev.empty()) ev.push_back(0);
    SA_CUDA(P->contrib.alloc((size_t)chunk * n));
    SA_CUDA(P->iota.upload(iota.data(), iota.size(), ctx->stream));
    SA_CUDA(P->per_ptr.upload(ptr.data(), ptr.size(), ctx->stream));
    SA_CUDA(P->per_ev.upload(ev.data(), ev.size(), ctx->stream));
    SA_CUDA(cudaStreamSynchronize(ctx->stream));
    P->chunk = chunk;
    P->determ = true;
    return SA_OK;
}

extern "C" int sa_plan_set_graph(sa_plan* plan, int enable) {
    if (!plan) return SA_ERR_ARG;
    plan->use_graph = enable != 0;
    return SA_OK;
}

extern "C" int sa_plan_kernel_timing(sa_plan* P, int enable) {
    if (!P) return SA_ERR_ARG;
    sa_ctx* ctx = P->ctx;
    SA_CUDA(cudaSetDevice(ctx->device));
    if (enable && !P->tk0) {
        SA_CUDA(cudaEventCreate(&P->tk0));
        SA_CUDA(cudaEventCreate(&P->tk1));
    }
    P->timing = enable != 0;
    return SA_OK;
}

extern "C" int sa_plan_kernel_ms(sa_plan* P, float* ms) {
    if (!P || !ms) return SA_ERR_ARG;
    sa_ctx* ctx = P->ctx;
    if (!P->tk0) return fail(ctx, SA_ERR_ARG, "kernel timing is not enabled");
    SA_CUDA(cudaEventSynchronize(P->tk1));
    SA_CUDA(cudaEventElapsedTime(ms, P->tk0, P->tk1));
    return SA_OK;
}

extern "C" int sa_plan_debug_fields(sa_plan* plan, double* T_out, double* Ta_out) {
    if (!plan) return SA_ERR_ARG;
    plan->dbg_T = T_out;
    plan->dbg_Ta = Ta_out;
    plan->have_graph = false;
    return SA_OK;
}

namespace {
// One evaluation, replayed from the plan's CUDA graph when the pointers repeat.
int plan_run(sa_plan* P, const double* svel, const double* m11, const double* m12,
             const double* m22, const double* tt_obs, const double* weight, const double* sadj,
             int calc_adj, double* syn, double* adj_s, double* chi, int* fwd_iters,
             int* adj_iters, int* status, void* stream) {
    sa_ctx* ctx = P->ctx;
    if (!svel) return fail(ctx, SA_ERR_ARG, "svel is required");
    if ((m11 == nullptr) != (m22 == nullptr) || (m11 == nullptr) != (m12 == nullptr))
        return fail(ctx, SA_ERR_ARG, "m11, m12, m22 must be all set or all NULL");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    if (!P->use_graph || P->timing)
        return plan_enqueue(P, svel, m11, m12, m22, tt_obs, weight, calc_adj, syn, adj_s, chi,
                            fwd_iters, adj_iters, status, st, sadj);
    GraphKey k{};
    const void* ptrs[17] = {svel, m11, m12, m22, tt_obs, weight, syn, adj_s, chi, fwd_iters,
                            adj_iters, status, P->dbg_T, P->dbg_Ta, sadj, P->kden_out, nullptr};
    std::memcpy(k.ptr, ptrs, sizeof(ptrs));
    k.calc_adj = calc_adj;
    if (!(P->have_graph && P->key == k)) {
        if (P->gexec) {
            cudaGraphExecDestroy(P->gexec);
            P->gexec = nullptr;
        }
        P->have_graph = false;
        // allocations happen outside the capture
        int rc = plan_media(P, svel, m11, m12, m22, m11 != nullptr, st);
        if (rc) return rc;
        SA_CUDA(cudaStreamSynchronize(st));
        cudaGraph_t graph = nullptr;
        SA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        rc = plan_enqueue(P, svel, m11, m12, m22, tt_obs, weight, calc_adj, syn, adj_s, chi,
                          fwd_iters, adj_iters, status, st, sadj);
        cudaError_t ce = cudaStreamEndCapture(st, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        SA_CUDA(ce);
        ce = cudaGraphInstantiate(&P->gexec, graph, 0);
        cudaGraphDestroy(graph);
        SA_CUDA(ce);
        P->key = k;
        P->have_graph = true;
    }
    SA_CUDA(cudaGraphLaunch(P->gexec, st));
    return SA_OK;
}
}  // namespace

extern "C" int sa_plan_forward_adjoint(sa_plan* P, const double* svel, const double* m11,
                                       const double* m12, const double* m22,
                                       const double* tt_obs, const double* weight, int calc_adj,
                                       double* syn, double* adj_s, double* chi, int* fwd_iters,
                                       int* adj_iters, int* status, void* stream) {
    if (!P) return SA_ERR_ARG;
    if (P->npair > 0 && (!tt_obs || !weight)) return fail(P->ctx, SA_ERR_ARG, "tt_obs/weight");
    return plan_run(P, svel, m11, m12, m22, tt_obs, weight, nullptr, calc_adj, syn, adj_s, chi,
                    fwd_iters, adj_iters, status, stream);
}

extern "C" int sa_plan_adjoint_source(sa_plan* P, const double* svel, const double* m11,
                                      const double* m12, const double* m22,
                                      const double* source_adj, double* syn, double* adj_s,
                                      int* status, void* stream) {
    if (!P) return SA_ERR_ARG;
    if (P->npair > 0 && !source_adj) return fail(P->ctx, SA_ERR_ARG, "source_adj is required");
    if (!adj_s) return fail(P->ctx, SA_ERR_ARG, "adj_s is required");
    return plan_run(P, svel, m11, m12, m22, nullptr, nullptr, source_adj, 1, syn, adj_s,
                    nullptr, nullptr, nullptr, status, stream);
}

extern "C" int sa_plan_set_adjoint(sa_plan* P, int kind) {
    if (!P) return SA_ERR_ARG;
    if (kind != 0 && kind != 1) return fail(P->ctx, SA_ERR_ARG, "adjoint kind 0 or 1");
    if (kind == 1 && P->prec != SA_FP64)
        return fail(P->ctx, SA_ERR_ARG, "the exact discrete adjoint needs an FP64 plan");
    if (kind != P->discrete) {
        P->discrete = kind;
        P->have_graph = false;   // recapture with the new kernel arguments
    }
    return SA_OK;
}

// ---- one launch over several plans (grid levels) ----------------------------

struct sa_multi {
    sa_ctx* ctx = nullptr;
    std::vector<sa_plan*> plans;
    std::vector<int> off;          // first queue entry of each level
    int prec = SA_FP32, ntotal = 0, nslots = 0;
    size_t slot_bytes = 0;
    DArr<unsigned char> args, scratch, sort_tmp;
    DArr<unsigned int> queue, key_a, key_b;
    DArr<int> code_in, code;
    size_t sort_bytes = 0;
    cudaEvent_t tk0 = nullptr, tk1 = nullptr;
    ~sa_multi() {
        if (tk0) cudaEventDestroy(tk0);
        if (tk1) cudaEventDestroy(tk1);
    }
};

extern "C" int sa_multi_create(sa_plan* const* plans, int nplans, sa_multi** out) {
    if (!plans || nplans < 1 || nplans > 127 || !out || !plans[0]) return SA_ERR_ARG;
    *out = nullptr;
    sa_ctx* ctx = plans[0]->ctx;
    SA_CUDA(cudaSetDevice(ctx->device));
    sa_multi* M = new sa_multi();
    M->ctx = ctx;
    M->prec = plans[0]->prec;
    const int maxs =
        M->prec == SA_FP64 ? batch64_max_slots(ctx->device) : batch32_max_slots(ctx->device);
    for (int i = 0; i < nplans; i++) {
        sa_plan* P = plans[i];
        if (!P || P->ctx != ctx || P->prec != M->prec || P->ne >= (1 << 24)) {
            delete M;
            return fail(ctx, SA_ERR_ARG, "sa_multi_create: plans of one context and precision, "
                                         "fewer than 2^24 events each");
        }
        M->plans.push_back(P);
        M->off.push_back(M->ntotal);
        M->ntotal += P->ne;
        M->slot_bytes = std::max(M->slot_bytes, P->slot_bytes);
    }
    const size_t nt = (size_t)std::max(M->ntotal, 1);
    size_t fr = 0, tot = 0;
    cudaError_t e = cudaMemGetInfo(&fr, &tot);
    int ns = std::min(maxs, std::max(M->ntotal, 1));
    while (ns > 1 && (size_t)ns * M->slot_bytes > fr / 10 * 7) ns--;
    M->nslots = ns;
    std::vector<int> code(nt, 0);
    for (int i = 0; i < nplans; i++)
        for (int k = 0; k < plans[i]->ne; k++) code[M->off[i] + k] = (i << 24) | k;
    const size_t argb = M->prec == SA_FP64 ? batch64_args_bytes() : batch32_args_bytes();
    M->sort_bytes = sort_events_temp_bytes((int)nt);
    if (e == cudaSuccess) e = M->args.alloc(argb * nplans);
    if (e == cudaSuccess) e = M->scratch.alloc((size_t)ns * M->slot_bytes);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(M->scratch.p, 0, (size_t)ns * M->slot_bytes, ctx->stream);
    if (e == cudaSuccess) e = M->queue.alloc(1);
    if (e == cudaSuccess) e = M->key_a.alloc(nt);
    if (e == cudaSuccess) e = M->key_b.alloc(nt);
    if (e == cudaSuccess) e = M->code_in.alloc(nt);
    if (e == cudaSuccess) e = M->code.upload(code.data(), nt, ctx->stream);
    if (e == cudaSuccess) e = M->sort_tmp.alloc(std::max<size_t>(M->sort_bytes, 1));
    if (e == cudaSuccess) e = cudaEventCreate(&M->tk0);
    if (e == cudaSuccess) e = cudaEventCreate(&M->tk1);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        delete M;
        return fail(ctx, e == cudaErrorMemoryAllocation ? SA_ERR_NOMEM : SA_ERR_CUDA,
                    std::string("sa_multi_create: ") + cudaGetErrorString(e));
    }
    *out = M;
    return SA_OK;
}

extern "C" void sa_multi_destroy(sa_multi* M) {
    if (!M) return;
    cudaSetDevice(M->ctx->device);
    delete M;
}

extern "C" int sa_multi_forward_adjoint(sa_multi* M, const double* const* svel,
                                        const double* const* m11, const double* const* m12,
                                        const double* const* m22, const double* const* tt_obs,
                                        const double* const* weight, int calc_adj,
                                        double* const* syn, double* const* adj_s,
                                        double* const* chi, int* const* status, void* stream) {
    if (!M || !svel || !tt_obs || !weight) return SA_ERR_ARG;
    sa_ctx* ctx = M->ctx;
    const int nlev = (int)M->plans.size();
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const bool general = m11 && m11[0];
    std::vector<BatchDesc> d(nlev);
    for (int i = 0; i < nlev; i++) {
        sa_plan* P = M->plans[i];
        const bool gi = m11 && m11[i];
        if (gi != general || (gi && (!m12 || !m22 || !m12[i] || !m22[i])))
            return fail(ctx, SA_ERR_ARG, "sa_multi: media for every plan or for none");
        if (!svel[i] || (P->npair > 0 && (!tt_obs[i] || !weight[i])))
            return fail(ctx, SA_ERR_ARG, "sa_multi: svel, tt_obs and weight for every plan");
        int rc = plan_media(P, svel[i], gi ? m11[i] : nullptr, gi ? m12[i] : nullptr,
                            gi ? m22[i] : nullptr, gi, st);
        if (rc) return rc;
        BatchDesc& b = d[i];
        b = plan_desc(P, gi);
        b.ev.tt_obs = tt_obs[i];
        b.ev.weight = weight[i];
        b.out.syn = syn ? syn[i] : nullptr;
        double* as = (calc_adj && adj_s) ? adj_s[i] : nullptr;
        b.out.adj_s = as;
        b.out.chi_ev = (calc_adj && chi && chi[i]) ? P->chi_ev.p : nullptr;
        b.out.fwd_iters = P->fit.p;
        b.out.adj_iters = P->ait.p;
        b.out.status = (status && status[i]) ? status[i] : P->status_tmp.p;
        b.mode = calc_adj ? MODE_FWD_ADJ : MODE_FWD;
        b.variant = M->prec == SA_FP32 ? M->plans[0]->variant : 0;
        if (as)
            SA_CUDA(cudaMemsetAsync(as, 0, (size_t)P->nx * P->ny * P->nper * sizeof(double), st));
    }
    Scratch sc{};
    sc.nslots = M->nslots;
    sc.slot_bytes = M->slot_bytes;
    sc.base = M->scratch.p;
    sc.queue = M->queue.p;
    sc.order = nullptr;
    SA_CUDA(cudaMemsetAsync(M->queue.p, 0, sizeof(unsigned int), st));
    SA_CUDA(cudaEventRecord(M->tk0, st));
    if (M->ntotal > 0) {
        const unsigned* code = reinterpret_cast<const unsigned*>(M->code.p);
        SA_CUDA(M->prec == SA_FP64
                    ? launch_batch64_multi(d.data(), nlev, M->args.p, M->ntotal, code, sc, st)
                    : launch_batch32_multi(d.data(), nlev, M->args.p, M->ntotal, code, sc, st));
    }
    SA_CUDA(cudaEventRecord(M->tk1, st));
    for (int i = 0; i < nlev; i++) {
        sa_plan* P = M->plans[i];
        if (P->ne == 0) {
            if (calc_adj && chi && chi[i]) SA_CUDA(cudaMemsetAsync(chi[i], 0, sizeof(double), st));
            SA_CUDA(cudaMemsetAsync(P->worst.p, 0, sizeof(int), st));
            continue;
        }
        if (calc_adj && chi && chi[i]) SA_CUDA(launch_sum_events(P->ne, P->chi_ev.p, chi[i], st));
        SA_CUDA(launch_fold_status(P->ne, d[i].out.status, P->worst.p, st));
        const unsigned scale = (unsigned)std::max<size_t>(1, (size_t)P->nx * P->ny / 256);
        SA_CUDA(launch_multi_cost(P->ne, P->fit.p, P->ait.p, scale, i, M->key_a.p + M->off[i],
                                  M->code_in.p + M->off[i], st));
    }
    // the next evaluation's queue: every plan's events by work, longest first
    if (M->ntotal > 0)
        SA_CUDA(launch_sort_events(M->ntotal, M->key_a.p, M->key_b.p, M->code_in.p, M->code.p,
                                   M->sort_tmp.p, M->sort_bytes, st));
    return SA_OK;
}

extern "C" int sa_multi_kernel_ms(sa_multi* M, float* ms) {
    if (!M || !ms) return SA_ERR_ARG;
    sa_ctx* ctx = M->ctx;
    SA_CUDA(cudaEventSynchronize(M->tk1));
    SA_CUDA(cudaEventElapsedTime(ms, M->tk0, M->tk1));
    return SA_OK;
}

extern "C" int sa_multi_status(sa_multi* M, int* worst) {
    if (!M || !worst) return SA_ERR_ARG;
    sa_ctx* ctx = M->ctx;
    *worst = 0;
    for (sa_plan* P : M->plans) {
        int w = 0;
        SA_CUDA(cudaMemcpy(&w, P->worst.p, sizeof(int), cudaMemcpyDeviceToHost));
        *worst = std::max(*worst, w);
    }
    return SA_OK;
}

namespace {
int plan_worst_status(sa_plan* P, cudaStream_t st) {
    sa_ctx* ctx = P->ctx;
    int w = 0;
    SA_CUDA(cudaMemcpyAsync(&w, P->worst.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SA_CUDA(cudaStreamSynchronize(st));
    if (w == ST_NOCONV) return fail(ctx, SA_ERR_NOCONV, "an event reached the sweep iteration cap");
    if (w == ST_NONFINITE) return fail(ctx, SA_ERR_NONFINITE, "non-finite travel-time or adjoint field");
    return SA_OK;
}
}  // namespace

extern "C" int sa_forward_for_events(sa_ctx* ctx, int precision, int nx, int ny, int nper,
                                     const double* xx_deg, const double* yy_deg,
                                     const double* svel, const double* m11, const double* m12,
                                     const double* m22, int ne, const double* evlo,
                                     const double* evla, const int* iper, const int* rec_ptr,
                                     const int* rec_idx, int nsta, const double* stlo,
                                     const double* stla, const double* tt_obs,
                                     const double* weight, int calc_adj, double* syn,
                                     double* adj_s, double* chi, int* fwd_iters,
                                     int* adj_iters) {
    sa_plan* P = nullptr;
    int rc = sa_plan_create(ctx, precision, nx, ny, nper, xx_deg, yy_deg, ne, evlo, evla, iper,
                            rec_ptr, rec_idx, nsta, stlo, stla, &P);
    if (rc) return rc;
    P->use_graph = false;
    cudaStream_t st = ctx->stream;
    const size_t np = (size_t)nx * ny * nper;
    const int npair = P->npair;
    const bool general = m11 != nullptr;
    DArr<double> d_svel, d_m11, d_m12, d_m22, d_tt, d_w, d_syn, d_adj, d_chi;
    DArr<int> d_fi, d_ai;
    auto done = [&](int code) {
        delete P;
        return code;
    };
#define SA_CUDA_P(call)                                                                     \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return done(fail(ctx, SA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_))); \
    } while (0)
    SA_CUDA_P(d_svel.upload(svel, np, st));
    if (general) {
        SA_CUDA_P(d_m11.upload(m11, np, st));
        SA_CUDA_P(d_m12.upload(m12, np, st));
        SA_CUDA_P(d_m22.upload(m22, np, st));
    }
    SA_CUDA_P(d_tt.upload(tt_obs, npair, st));
    SA_CUDA_P(d_w.upload(weight, npair, st));
    SA_CUDA_P(d_syn.alloc(npair));
    SA_CUDA_P(d_adj.alloc(np));
    SA_CUDA_P(d_chi.alloc(1));
    SA_CUDA_P(d_fi.alloc(std::max(ne, 1)));
    SA_CUDA_P(d_ai.alloc(std::max(ne, 1)));
    rc = sa_plan_forward_adjoint(P, d_svel.p, general ? d_m11.p : nullptr,
                                 general ? d_m12.p : nullptr, general ? d_m22.p : nullptr, d_tt.p,
                                 d_w.p, calc_adj, d_syn.p, d_adj.p, d_chi.p, d_fi.p, d_ai.p,
                                 nullptr, st);
    if (rc) return done(rc);
    if (syn && npair) SA_CUDA_P(cudaMemcpyAsync(syn, d_syn.p, npair * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (calc_adj && adj_s) SA_CUDA_P(cudaMemcpyAsync(adj_s, d_adj.p, np * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (calc_adj && chi) SA_CUDA_P(cudaMemcpyAsync(chi, d_chi.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (fwd_iters && ne) SA_CUDA_P(cudaMemcpyAsync(fwd_iters, d_fi.p, ne * sizeof(int), cudaMemcpyDeviceToHost, st));
    if (calc_adj && adj_iters && ne) SA_CUDA_P(cudaMemcpyAsync(adj_iters, d_ai.p, ne * sizeof(int), cudaMemcpyDeviceToHost, st));
    rc = plan_worst_status(P, st);
    return done(rc);
#undef SA_CUDA_P
}

// Single-solve drop-ins reuse the batch engine with one event.
namespace {
int single_solve(sa_ctx* ctx, int precision, int nx, int ny, const double* xx_deg,
                 const double* yy_deg, const double* spha, const double* sphb,
                 const double* sphc, const double* fun_or_T, double x0, double y0, int nr,
                 const double* xrec, const double* yrec, const double* sadj, bool adjoint,
                 double* out, int* niter) {
    if (!ctx) return SA_ERR_ARG;
    if (nx < 3 || ny < 3) return fail(ctx, SA_ERR_ARG, "Grid must be at least 3x3");
    if (!xx_deg || !yy_deg || !spha || !sphb || !sphc || !fun_or_T || !out)
        return fail(ctx, SA_ERR_ARG, "null input");
    if (nr < 0 || (nr > 0 && (!xrec || !yrec || !sadj))) return fail(ctx, SA_ERR_ARG, "receivers");
    const size_t n = (size_t)nx * ny;
    std::vector<int> rp = {0, nr}, ri(std::max(nr, 1));
    for (int i = 0; i < nr; i++) ri[i] = i;
    const int iper = 0;
    sa_plan* P = nullptr;
    int rc = sa_plan_create(ctx, precision, nx, ny, 1, xx_deg, yy_deg, 1, &x0, &y0, &iper,
                            rp.data(), ri.data(), nr, nr ? xrec : nullptr, nr ? yrec : nullptr, &P);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    DArr<double> m11, m12, m22, svel, fin, o, sa_, ones, tt;
    DArr<int> it, stt;
    std::vector<double> neg(n);
    for (size_t k = 0; k < n; k++) neg[k] = -sphc[k];    // media uses sphc = -m12
    auto done = [&](int code) {
        delete P;
        return code;
    };
    auto chk = [&](cudaError_t e) { return e == cudaSuccess ? 0 : fail(ctx, SA_ERR_CUDA, cudaGetErrorString(e)); };
    if ((rc = chk(m11.upload(spha, n, st))) || (rc = chk(m12.upload(neg.data(), n, st))) ||
        (rc = chk(m22.upload(sphb, n, st))) || (rc = chk(fin.upload(fun_or_T, n, st))) ||
        (rc = chk(o.alloc(n))) || (rc = chk(it.alloc(1))) || (rc = chk(stt.alloc(1))) ||
        (rc = chk(svel.alloc(n))) || (rc = chk(cudaMemsetAsync(svel.p, 0, n * sizeof(double), st))))
        return done(rc);
    if (nr && (rc = chk(sa_.upload(sadj, nr, st)))) return done(rc);
    // media planes from spha/sphb/sphc; the slowness plane is set directly
    rc = plan_media(P, svel.p, m11.p, m12.p, m22.p, true, st);
    if (rc) return done(rc);
    if ((rc = chk(cudaMemcpyAsync(P->fun64.p, fin.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st))))
        return done(rc);
    if (precision == SA_FP32 &&
        (rc = chk(launch_media32(nx, ny, 1, P->fun64.p, P->mt64.p, P->fun32.p, P->mt32.p, st))))
        return done(rc);
    BatchDesc d = plan_desc(P, true);
    d.ev.sadj = sa_.p;
    d.ev.T_in = fin.p;
    d.out.status = stt.p;
    if (adjoint) {
        d.mode = MODE_ADJ_ONLY;
        d.out.Ta_out = o.p;
        d.out.adj_iters = it.p;
    } else {
        d.mode = MODE_FWD;
        d.out.T_out = o.p;
        d.out.fwd_iters = it.p;
        std::vector<double> z(std::max(nr, 1), 0.0);
        if ((rc = chk(tt.upload(z.data(), std::max(nr, 1), st))) ||
            (rc = chk(ones.upload(z.data(), std::max(nr, 1), st))))
            return done(rc);
        d.ev.tt_obs = tt.p;
        d.ev.weight = ones.p;
    }
    if ((rc = chk(cudaMemsetAsync(P->queue.p, 0, sizeof(unsigned int), st)))) return done(rc);
    if ((rc = chk(precision == SA_FP64 ? launch_batch64(d, st) : launch_batch32(d, st))))
        return done(rc);
    int h_it = 0, h_st = 0;
    if ((rc = chk(cudaMemcpyAsync(out, o.p, n * sizeof(double), cudaMemcpyDeviceToHost, st))) ||
        (rc = chk(cudaMemcpyAsync(&h_it, it.p, sizeof(int), cudaMemcpyDeviceToHost, st))) ||
        (rc = chk(cudaMemcpyAsync(&h_st, stt.p, sizeof(int), cudaMemcpyDeviceToHost, st))) ||
        (rc = chk(cudaStreamSynchronize(st))))
        return done(rc);
    if (niter) *niter = h_it;
    if (h_st == ST_NOCONV) return done(fail(ctx, SA_ERR_NOCONV, "iteration cap reached"));
    if (h_st == ST_NONFINITE) return done(fail(ctx, SA_ERR_NONFINITE, "non-finite field"));
    return done(SA_OK);
}
}  // namespace

extern "C" int sa_eik_fwd_field(sa_ctx* ctx, int precision, int nx, int ny, const double* xx_deg,
                                const double* yy_deg, const double* spha, const double* sphb,
                                const double* sphc, const double* fun, double x0_deg,
                                double y0_deg, double* T_out, int* niter) {
    return single_solve(ctx, precision, nx, ny, xx_deg, yy_deg, spha, sphb, sphc, fun, x0_deg,
                        y0_deg, 0, nullptr, nullptr, nullptr, false, T_out, niter);
}

extern "C" int sa_eik_adj_field(sa_ctx* ctx, int precision, int nx, int ny, const double* xx_deg,
                                const double* yy_deg, const double* spha, const double* sphb,
                                const double* sphc, const double* T, int nr,
                                const double* xrec_deg, const double* yrec_deg,
                                const double* source_adj, double* Ta_out, int* niter) {
    return single_solve(ctx, precision, nx, ny, xx_deg, yy_deg, spha, sphb, sphc, T, 0.0, 0.0,
                        nr, xrec_deg, yrec_deg, source_adj, true, Ta_out, niter);
}

// ---------------------------------------------------------------------------
// Dispersion, depth kernels and kernel combination
// ---------------------------------------------------------------------------
namespace {
const void* layer_const_dev(sa_ctx* ctx, int nz, const double* zgrid, int* rc) {
    *rc = SA_OK;
    LayerConstCache& g_lc = ctx->lc;
    if (g_lc.nz == nz && std::equal(g_lc.z.begin(), g_lc.z.end(), zgrid)) return g_lc.dev.p;
    std::vector<unsigned char> h(layer_const_bytes());
    if (build_layer_const(nz, zgrid, h.data()) != 0) {
        *rc = fail(ctx, SA_ERR_ARG, "nz + 1 exceeds the supported layer count (64)");
        return nullptr;
    }
    cudaError_t e = g_lc.dev.upload(h.data(), h.size(), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        *rc = fail(ctx, SA_ERR_CUDA, cudaGetErrorString(e));
        return nullptr;
    }
    g_lc.nz = nz;
    g_lc.z.assign(zgrid, zgrid + nz);
    return g_lc.dev.p;
}

const double* periods_dev(sa_ctx* ctx, int nper, const double* periods, int* rc) {
    *rc = SA_OK;
    PeriodCache& g_pc = ctx->pc;
    if ((int)g_pc.p.size() == nper && std::equal(g_pc.p.begin(), g_pc.p.end(), periods))
        return g_pc.dev.p;
    cudaError_t e = g_pc.dev.upload(periods, nper, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        *rc = fail(ctx, SA_ERR_CUDA, cudaGetErrorString(e));
        return nullptr;
    }
    g_pc.p.assign(periods, periods + nper);
    return g_pc.dev.p;
}
}  // namespace

extern "C" int sa_surfdisp_columns(sa_ctx* ctx, int nx, int ny, int nz, const double* zgrid,
                                   const double* vs3d, int nper, const double* periods,
                                   int iwave, int igr, double* svel, int* status, void* stream) {
    if (!ctx) return SA_ERR_ARG;
    if (nx < 1 || ny < 1 || nz < 2 || nper < 1 || nper > 64 || !zgrid || !periods || !vs3d || !svel)
        return fail(ctx, SA_ERR_ARG, "sa_surfdisp_columns: bad sizes or null pointers");
    if (iwave != 1 && iwave != 2)
        return fail(ctx, SA_ERR_ARG, "iwave must be 1 (Love) or 2 (Rayleigh)");
    SA_CUDA(cudaSetDevice(ctx->device));
    int rc = SA_OK;
    const void* L = layer_const_dev(ctx, nz, zgrid, &rc);
    if (rc) return rc;
    const double* p = periods_dev(ctx, nper, periods, &rc);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    SA_CUDA(launch_surfdisp_columns(nx, ny, nz, vs3d, nper, p, 1, iwave, igr, L, svel, status, st));
    return SA_OK;
}

extern "C" int sa_depthkernel_columns(sa_ctx* ctx, int nx, int ny, int nz, const double* zgrid,
                                      const double* vs3d, int nper, const double* periods,
                                      const double* cp, double* sen_vs, double* sen_vp,
                                      double* sen_rho, void* stream) {
    if (!ctx) return SA_ERR_ARG;
    if (nx < 1 || ny < 1 || nz < 2 || nper < 1 || nper > 64 || !zgrid || !periods || !vs3d ||
        !cp || !sen_vs || !sen_vp || !sen_rho)
        return fail(ctx, SA_ERR_ARG, "sa_depthkernel_columns: bad sizes or null pointers");
    SA_CUDA(cudaSetDevice(ctx->device));
    int rc = SA_OK;
    const void* L = layer_const_dev(ctx, nz, zgrid, &rc);
    if (rc) return rc;
    const double* p = periods_dev(ctx, nper, periods, &rc);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    SA_CUDA(launch_depthkernel(nx, ny, nz, vs3d, nper, p, cp, L, sen_vs, sen_vp, sen_rho, st));
    return SA_OK;
}

extern "C" int sa_depthkernel_columns_group(sa_ctx* ctx, int nx, int ny, int nz,
                                            const double* zgrid, const double* vs3d, int nper,
                                            const double* periods, double* sen_vs,
                                            double* sen_vp, double* sen_rho, int* status,
                                            void* stream) {
    if (!ctx) return SA_ERR_ARG;
    if (nx < 1 || ny < 1 || nz < 2 || nper < 1 || nper > 64 || !zgrid || !periods || !vs3d ||
        !sen_vs || !sen_vp || !sen_rho)
        return fail(ctx, SA_ERR_ARG, "sa_depthkernel_columns_group: bad sizes or null pointers");
    SA_CUDA(cudaSetDevice(ctx->device));
    int rc = SA_OK;
    const void* L = layer_const_dev(ctx, nz, zgrid, &rc);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    // periods t(1 +- 0.5*0.01) (src/surfdisp.cpp:223-228)
    const double dt = 0.01;
    std::vector<double> t3(3 * (size_t)nper);
    for (int i = 0; i < nper; ++i) {
        t3[i] = periods[i];
        t3[nper + i] = periods[i] * (1.0 + 0.5 * dt);
        t3[2 * nper + i] = periods[i] * (1.0 - 0.5 * dt);
    }
    const size_t plane = (size_t)nx * ny * nper;
    DArr<double> dper, cps;
    DArr<int> st3;
    SA_CUDA(dper.upload(t3.data(), t3.size(), st));
    SA_CUDA(cps.alloc(3 * plane));
    SA_CUDA(st3.alloc(3 * (size_t)nx * ny));
    for (int k = 0; k < 3; k++)
        SA_CUDA(launch_surfdisp_columns(nx, ny, nz, vs3d, nper, dper.p + k * nper, 1, 2, 0, L,
                                        cps.p + k * plane, st3.p + k * (size_t)nx * ny, st));
    SA_CUDA(launch_depthkernel_group(nx, ny, nz, vs3d, nper, dper.p, dper.p + nper,
                                     dper.p + 2 * nper, cps.p, cps.p + plane, cps.p + 2 * plane, L,
                                     sen_vs, sen_vp, sen_rho, st));
    std::vector<int> hs(3 * (size_t)nx * ny);
    SA_CUDA(cudaMemcpyAsync(hs.data(), st3.p, hs.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    SA_CUDA(cudaStreamSynchronize(st));
    int bad = 0;
    for (size_t c = 0; c < (size_t)nx * ny; c++) {
        const int v = hs[c] | hs[(size_t)nx * ny + c] | hs[2 * (size_t)nx * ny + c];
        if (status) status[c] = v;
        bad |= v;
    }
    if (bad) return fail(ctx, SA_ERR_NOROOT, "Dispersion calculation failed");
    return SA_OK;
}

extern "C" int sa_depthkernel_columns_love(sa_ctx* ctx, int nx, int ny, int nz,
                                           const double* zgrid, const double* vs3d, int nper,
                                           const double* periods, int igr, double* sen_vs,
                                           double* sen_rho, int* status, void* stream) {
    if (!ctx) return SA_ERR_ARG;
    if (nx < 1 || ny < 1 || nz < 2 || nper < 1 || nper > 64 || !zgrid || !periods || !vs3d ||
        !sen_vs || !sen_rho || (igr != 0 && igr != 1))
        return fail(ctx, SA_ERR_ARG, "sa_depthkernel_columns_love: bad sizes, igr or pointers");
    SA_CUDA(cudaSetDevice(ctx->device));
    int rc = SA_OK;
    const void* L = layer_const_dev(ctx, nz, zgrid, &rc);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    // periods t(1 +- 0.5*0.01) (src/surfdisp.cpp:361-366)
    const double dt = 0.01;
    std::vector<double> t3(3 * (size_t)nper);
    for (int i = 0; i < nper; ++i) {
        t3[i] = periods[i];
        t3[nper + i] = periods[i] * (1.0 + 0.5 * dt);
        t3[2 * nper + i] = periods[i] * (1.0 - 0.5 * dt);
    }
    const int nrun = igr ? 3 : 1;
    const size_t plane = (size_t)nx * ny * nper, ncol = (size_t)nx * ny;
    DArr<double> dper, cps;
    DArr<int> st3;
    SA_CUDA(dper.upload(t3.data(), t3.size(), st));
    SA_CUDA(cps.alloc(3 * plane));
    SA_CUDA(st3.alloc(3 * ncol));
    SA_CUDA(cudaMemsetAsync(st3.p, 0, 3 * ncol * sizeof(int), st));
    for (int k = 0; k < nrun; k++)   // Love phase velocities (iwave 1)
        SA_CUDA(launch_surfdisp_columns(nx, ny, nz, vs3d, nper, dper.p + k * nper, 1, 1, 0, L,
                                        cps.p + k * plane, st3.p + k * ncol, st));
    SA_CUDA(launch_depthkernel_love(nx, ny, nz, vs3d, nper, dper.p, dper.p + nper,
                                    dper.p + 2 * nper, cps.p, cps.p + plane, cps.p + 2 * plane,
                                    igr, L, sen_vs, sen_rho, st));
    std::vector<int> hs(3 * ncol);
    SA_CUDA(cudaMemcpyAsync(hs.data(), st3.p, hs.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    SA_CUDA(cudaStreamSynchronize(st));
    int bad = 0;
    for (size_t c = 0; c < ncol; c++) {
        const int v = hs[c] | hs[ncol + c] | hs[2 * ncol + c];
        if (status) status[c] = v;
        bad |= v;
    }
    if (bad) return fail(ctx, SA_ERR_NOROOT, "Dispersion calculation failed");
    return SA_OK;
}

extern "C" int sa_combine_kernels_vs(sa_ctx* ctx, int nx, int ny, int nz, int nper,
                                     const double* adj_s, const double* vs3d, const double* vp3d,
                                     const double* sen_vs, const double* sen_vp,
                                     const double* sen_rho, double* ker_vs, void* stream) {
    if (!ctx) return SA_ERR_ARG;
    if (nx < 1 || ny < 1 || nz < 1 || nper < 1 || !adj_s || !vs3d || !sen_vs ||
        !sen_vp || !sen_rho || !ker_vs)
        return fail(ctx, SA_ERR_ARG, "sa_combine_kernels_vs: bad sizes or null pointers");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    SA_CUDA(launch_combine_vs(nx, ny, nz, nper, adj_s, vs3d, vp3d, sen_vs, sen_vp, sen_rho, ker_vs, st));
    return SA_OK;
}

// ---- one misfit-gradient evaluation ------------------------------------------

struct sa_grad {
    sa_plan* plan = nullptr;
    int nz = 0;
    DArr<unsigned char> lc;
    DArr<double> periods, svel, adj_s, sen_vs, sen_vp, sen_rho;
    DArr<double> sen_hs;     // half-space layer kernels (derivative convention)
    DArr<double> dcdvs;      // exact dc/dvs per node (convention 2)
    DArr<double> area;       // [ny] cell area dx R cos(lat) dy R, km^2
    DArr<int> colst, worst;
    // data type: 0 Rayleigh phase, 1 Rayleigh group (sa_grad_set_data_type).
    // Group data: svel are group velocities; the depth kernels come from the
    // phase velocities at t, t(1 + 0.005), t(1 - 0.005) (per3, cps3) and
    // sregnpu; colst then holds 4 status planes (group, 3 phase runs)
    int igr = 0;
    int iwave = 2;           // 2 Rayleigh, 1 Love (sa_grad_set_wave_type)
    DArr<double> per3, cps3;
    bool kden = false;       // is_kden (sa_grad_set_kden): kden_s accumulated per run
    DArr<double> kden_s;
    cudaStream_t side = nullptr;
    cudaEvent_t e_disp = nullptr, e_sen = nullptr;
    ~sa_grad() {
        if (e_disp) cudaEventDestroy(e_disp);
        if (e_sen) cudaEventDestroy(e_sen);
        if (side) cudaStreamDestroy(side);
    }
};

extern "C" int sa_grad_create(sa_plan* plan, int nz, const double* zgrid, const double* periods,
                              sa_grad** out) {
    if (!plan || !out) return SA_ERR_ARG;
    *out = nullptr;
    sa_ctx* ctx = plan->ctx;
    const int nper = plan->nper;
    if (nz < 2 || nper > 64 || !zgrid || !periods)
        return fail(ctx, SA_ERR_ARG, "sa_grad_create: nz >= 2, nper <= 64, zgrid and periods");
    SA_CUDA(cudaSetDevice(ctx->device));
    std::vector<unsigned char> h(layer_const_bytes());
    if (build_layer_const(nz, zgrid, h.data()) != 0)
        return fail(ctx, SA_ERR_ARG, "nz + 1 exceeds the supported layer count (64)");
    sa_grad* g = new sa_grad();
    g->plan = plan;
    g->nz = nz;
    const size_t ncol = (size_t)plan->nx * plan->ny, n4 = ncol * nz * nper;
    cudaError_t e = g->lc.upload(h.data(), h.size(), ctx->stream);
    if (e == cudaSuccess) e = g->periods.upload(periods, nper, ctx->stream);
    if (e == cudaSuccess) e = g->svel.alloc(ncol * nper);
    if (e == cudaSuccess) e = g->adj_s.alloc(ncol * nper);
    if (e == cudaSuccess) e = g->sen_vs.alloc(n4);
    if (e == cudaSuccess) e = g->sen_vp.alloc(n4);
    if (e == cudaSuccess) e = g->sen_rho.alloc(n4);
    if (e == cudaSuccess) e = g->colst.alloc(ncol);
    if (e == cudaSuccess) e = g->worst.alloc(1);
    if (e == cudaSuccess) {
        std::vector<double> yr(plan->ny), area(plan->ny);
        e = cudaMemcpy(yr.data(), plan->yy.p, plan->ny * sizeof(double), cudaMemcpyDeviceToHost);
        for (int i = 0; i < plan->ny; i++)
            area[i] = plan->dx * R_EARTH * std::cos(yr[i]) * plan->dy * R_EARTH;
        if (e == cudaSuccess) e = g->area.upload(area.data(), plan->ny, ctx->stream);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->e_disp, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->e_sen, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        delete g;
        return fail(ctx, e == cudaErrorMemoryAllocation ? SA_ERR_NOMEM : SA_ERR_CUDA,
                    std::string("sa_grad_create: ") + cudaGetErrorString(e));
    }
    *out = g;
    return SA_OK;
}

extern "C" void sa_grad_destroy(sa_grad* g) {
    if (!g) return;
    cudaSetDevice(g->plan->ctx->device);
    delete g;
}

namespace {
// The data type's velocities (phase or group) into svel, column statuses
// into g->colst, on `st`.
int grad_velocities(sa_grad* g, const double* vs3d, double* svel, cudaStream_t st) {
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    SA_CUDA(launch_surfdisp_columns(P->nx, P->ny, g->nz, vs3d, P->nper, g->periods.p, 1,
                                    g->iwave, g->igr, g->lc.p, svel, g->colst.p, st));
    return SA_OK;
}
// The data type's depth kernels on `st` (phase: sregn96_hti at svel; group:
// three phase-velocity runs and sregnpu), sen_hs optional (phase only).
int grad_depth_kernels(sa_grad* g, const double* vs3d, const double* svel, double* sen_hs,
                       cudaStream_t st) {
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    const int nx = P->nx, ny = P->ny, nz = g->nz, nper = P->nper;
    if (g->igr == 0) {
        if (g->iwave == 1)   // SurfGrid::compute_dispersion_kernel sends phase data to
            return fail(ctx, SA_ERR_ARG,   // depthkernelHTI1d, which takes Rayleigh only
                        "Love phase-velocity data: the reference's kernels are Rayleigh only "
                        "(src/surf_grid.cpp:282-286, src/surfdisp.cpp:484-487)");
        SA_CUDA(launch_depthkernel(nx, ny, nz, vs3d, nper, g->periods.p, svel, g->lc.p,
                                   g->sen_vs.p, g->sen_vp.p, g->sen_rho.p, st, sen_hs));
        return SA_OK;
    }
    const size_t plane = (size_t)nx * ny * nper, ncol = (size_t)nx * ny;
    for (int k = 0; k < 3; k++)
        SA_CUDA(launch_surfdisp_columns(nx, ny, nz, vs3d, nper, g->per3.p + k * nper, 1,
                                        g->iwave, 0, g->lc.p, g->cps3.p + k * plane,
                                        g->colst.p + (k + 1) * ncol, st));
    if (g->iwave == 1) {   // Love group kernels (no vp kernel)
        SA_CUDA(launch_depthkernel_love(nx, ny, nz, vs3d, nper, g->per3.p, g->per3.p + nper,
                                        g->per3.p + 2 * nper, g->cps3.p, g->cps3.p + plane,
                                        g->cps3.p + 2 * plane, 1, g->lc.p, g->sen_vs.p,
                                        g->sen_rho.p, st));
        SA_CUDA(cudaMemsetAsync(g->sen_vp.p, 0, plane * nz * sizeof(double), st));
        return SA_OK;
    }
    SA_CUDA(launch_depthkernel_group(nx, ny, nz, vs3d, nper, g->per3.p, g->per3.p + nper,
                                     g->per3.p + 2 * nper, g->cps3.p, g->cps3.p + plane,
                                     g->cps3.p + 2 * plane, g->lc.p, g->sen_vs.p, g->sen_vp.p,
                                     g->sen_rho.p, st));
    return SA_OK;
}
int grad_ncolst(const sa_grad* g) {
    return (g->igr ? 4 : 1) * g->plan->nx * g->plan->ny;
}
}  // namespace

extern "C" int sa_grad_set_wave_type(sa_grad* g, int iwave) {
    if (!g) return SA_ERR_ARG;
    sa_ctx* ctx = g->plan->ctx;
    if (iwave != 1 && iwave != 2) return fail(ctx, SA_ERR_ARG, "wave type: 1 Love, 2 Rayleigh");
    g->iwave = iwave;
    return SA_OK;
}

extern "C" int sa_grad_set_data_type(sa_grad* g, int igr) {
    if (!g) return SA_ERR_ARG;
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    if (igr != 0 && igr != 1) return fail(ctx, SA_ERR_ARG, "data type: 0 phase, 1 group");
    SA_CUDA(cudaSetDevice(ctx->device));
    const int nper = P->nper;
    const size_t ncol = (size_t)P->nx * P->ny;
    if (igr == 1) {
        std::vector<double> hp(nper), t3(3 * (size_t)nper);
        SA_CUDA(cudaMemcpy(hp.data(), g->periods.p, nper * sizeof(double), cudaMemcpyDeviceToHost));
        const double dt = 0.01;   // src/surfdisp.cpp:223-228
        for (int i = 0; i < nper; ++i) {
            t3[i] = hp[i];
            t3[nper + i] = hp[i] * (1.0 + 0.5 * dt);
            t3[2 * nper + i] = hp[i] * (1.0 - 0.5 * dt);
        }
        SA_CUDA(g->per3.upload(t3.data(), t3.size(), ctx->stream));
        SA_CUDA(g->cps3.alloc(3 * ncol * nper));
        SA_CUDA(g->colst.alloc(4 * ncol));
        SA_CUDA(cudaMemsetAsync(g->colst.p, 0, 4 * ncol * sizeof(int), ctx->stream));
        SA_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    g->igr = igr;
    return SA_OK;
}

extern "C" int sa_grad_set_kden(sa_grad* g, int enable) {
    if (!g) return SA_ERR_ARG;
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    SA_CUDA(cudaSetDevice(ctx->device));
    if (enable) SA_CUDA(g->kden_s.alloc((size_t)P->nx * P->ny * P->nper));
    g->kden = enable != 0;
    return sa_plan_kden_output(P, g->kden ? g->kden_s.p : nullptr);
}

extern "C" int sa_grad_ker_den(sa_grad* g, const double* vs3d, const double* vp3d,
                               double* ker_den, void* stream) {
    if (!g) return SA_ERR_ARG;
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    if (!g->kden) return fail(ctx, SA_ERR_ARG, "kernel density not enabled (sa_grad_set_kden)");
    if (!vs3d || !ker_den) return fail(ctx, SA_ERR_ARG, "vs3d and ker_den are required");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    SA_CUDA(cudaStreamWaitEvent(st, g->e_sen, 0));
    // preproc::combine_kernels' ker_den (src/preproc.cpp:294-300)
    SA_CUDA(launch_combine_vs(P->nx, P->ny, g->nz, P->nper, g->kden_s.p, vs3d, vp3d,
                              g->sen_vs.p, g->sen_vp.p, g->sen_rho.p, ker_den, st));
    return SA_OK;
}

extern "C" int sa_grad_run(sa_grad* g, const double* vs3d, const double* vp3d,
                           const double* tt_obs, const double* weight, double* ker_vs,
                           double* chi, double* svel_out, double* adj_s_out, int* status,
                           void* stream) {
    if (!g) return SA_ERR_ARG;
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    if (!vs3d || !ker_vs || !chi) return fail(ctx, SA_ERR_ARG, "vs3d, ker_vs and chi are required");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const int nx = P->nx, ny = P->ny, nz = g->nz, nper = P->nper;
    double* svel = svel_out ? svel_out : g->svel.p;
    double* adj_s = adj_s_out ? adj_s_out : g->adj_s.p;
    // SurfGrid::fwdsurf (Rayleigh phase or group velocities, spherical earth)
    int rc = grad_velocities(g, vs3d, svel, st);
    if (rc) return rc;
    SA_CUDA(cudaEventRecord(g->e_disp, st));
    // forward_for_event over every event (accumulates adj_s and the misfit)
    rc = sa_plan_forward_adjoint(P, svel, nullptr, nullptr, nullptr, tt_obs, weight, 1, nullptr,
                                 adj_s, chi, nullptr, nullptr, nullptr, st);
    if (rc) return rc;
    if (P->discrete) {
        // exact discrete adjoint (sa_plan_set_adjoint): adj_s = dchi/dsvel,
        // chained with the derivatives of the phase-velocity roots
        if (g->igr != 0 || g->iwave != 2)
            return fail(ctx, SA_ERR_ARG, "the exact gradient is for Rayleigh phase data");
        SA_CUDA(g->dcdvs.alloc((size_t)nx * ny * nz * nper));
        SA_CUDA(launch_dispersion_dcdvs(nx, ny, nz, vs3d, nper, g->periods.p, svel, g->lc.p,
                                        g->dcdvs.p, st));
        SA_CUDA(launch_combine_exact(nx, ny, nz, nper, adj_s, g->dcdvs.p, ker_vs, st));
        SA_CUDA(launch_grad_status(grad_ncolst(g), g->colst.p, P->worst.p,
                                   status ? status : g->worst.p, st));
        return SA_OK;
    }
    // compute_dispersion_kernel on a second stream: it needs only vs3d and the
    // velocities, so it runs while the event batch drains
    SA_CUDA(cudaStreamWaitEvent(g->side, g->e_disp, 0));
    rc = grad_depth_kernels(g, vs3d, svel, nullptr, g->side);
    if (rc) return rc;
    SA_CUDA(cudaEventRecord(g->e_sen, g->side));
    SA_CUDA(cudaStreamWaitEvent(st, g->e_sen, 0));
    // combine_kernels (vs-only parametrisation)
    SA_CUDA(launch_combine_vs(nx, ny, nz, nper, adj_s, vs3d, vp3d, g->sen_vs.p, g->sen_vp.p,
                              g->sen_rho.p, ker_vs, st));
    SA_CUDA(launch_grad_status(grad_ncolst(g), g->colst.p, P->worst.p,
                               status ? status : g->worst.p, st));
    return SA_OK;
}

extern "C" int sa_grad_forward(sa_grad* g, const double* vs3d, double* syn, double* svel_out,
                               int* status, void* stream) {
    if (!g) return SA_ERR_ARG;
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    if (!vs3d || !syn) return fail(ctx, SA_ERR_ARG, "vs3d and syn are required");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const int nx = P->nx, ny = P->ny, nz = g->nz, nper = P->nper;
    double* svel = svel_out ? svel_out : g->svel.p;
    (void)nz;
    (void)nper;
    int rc = grad_velocities(g, vs3d, svel, st);
    if (rc) return rc;
    // forward only: tt_obs / weight are not read (no residuals)
    rc = plan_run(P, svel, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, syn, nullptr,
                  nullptr, nullptr, nullptr, nullptr, st);
    if (rc) return rc;
    SA_CUDA(launch_grad_status(nx * ny, g->colst.p, P->worst.p, status ? status : g->worst.p, st));
    return SA_OK;
}

extern "C" int sa_grad_vjp(sa_grad* g, const double* vs3d, const double* vp3d,
                           const double* source_adj, int convention, double* grad,
                           double* svel_out, double* adj_s_out, int* status, void* stream) {
    if (!g) return SA_ERR_ARG;
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    if (!vs3d || !grad || (P->npair > 0 && !source_adj))
        return fail(ctx, SA_ERR_ARG, "vs3d, source_adj and grad are required");
    if (convention < 0 || convention > 2) return fail(ctx, SA_ERR_ARG, "convention 0, 1 or 2");
    if (convention >= 1 && (g->igr != 0 || g->iwave != 2))
        return fail(ctx, SA_ERR_ARG, "conventions 1 and 2 are for Rayleigh phase data");
    if ((convention == 2) != (P->discrete == 1))
        return fail(ctx, SA_ERR_ARG,
                    "convention 2 goes with the exact discrete adjoint (sa_plan_set_adjoint)");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const int nx = P->nx, ny = P->ny, nz = g->nz, nper = P->nper;
    double* svel = svel_out ? svel_out : g->svel.p;
    double* adj_s = adj_s_out ? adj_s_out : g->adj_s.p;
    if (convention == 2) {
        // the exact gradient of the discrete forward model: fwdsurf, every
        // forward field to a fixed point, the discrete adjoint (adj_s =
        // dchi/dsvel), the derivatives of the phase-velocity roots
        SA_CUDA(g->dcdvs.alloc((size_t)nx * ny * nz * nper));
        int rc = grad_velocities(g, vs3d, svel, st);
        if (rc) return rc;
        rc = plan_run(P, svel, nullptr, nullptr, nullptr, nullptr, nullptr, source_adj, 1,
                      nullptr, adj_s, nullptr, nullptr, nullptr, nullptr, st);
        if (rc) return rc;
        SA_CUDA(launch_dispersion_dcdvs(nx, ny, nz, vs3d, nper, g->periods.p, svel, g->lc.p,
                                        g->dcdvs.p, st));
        SA_CUDA(launch_combine_exact(nx, ny, nz, nper, adj_s, g->dcdvs.p, grad, st));
        SA_CUDA(launch_grad_status(grad_ncolst(g), g->colst.p, P->worst.p,
                                   status ? status : g->worst.p, st));
        return SA_OK;
    }
    if (convention == 1) SA_CUDA(g->sen_hs.alloc((size_t)nx * ny * nper * 3));
    int rc = grad_velocities(g, vs3d, svel, st);
    if (rc) return rc;
    SA_CUDA(cudaEventRecord(g->e_disp, st));
    // every forward field recomputed, the adjoint driven by source_adj
    rc = plan_run(P, svel, nullptr, nullptr, nullptr, nullptr, nullptr, source_adj, 1, nullptr,
                  adj_s, nullptr, nullptr, nullptr, nullptr, st);
    if (rc) return rc;
    SA_CUDA(cudaStreamWaitEvent(g->side, g->e_disp, 0));
    rc = grad_depth_kernels(g, vs3d, svel, convention == 1 ? g->sen_hs.p : nullptr, g->side);
    if (rc) return rc;
    SA_CUDA(cudaEventRecord(g->e_sen, g->side));
    SA_CUDA(cudaStreamWaitEvent(st, g->e_sen, 0));
    if (convention == 0)
        SA_CUDA(launch_combine_vs(nx, ny, nz, nper, adj_s, vs3d, vp3d, g->sen_vs.p, g->sen_vp.p,
                                  g->sen_rho.p, grad, st));
    else
        SA_CUDA(launch_combine_vs_derivative(nx, ny, nz, nper, adj_s, vs3d, vp3d, g->sen_vs.p,
                                             g->sen_vp.p, g->sen_rho.p, g->sen_hs.p, g->area.p,
                                             g->lc.p, grad, st));
    SA_CUDA(launch_grad_status(grad_ncolst(g), g->colst.p, P->worst.p,
                               status ? status : g->worst.p, st));
    return SA_OK;
}

extern "C" int sa_grad_root_derivatives(sa_grad* g, const double* vs3d, double* dcdvs,
                                        void* stream) {
    if (!g) return SA_ERR_ARG;
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    if (!vs3d || !dcdvs) return fail(ctx, SA_ERR_ARG, "vs3d and dcdvs are required");
    if (g->igr != 0 || g->iwave != 2)
        return fail(ctx, SA_ERR_ARG, "root derivatives are for Rayleigh phase velocities");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    int rc = grad_velocities(g, vs3d, g->svel.p, st);
    if (rc) return rc;
    SA_CUDA(launch_dispersion_dcdvs(P->nx, P->ny, g->nz, vs3d, P->nper, g->periods.p, g->svel.p,
                                    g->lc.p, dcdvs, st));
    return SA_OK;
}

extern "C" int sa_grad_sen(sa_grad* g, double* sen_vs, double* sen_vp, double* sen_rho,
                           void* stream) {
    if (!g) return SA_ERR_ARG;
    sa_ctx* ctx = g->plan->ctx;
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const size_t bytes = (size_t)g->plan->nx * g->plan->ny * g->nz * g->plan->nper * sizeof(double);
    double* dst[3] = {sen_vs, sen_vp, sen_rho};
    const double* src[3] = {g->sen_vs.p, g->sen_vp.p, g->sen_rho.p};
    for (int i = 0; i < 3; ++i)
        if (dst[i]) SA_CUDA(cudaMemcpyAsync(dst[i], src[i], bytes, cudaMemcpyDeviceToDevice, st));
    return SA_OK;
}

extern "C" int sa_grad_combine(sa_grad* g, const double* vs3d, const double* vp3d,
                               const double* adj_s, double* ker_vs, void* stream) {
    if (!g) return SA_ERR_ARG;
    sa_plan* P = g->plan;
    sa_ctx* ctx = P->ctx;
    if (!vs3d || !adj_s || !ker_vs) return fail(ctx, SA_ERR_ARG, "vs3d, adj_s and ker_vs are required");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    // the depth kernels of the last run were written on the side stream
    SA_CUDA(cudaStreamWaitEvent(st, g->e_sen, 0));
    SA_CUDA(launch_combine_vs(P->nx, P->ny, g->nz, P->nper, adj_s, vs3d, vp3d, g->sen_vs.p,
                              g->sen_vp.p, g->sen_rho.p, ker_vs, st));
    return SA_OK;
}

// ---- PostProc::pde_smooth ------------------------------------------------------

namespace {
constexpr double PI_D = 3.14159265358979323846264338327950288;   // include/config.h:54
constexpr double DEG2RAD_D = PI_D / 180.0;                         // include/config.h:68
}  // namespace

// Step count and diffusion coefficients of src/postproc.cpp:394-434.
extern "C" int sa_pde_smooth_nstep(int ny, double dx_deg, double dy_deg, double dz_km,
                                   const double* ygrid, double sigma_h, double sigma_v,
                                   int* nstep, double* ch_out, double* cv_out) {
    if (ny < 1 || !ygrid || !nstep) return SA_ERR_ARG;
    if (!(sigma_h > 0.0) || !(sigma_v > 0.0)) return SA_ERR_ARG;   // :397-400
    double lat_max = std::max(std::abs(ygrid[0]), std::abs(ygrid[ny - 1]));
    lat_max = std::min(lat_max, 89.0);
    const double cos2_lat_max = std::pow(std::cos(lat_max * DEG2RAD_D), 2);
    const double cmax_h = std::min(dx_deg * dx_deg * cos2_lat_max, dy_deg * dy_deg) / 6.0;
    const double cmax_v = dz_km * dz_km / 6.0;
    if (cmax_h <= 1e-12 || cmax_v <= 1e-12) return SA_ERR_ARG;   // :414-417
    const double dt = 1.0;
    const double nh = std::ceil(sigma_h * sigma_h / (2.0 * cmax_h * dt));
    const double nv = std::ceil(sigma_v * sigma_v / (2.0 * cmax_v * dt));
    if (!(nh < 2e9) || !(nv < 2e9)) return SA_ERR_ARG;
    const int ns = std::max({(int)nh, (int)nv, 1});
    *nstep = ns;
    if (ch_out) *ch_out = sigma_h * sigma_h / (2.0 * ns * dt);
    if (cv_out) *cv_out = sigma_v * sigma_v / (2.0 * ns * dt);
    return SA_OK;
}

extern "C" int sa_pde_smooth(sa_ctx* ctx, int nx, int ny, int nz, double dx_deg, double dy_deg,
                             double dz_km, const double* ygrid, const double* zgrid,
                             double sigma_h, double sigma_v, double* field, double* work,
                             int* nstep_out, void* stream) {
    if (!ctx) return SA_ERR_ARG;
    if (nx < 3 || ny < 3 || nz < 3 || !ygrid || !zgrid || !field)
        return fail(ctx, SA_ERR_ARG, "sa_pde_smooth: grid must be at least 3x3x3");
    int ns = 0;
    double ch = 0, cv = 0;
    if (sa_pde_smooth_nstep(ny, dx_deg, dy_deg, dz_km, ygrid, sigma_h, sigma_v, &ns, &ch, &cv))
        return fail(ctx, SA_ERR_ARG,
                    "Invalid sigma values or grid spacing for PDE-based smoothing");
    if (nstep_out) *nstep_out = ns;
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    // per-row and per-depth factors in the reference's evaluation order (:74-123)
    const double dx2_inv = 1.0 / (dx_deg * dx_deg);
    const double dy2_inv = 1.0 / (dy_deg * dy_deg);
    const double dz2_inv = 1.0 / (dz_km * dz_km);
    const double dy_inv_half = 1.0 / (2.0 * dy_deg);
    const double dz_inv_half = 1.0 / (2.0 * dz_km);
    std::vector<double> rowX(ny, 0.0), rowY(ny, 0.0), depE(nz, 0.0);
    for (int iy = 1; iy < ny - 1; ++iy) {
        const double lat_rad = (ygrid[0] + iy * dy_deg) * DEG2RAD_D;   // src/decomposer.cpp:116-118
        const double cos_lat = std::cos(lat_rad);
        const double dy2_corr_inv = 1.0 / (cos_lat * cos_lat);
        const double tan_lat = std::tan(lat_rad);
        rowX[iy] = ch * dx2_inv * dy2_corr_inv;
        rowY[iy] = ch * DEG2RAD_D * tan_lat * dy_inv_half;
    }
    for (int k = 0; k < nz; ++k) {
        const double r_inv = 2.0 / (R_EARTH - zgrid[k]);
        depE[k] = cv * r_inv * dz_inv_half;
    }
    DArr<double> d_rx, d_ry, d_de, d_work;
    SA_CUDA(d_rx.upload(rowX.data(), ny, st));
    SA_CUDA(d_ry.upload(rowY.data(), ny, st));
    SA_CUDA(d_de.upload(depE.data(), nz, st));
    double* w = work;
    if (!w) {
        SA_CUDA(d_work.alloc((size_t)nx * ny * nz));
        w = d_work.p;
    }
    SA_CUDA(launch_pde_smooth(nx, ny, nz, ch * dy2_inv, cv * dz2_inv, d_rx.p, d_ry.p, d_de.p, ns,
                              field, w, st));
    // the factor arrays (and an internal work array) are released on return
    SA_CUDA(cudaStreamSynchronize(st));
    return SA_OK;
}

// ---- optimizer (src/optimize.cpp, src/inversion.cpp:302-323, :465-490) -----------

namespace {
constexpr int LBFGS_STORE = 5;   // MAX_LBFGS_STORE, include/config.h:90

// Reduction helper: runs on `st`, waits, returns the scalar.
int reduce_to_host(sa_ctx* ctx, cudaError_t launched, double* scratch, double* out,
                   cudaStream_t st) {
    SA_CUDA(launched);
    SA_CUDA(cudaMemcpyAsync(out, scratch + reduce_scratch_doubles() - 1, sizeof(double),
                            cudaMemcpyDeviceToHost, st));
    SA_CUDA(cudaStreamSynchronize(st));
    return SA_OK;
}
}  // namespace

struct sa_lbfgs {
    sa_ctx* ctx = nullptr;
    size_t n = 0;
    // ring of the last LBFGS_STORE + 1 iterates: model (vs) and gradient
    DArr<double> model[LBFGS_STORE + 1], grad[LBFGS_STORE + 1];
    int stored_iter[LBFGS_STORE + 1];
    DArr<double> s[LBFGS_STORE], y[LBFGS_STORE], red;
};

extern "C" int sa_lbfgs_create(sa_ctx* ctx, size_t n, sa_lbfgs** out) {
    if (!ctx || !out || n == 0) return SA_ERR_ARG;
    *out = nullptr;
    SA_CUDA(cudaSetDevice(ctx->device));
    sa_lbfgs* L = new sa_lbfgs();
    L->ctx = ctx;
    L->n = n;
    for (int i = 0; i <= LBFGS_STORE; i++) L->stored_iter[i] = -1;
    cudaError_t e = L->red.alloc(reduce_scratch_doubles());
    if (e != cudaSuccess) {
        delete L;
        return fail(ctx, SA_ERR_NOMEM, "sa_lbfgs_create: device allocation failed");
    }
    *out = L;
    return SA_OK;
}

extern "C" void sa_lbfgs_destroy(sa_lbfgs* L) {
    if (!L) return;
    cudaSetDevice(L->ctx->device);
    delete L;
}

extern "C" int sa_lbfgs_store(sa_lbfgs* L, int iter, const double* model, const double* grad) {
    if (!L) return SA_ERR_ARG;
    sa_ctx* ctx = L->ctx;
    if (iter < 0 || !model || !grad) return fail(ctx, SA_ERR_ARG, "sa_lbfgs_store: arguments");
    SA_CUDA(cudaSetDevice(ctx->device));
    const int slot = iter % (LBFGS_STORE + 1);
    SA_CUDA(L->model[slot].alloc(L->n));
    SA_CUDA(L->grad[slot].alloc(L->n));
    SA_CUDA(cudaMemcpyAsync(L->model[slot].p, model, L->n * sizeof(double),
                            cudaMemcpyDeviceToDevice, ctx->stream));
    SA_CUDA(cudaMemcpyAsync(L->grad[slot].p, grad, L->n * sizeof(double),
                            cudaMemcpyDeviceToDevice, ctx->stream));
    SA_CUDA(cudaStreamSynchronize(ctx->stream));
    L->stored_iter[slot] = iter;
    return SA_OK;
}

extern "C" int sa_lbfgs_direction(sa_lbfgs* L, int iter, double* dir) {
    if (!L) return SA_ERR_ARG;
    sa_ctx* ctx = L->ctx;
    if (iter < 0 || !dir) return fail(ctx, SA_ERR_ARG, "sa_lbfgs_direction: arguments");
    const int nh = std::min(iter, LBFGS_STORE);   // src/optimize.cpp:153-154
    const int h0 = iter - nh;
    for (int k = h0; k <= iter; k++)
        if (L->stored_iter[k % (LBFGS_STORE + 1)] != k)
            return fail(ctx, SA_ERR_ARG, "sa_lbfgs_direction: iterate " + std::to_string(k) +
                                             " was not stored");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t n = L->n;
    auto M = [&](int k) { return L->model[k % (LBFGS_STORE + 1)].p; };
    auto G = [&](int k) { return L->grad[k % (LBFGS_STORE + 1)].p; };
    double rho[LBFGS_STORE] = {0}, alpha[LBFGS_STORE] = {0};
    int rc;
    for (int h = 0; h < nh; h++) {
        SA_CUDA(L->s[h].alloc(n));
        SA_CUDA(L->y[h].alloc(n));
        SA_CUDA(launch_lbfgs_pair(n, M(h0 + h), M(h0 + h + 1), G(h0 + h), G(h0 + h + 1),
                                  L->s[h].p, L->y[h].p, st));
        double sy = 0;
        if ((rc = reduce_to_host(ctx, launch_dot(n, L->s[h].p, L->y[h].p, L->red.p, st), L->red.p,
                                 &sy, st)))
            return rc;
        rho[h] = (sy > 0.0) ? (1.0 / sy) : 0.0;   // :203
    }
    // q <- g_iter
    SA_CUDA(cudaMemcpyAsync(dir, G(iter), n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    for (int h = nh - 1; h >= 0; --h) {   // :209-214
        double sq = 0;
        if ((rc = reduce_to_host(ctx, launch_dot(n, L->s[h].p, dir, L->red.p, st), L->red.p, &sq,
                                 st)))
            return rc;
        alpha[h] = rho[h] * sq;
        SA_CUDA(launch_axpy(n, 0, alpha[h], L->y[h].p, dir, st));
    }
    if (nh > 0) {   // :219-228
        double yy = 0, sy = 0;
        const int last = nh - 1;
        if ((rc = reduce_to_host(ctx, launch_dot(n, L->y[last].p, L->y[last].p, L->red.p, st),
                                 L->red.p, &yy, st)))
            return rc;
        if ((rc = reduce_to_host(ctx, launch_dot(n, L->s[last].p, L->y[last].p, L->red.p, st),
                                 L->red.p, &sy, st)))
            return rc;
        const double gamma = (sy > 0.0 && yy > 0.0) ? (sy / yy) : 1.0;
        SA_CUDA(launch_axpy(n, 1, gamma, nullptr, dir, st));
    }
    for (int h = 0; h < nh; ++h) {   // :231-236
        double yr = 0;
        if ((rc = reduce_to_host(ctx, launch_dot(n, L->y[h].p, dir, L->red.p, st), L->red.p, &yr,
                                 st)))
            return rc;
        const double beta = rho[h] * yr;
        SA_CUDA(launch_axpy(n, 2, alpha[h] - beta, L->s[h].p, dir, st));
    }
    SA_CUDA(cudaStreamSynchronize(st));
    return SA_OK;
}

namespace {
double* ctx_red(sa_ctx* ctx, int* rc) {
    cudaError_t e = ctx->red.alloc(reduce_scratch_doubles());
    *rc = e == cudaSuccess ? SA_OK : fail(ctx, SA_ERR_NOMEM, "reduction scratch");
    return ctx->red.p;
}
}  // namespace

extern "C" int sa_dot(sa_ctx* ctx, size_t n, const double* a, const double* b, double* out) {
    if (!ctx || !a || !b || !out) return SA_ERR_ARG;
    SA_CUDA(cudaSetDevice(ctx->device));
    int rc = SA_OK;
    double* red = ctx_red(ctx, &rc);
    if (rc) return rc;
    return reduce_to_host(ctx, launch_dot(n, a, b, red, ctx->stream), red, out, ctx->stream);
}

extern "C" int sa_kernel_precondition(sa_ctx* ctx, size_t n, const double* ker_den, double* ker,
                                      void* stream) {
    if (!ctx || !ker_den || !ker) return SA_ERR_ARG;
    SA_CUDA(cudaSetDevice(ctx->device));
    int rc = SA_OK;
    double* red = ctx_red(ctx, &rc);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    SA_CUDA(launch_kernel_precondition(n, ker_den, red, ker, st));
    return SA_OK;
}

extern "C" int sa_grad_normalization(sa_ctx* ctx, size_t n, double* g, double* max_out) {
    if (!ctx || !g) return SA_ERR_ARG;
    SA_CUDA(cudaSetDevice(ctx->device));
    int rc = SA_OK;
    double* red = ctx_red(ctx, &rc);
    if (rc) return rc;
    double m = 0;
    if ((rc = reduce_to_host(ctx, launch_absmax(n, g, red, ctx->stream), red, &m, ctx->stream)))
        return rc;
    if (max_out) *max_out = m;
    if (m < 2.220446049250313e-16) return SA_OK;   // REAL_EPS guard, src/inversion.cpp:316
    SA_CUDA(launch_axpy(n, 3, m, nullptr, g, ctx->stream));
    SA_CUDA(cudaStreamSynchronize(ctx->stream));
    return SA_OK;
}

extern "C" int sa_descent_angle(sa_ctx* ctx, size_t n, const double* dir, const double* grad,
                                double* deg) {
    if (!ctx || !dir || !grad || !deg) return SA_ERR_ARG;
    double d = 0, gg = 0, dd = 0;
    int rc;
    if ((rc = sa_dot(ctx, n, grad, dir, &d))) return rc;
    if ((rc = sa_dot(ctx, n, grad, grad, &gg))) return rc;
    if ((rc = sa_dot(ctx, n, dir, dir, &dd))) return rc;
    const double gn = std::sqrt(gg), dn = std::sqrt(dd);   // src/optimize.cpp:46-47
    if (gn < 2.220446049250313e-16 || dn < 2.220446049250313e-16) {
        *deg = 90.0;
        return SA_OK;
    }
    double c = d / (gn * dn);
    c = std::max(-1.0, std::min(1.0, c));
    *deg = std::acos(c) * (180.0 / PI_D);
    return SA_OK;
}

extern "C" int sa_wolfe_condition(double gd, double kd, double alpha, double* alpha_L,
                                  double* alpha_R, double f0, double f1, int subiter, double c1,
                                  double c2, int max_sub_niter, double alpha_init,
                                  double* next_alpha) {
    if (!alpha_L || !alpha_R || !next_alpha) return -1;
    const double q = -gd, q1 = -kd;   // src/optimize.cpp:86-89
    const bool armijo = f1 <= f0 + alpha * c1 * q;
    const bool curvature = q1 >= c2 * q;
    int status;
    if (armijo && curvature) {
        status = 0;
        *next_alpha = alpha;
    } else if (!armijo) {
        *alpha_R = alpha;
        *next_alpha = (*alpha_L + *alpha_R) * 0.5;
        status = 1;
    } else {
        *alpha_L = alpha;
        const double cand = (*alpha_R > 0.0) ? (*alpha_L + *alpha_R) * 0.5 : alpha * 2.0;
        if (cand > alpha_init) {
            *next_alpha = alpha_init;
            status = 0;
        } else {
            *next_alpha = cand;
            status = 1;
        }
    }
    if (status == 1 && subiter == max_sub_niter - 1) {
        status = 2;
        *next_alpha = alpha;
    }
    return status;
}

extern "C" int sa_model_update_vs(sa_ctx* ctx, size_t n, const double* vs, const double* dir,
                                  double alpha, double* vs_out, double* vp_out, double* rho_out,
                                  void* stream) {
    if (!ctx || !vs || !dir || !vs_out) return SA_ERR_ARG;
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    SA_CUDA(launch_model_update_vs(n, vs, dir, alpha, vs_out, vp_out, rho_out, st));
    return SA_OK;
}

// ---- topography (src/surf_grid.cpp:80-166, :307-354; src/topo.cpp:46-114) -------

extern "C" int sa_grid_topography(sa_ctx* ctx, int nx_raw, int ny_raw, const double* lon_raw,
                                  const double* lat_raw, const double* z_raw, int nx, int ny,
                                  const double* x, const double* y, double* z_out) {
    if (!ctx) return SA_ERR_ARG;
    if (nx_raw < 2 || ny_raw < 2 || nx < 2 || ny < 2 || !lon_raw || !lat_raw || !z_raw || !x ||
        !y || !z_out)
        return fail(ctx, SA_ERR_ARG, "sa_grid_topography: bad sizes or null pointers");
    // Topography::check_bounds (src/topo.cpp:68-95)
    const double lo0 = *std::min_element(lon_raw, lon_raw + nx_raw);
    const double lo1 = *std::max_element(lon_raw, lon_raw + nx_raw);
    const double la0 = *std::min_element(lat_raw, lat_raw + ny_raw);
    const double la1 = *std::max_element(lat_raw, lat_raw + ny_raw);
    if (*std::min_element(x, x + nx) < lo0 || *std::max_element(x, x + nx) > lo1 ||
        *std::min_element(y, y + ny) < la0 || *std::max_element(y, y + ny) > la1)
        return fail(ctx, SA_ERR_ARG, "Model grid extends beyond topography bounds");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    DArr<double> dxr, dyr, dzr, dx, dy;
    SA_CUDA(dxr.upload(lon_raw, nx_raw, st));
    SA_CUDA(dyr.upload(lat_raw, ny_raw, st));
    SA_CUDA(dzr.upload(z_raw, (size_t)nx_raw * ny_raw, st));
    SA_CUDA(dx.upload(x, nx, st));
    SA_CUDA(dy.upload(y, ny, st));
    SA_CUDA(launch_grid_topo(nx_raw, ny_raw, dxr.p, dyr.p, dzr.p, nx, ny, dx.p, dy.p, z_out, st));
    SA_CUDA(cudaStreamSynchronize(st));
    return SA_OK;
}

extern "C" int sa_topo_media(sa_ctx* ctx, int nx, int ny, const double* lon, const double* lat,
                             const double* z_gridded, int nper, const double* sigma_deg,
                             double* m11, double* m12, double* m22, double* angle,
                             void* stream) {
    if (!ctx) return SA_ERR_ARG;
    if (nx < 3 || ny < 3 || nper < 1 || !lon || !lat || !z_gridded || !sigma_deg || !m11 ||
        !m12 || !m22 || !angle)
        return fail(ctx, SA_ERR_ARG, "sa_topo_media: bad sizes or null pointers");
    for (int ip = 0; ip < nper; ip++)
        if (!(sigma_deg[ip] > 0.0)) return fail(ctx, SA_ERR_ARG, "sa_topo_media: sigma <= 0");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const size_t n = (size_t)nx * ny;
    DArr<double> dlon, dlat, zs;
    SA_CUDA(dlon.upload(lon, nx, st));
    SA_CUDA(dlat.upload(lat, ny, st));
    SA_CUDA(zs.alloc(n));
    for (int ip = 0; ip < nper; ip++) {
        // each period starts from the unsmoothed gridded topography (:93-96, :113-114)
        SA_CUDA(launch_gauss_geo(nx, ny, z_gridded, dlon.p, dlat.p, sigma_deg[ip], zs.p, st));
        SA_CUDA(launch_topo_media(nx, ny, zs.p, dlon.p, dlat.p, m11 + ip * n, m12 + ip * n,
                                  m22 + ip * n, angle + ip * n, st));
    }
    SA_CUDA(cudaStreamSynchronize(st));
    return SA_OK;
}

extern "C" int sa_correct_depth_with_topo(sa_ctx* ctx, int nx, int ny, int nz, int nper,
                                          const double* zgrid, const double* angle,
                                          double* sen_vs, double* sen_vp, double* sen_rho,
                                          void* stream) {
    if (!ctx) return SA_ERR_ARG;
    if (nx < 1 || ny < 1 || nz < 2 || nz > 64 || nper < 1 || !zgrid || !angle)
        return fail(ctx, SA_ERR_ARG, "sa_correct_depth_with_topo: bad sizes (2 <= nz <= 64)");
    SA_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    DArr<double> dz;
    SA_CUDA(dz.upload(zgrid, nz, st));
    SA_CUDA(launch_depth_topo(nx, ny, nz, nper, dz.p, angle, sen_vs, sen_vp, sen_rho, st));
    SA_CUDA(cudaStreamSynchronize(st));
    return SA_OK;
}
