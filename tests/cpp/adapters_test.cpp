// Host adapters over libsurfatt_gpu.so in the reference's data layouts, as a
// maintainer would write them into SurfATTPP (the C++ side of the drop-in
// boundary), compiled as plain C++20 against include/surfatt_gpu.h and the
// CUDA runtime.  std::vector stands in for Eigen (column-major nx x ny
// matrices are the same flat arrays); SrcRec::events_local is a std::map
// keyed "{evtname}_{iper}" as in src/src_rec.cpp:138-228; SurfGrid::svel is
// [(ix*ny + iy)*nper + iper] as include/surf_grid.h:63-65.
//
// Usage: adapters_test <input.bin> <output.bin> [table.csv]
// The input holds a surface grid, a vs model, periods, events and observed
// times (written by tests/test_gpu_cpp_adapters.py); the program runs
//   fwdsurf                    (SurfGrid::fwdsurf -> sa_surfdisp_columns)
//   forward_for_event          (preproc:: -> sa_plan_create / sa_plan_forward_adjoint)
//   run_forward_adjoint        (Inversion:: -> sa_grad_create / sa_grad_run)
//   FSM_UW_PS_lonlat_2d        (eikonal:: -> sa_eik_fwd_field), one event
// in FP64 and writes the results; with a CSV it also prints the event table
// built by sa_srcrec_load.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "surfatt_gpu.h"

namespace {

sa_ctx* g_ctx = nullptr;

void check(int rc) {
    if (rc == SA_OK) return;
    const std::string msg = sa_ctx_error(g_ctx);
    if (rc == SA_ERR_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error("status " + std::to_string(rc) + ": " + msg);
}
void cuda(cudaError_t e) {
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
}

template <class T>
struct Dev {   // a device array
    T* p = nullptr;
    size_t n = 0;
    explicit Dev(size_t count) : n(count) { cuda(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T))); }
    Dev(const std::vector<T>& h) : Dev(h.size()) { put(h); }
    ~Dev() { cudaFree(p); }
    void put(const std::vector<T>& h) {
        cuda(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    std::vector<T> get() const {
        std::vector<T> h(n);
        cuda(cudaMemcpy(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost));
        return h;
    }
};

// ---- reference-shaped data carriers ----------------------------------------
struct event_info {                  // include/src_rec.h:15-35
    double evlo = 0, evla = 0;
    int iper = 0;
    std::vector<int> rec_indices;    // observation rows
    std::vector<double> syn_data;
};
struct SrcRec {
    std::vector<double> stlo, stla, tt, weight;          // per observation
    std::map<std::string, event_info> events_local;
};
struct SurfGrid {
    int nx = 0, ny = 0, nper = 0;
    std::vector<double> svel;                            // [(ix*ny + iy)*nper + iper]
    std::vector<std::vector<double>> adj_s_local;        // nper x (nx*ny), column-major
    size_t surf_idx(int ix, int iy, int ip) const { return ((size_t)ix * ny + iy) * nper + ip; }
};

// ---- adapters ----------------------------------------------------------------
// SurfGrid::fwdsurf (src/surf_grid.cpp:194-245): vs3d (nx, ny, nz) row-major
void fwdsurf(SurfGrid& sg, const std::vector<double>& vs3d, int nz,
             const std::vector<double>& zgrid, const std::vector<double>& periods) {
    const int nx = sg.nx, ny = sg.ny, np = sg.nper;
    Dev<double> d_vs(vs3d), d_sv((size_t)np * nx * ny);
    Dev<int> d_st((size_t)nx * ny);
    check(sa_surfdisp_columns(g_ctx, nx, ny, nz, zgrid.data(), d_vs.p, np, periods.data(), 2, 0,
                              d_sv.p, d_st.p, nullptr));
    cuda(cudaDeviceSynchronize());
    for (int s : d_st.get())
        if (s) throw std::runtime_error("Dispersion calculation failed");
    const std::vector<double> planes = d_sv.get();             // [iper][iy][ix]
    sg.svel.assign((size_t)nx * ny * np, 0.0);
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy)
            for (int p = 0; p < np; ++p)
                sg.svel[sg.surf_idx(ix, iy, p)] = planes[((size_t)p * ny + iy) * nx + ix];
}

struct Events {   // CSR form of events_local in map order
    std::vector<double> evlo, evla;
    std::vector<int> iper, ptr{0}, idx;
};
Events csr(const SrcRec& sr) {
    Events e;
    for (const auto& [name, info] : sr.events_local) {
        e.evlo.push_back(info.evlo);
        e.evla.push_back(info.evla);
        e.iper.push_back(info.iper);
        e.idx.insert(e.idx.end(), info.rec_indices.begin(), info.rec_indices.end());
        e.ptr.push_back((int)e.idx.size());
    }
    return e;
}

// preproc::forward_for_event (src/preproc.cpp:71-148), isotropic surface
double forward_for_event(SrcRec& sr, SurfGrid& sg, const std::vector<double>& xx,
                         const std::vector<double>& yy, bool calc_adj) {
    const int nx = sg.nx, ny = sg.ny, np = sg.nper;
    const Events e = csr(sr);
    sa_plan* plan = nullptr;
    check(sa_plan_create(g_ctx, SA_FP64, nx, ny, np, xx.data(), yy.data(), (int)e.evlo.size(),
                         e.evlo.data(), e.evla.data(), e.iper.data(), e.ptr.data(), e.idx.data(),
                         (int)sr.stlo.size(), sr.stlo.data(), sr.stla.data(), &plan));
    std::vector<double> planes((size_t)np * nx * ny), tt(e.idx.size()), w(e.idx.size());
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy)
            for (int p = 0; p < np; ++p)
                planes[((size_t)p * ny + iy) * nx + ix] = sg.svel[sg.surf_idx(ix, iy, p)];
    for (size_t i = 0; i < e.idx.size(); ++i) {
        tt[i] = sr.tt[e.idx[i]];
        w[i] = sr.weight[e.idx[i]];
    }
    Dev<double> d_sv(planes), d_tt(tt), d_w(w), d_syn(e.idx.size()), d_adj(planes.size()),
        d_chi(1);
    check(sa_plan_forward_adjoint(plan, d_sv.p, nullptr, nullptr, nullptr, d_tt.p, d_w.p,
                                  calc_adj ? 1 : 0, d_syn.p, d_adj.p, d_chi.p, nullptr, nullptr,
                                  nullptr, nullptr));
    cuda(cudaDeviceSynchronize());
    const std::vector<double> syn = d_syn.get(), adj = d_adj.get();
    size_t k = 0;
    for (auto& [name, info] : sr.events_local) {
        info.syn_data.assign(syn.begin() + k, syn.begin() + k + info.rec_indices.size());
        k += info.rec_indices.size();
    }
    sg.adj_s_local.assign(np, std::vector<double>((size_t)nx * ny));
    for (int p = 0; p < np; ++p)       // plane [iy][ix] == column-major nx x ny
        std::copy(adj.begin() + (size_t)p * nx * ny, adj.begin() + (size_t)(p + 1) * nx * ny,
                  sg.adj_s_local[p].begin());
    sa_plan_destroy(plan);
    return calc_adj ? d_chi.get()[0] : 0.0;
}

// Inversion::run_forward_adjoint(true) up to combine_kernels
// (src/inversion.cpp:245-276): ker_vs (nx, ny, nz) row-major
double run_forward_adjoint(SrcRec& sr, int nx, int ny, int nz, const std::vector<double>& xx,
                           const std::vector<double>& yy, const std::vector<double>& zgrid,
                           const std::vector<double>& periods, const std::vector<double>& vs3d,
                           std::vector<double>& ker_vs) {
    const Events e = csr(sr);
    const int np = (int)periods.size();
    sa_plan* plan = nullptr;
    check(sa_plan_create(g_ctx, SA_FP64, nx, ny, np, xx.data(), yy.data(), (int)e.evlo.size(),
                         e.evlo.data(), e.evla.data(), e.iper.data(), e.ptr.data(), e.idx.data(),
                         (int)sr.stlo.size(), sr.stlo.data(), sr.stla.data(), &plan));
    sa_grad* grad = nullptr;
    check(sa_grad_create(plan, nz, zgrid.data(), periods.data(), &grad));
    std::vector<double> tt(e.idx.size()), w(e.idx.size());
    for (size_t i = 0; i < e.idx.size(); ++i) {
        tt[i] = sr.tt[e.idx[i]];
        w[i] = sr.weight[e.idx[i]];
    }
    Dev<double> d_vs(vs3d), d_tt(tt), d_w(w), d_ker(vs3d.size()), d_chi(1);
    Dev<int> d_st(1);
    check(sa_grad_run(grad, d_vs.p, nullptr, d_tt.p, d_w.p, d_ker.p, d_chi.p, nullptr, nullptr,
                      d_st.p, nullptr));
    cuda(cudaDeviceSynchronize());
    if (d_st.get()[0] != 0) throw std::runtime_error("run_forward_adjoint: status");
    ker_vs = d_ker.get();
    const double chi = d_chi.get()[0];
    sa_grad_destroy(grad);
    sa_plan_destroy(plan);
    return chi;
}

// eikonal::FSM_UW_PS_lonlat_2d (src/eikonal_solver.cpp:22-318), host arrays
std::vector<double> FSM_UW_PS_lonlat_2d(const std::vector<double>& xx,
                                        const std::vector<double>& yy,
                                        const std::vector<double>& spha,
                                        const std::vector<double>& sphb,
                                        const std::vector<double>& sphc,
                                        const std::vector<double>& fun, double x0, double y0) {
    const int nx = (int)xx.size(), ny = (int)yy.size();
    if (nx < 3 || ny < 3) throw std::invalid_argument("Grid must be at least 3x3");
    std::vector<double> T((size_t)nx * ny);
    int it = 0;
    const int rc = sa_eik_fwd_field(g_ctx, SA_FP64, nx, ny, xx.data(), yy.data(), spha.data(),
                                    sphb.data(), sphc.data(), fun.data(), x0, y0, T.data(), &it);
    if (rc == SA_ERR_NOCONV)
        std::fprintf(stderr, "[eikonal] WARNING: FSM did not converge after 2000 iterations\n");
    else check(rc);
    return T;
}

// ---- binary I/O with the test ----------------------------------------------
struct Reader {
    FILE* f;
    explicit Reader(const char* path) : f(std::fopen(path, "rb")) {
        if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    }
    ~Reader() { std::fclose(f); }
    int64_t i() {
        int64_t v;
        if (std::fread(&v, 8, 1, f) != 1) throw std::runtime_error("short input");
        return v;
    }
    template <class T>
    std::vector<T> vec() {
        const int64_t n = i();
        std::vector<T> v(n);
        if (n && std::fread(v.data(), sizeof(T), n, f) != (size_t)n)
            throw std::runtime_error("short input");
        return v;
    }
};
struct Writer {
    FILE* f;
    explicit Writer(const char* path) : f(std::fopen(path, "wb")) {
        if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    }
    ~Writer() { std::fclose(f); }
    void vec(const std::vector<double>& v) {
        const int64_t n = (int64_t)v.size();
        std::fwrite(&n, 8, 1, f);
        std::fwrite(v.data(), 8, v.size(), f);
    }
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s input.bin output.bin [table.csv]\n", argv[0]);
        return 2;
    }
    try {
        check(sa_ctx_create(0, &g_ctx));
        Reader in(argv[1]);
        const int nx = (int)in.i(), ny = (int)in.i(), nz = (int)in.i();
        const auto xx = in.vec<double>(), yy = in.vec<double>(), zgrid = in.vec<double>();
        const auto periods = in.vec<double>(), vs3d = in.vec<double>();
        const auto evlo = in.vec<double>(), evla = in.vec<double>();
        const auto iper = in.vec<int32_t>(), ptr = in.vec<int32_t>(), idx = in.vec<int32_t>();
        const auto stlo = in.vec<double>(), stla = in.vec<double>();
        const auto tt = in.vec<double>(), wt = in.vec<double>();
        // SrcRec: one observation row per (event, receiver); events keyed as
        // the reference's map ("{evtname}_{iper}"; here "EV{index:04d}_{iper}")
        SrcRec sr;
        for (size_t e = 0; e + 1 < ptr.size(); ++e) {
            char key[64];
            std::snprintf(key, sizeof(key), "EV%04zu_%d", e, iper[e]);
            event_info info;
            info.evlo = evlo[e];
            info.evla = evla[e];
            info.iper = iper[e];
            for (int r = ptr[e]; r < ptr[e + 1]; ++r) {
                info.rec_indices.push_back((int)sr.stlo.size());
                sr.stlo.push_back(stlo[idx[r]]);
                sr.stla.push_back(stla[idx[r]]);
                sr.tt.push_back(tt[r]);
                sr.weight.push_back(wt[r]);
            }
            sr.events_local[key] = info;
        }
        SurfGrid sg;
        sg.nx = nx;
        sg.ny = ny;
        sg.nper = (int)periods.size();
        fwdsurf(sg, vs3d, nz, zgrid, periods);
        const double chi = forward_for_event(sr, sg, xx, yy, true);
        std::vector<double> syn;
        for (const auto& [name, info] : sr.events_local)
            syn.insert(syn.end(), info.syn_data.begin(), info.syn_data.end());
        std::vector<double> adj;
        for (const auto& plane : sg.adj_s_local) adj.insert(adj.end(), plane.begin(), plane.end());
        std::vector<double> ker;
        const double chi2 = run_forward_adjoint(sr, nx, ny, nz, xx, yy, zgrid, periods, vs3d, ker);
        // one eikonal:: solve: the first event, isotropic metric
        const size_t n = (size_t)nx * ny;
        std::vector<double> one(n, 1.0), zero(n, 0.0), fun(n);
        const int p0 = sr.events_local.begin()->second.iper;
        for (int ix = 0; ix < nx; ++ix)
            for (int iy = 0; iy < ny; ++iy) fun[ix + (size_t)nx * iy] = 1.0 / sg.svel[sg.surf_idx(ix, iy, p0)];
        const auto T = FSM_UW_PS_lonlat_2d(xx, yy, one, one, zero, fun,
                                           sr.events_local.begin()->second.evlo,
                                           sr.events_local.begin()->second.evla);
        Writer out(argv[2]);
        out.vec(sg.svel);
        out.vec(syn);
        out.vec(adj);
        out.vec({chi, chi2});
        out.vec(ker);
        out.vec(T);
        if (argc > 3) {   // SrcRec::load / get_events through the library
            sa_srcrec* t = nullptr;
            check(sa_srcrec_load(argv[3], &t));
            int nobs = 0, nperiod = 0, nev = 0;
            check(sa_srcrec_sizes(t, &nobs, &nperiod, &nev));
            std::printf("table %d observations %d periods %d events first %s last %s\n", nobs,
                        nperiod, nev, sa_srcrec_event_name(t, 0), sa_srcrec_event_name(t, nev - 1));
            sa_srcrec_destroy(t);
        }
        sa_ctx_destroy(g_ctx);
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "adapters_test: %s\n", ex.what());
        return 1;
    }
    return 0;
}
