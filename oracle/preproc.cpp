// CPU oracle: per-event forward/adjoint driver, kernel accumulation, kernel
// combination and the Brocher relations.  TEST INFRASTRUCTURE ONLY.
#include "oracle.h"
#include "omath.h"

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

// include/utils.h:185-187
extern "C" double orc_vs2vp(double vs) {
    return 0.9409 + 2.0947 * vs - 0.8206 * vs * vs + 0.2683 * vs * vs * vs - 0.0251 * vs * vs * vs * vs;
}
// include/utils.h:223-225
extern "C" double orc_vp2rho(double vp) {
    return 1.6612 * vp - 0.4721 * vp * vp + 0.0671 * vp * vp * vp - 0.0043 * vp * vp * vp * vp
         + 0.000106 * vp * vp * vp * vp * vp;
}
// include/utils.h:210-212
extern "C" double orc_dalpha_dbeta(double vs) {
    return 2.0947 - 2 * 0.8206 * vs + 3 * 0.2683 * vs * vs - 4 * 0.0251 * vs * vs * vs;
}
// include/utils.h:198-200
extern "C" double orc_drho_dalpha(double vp) {
    return 1.6612 - 2 * 0.4721 * vp + 3 * 0.0671 * vp * vp - 4 * 0.0043 * vp * vp * vp
         + 5 * 0.000106 * vp * vp * vp * vp;
}

namespace {

struct EventRange {
    int nx, ny, nper;
    const double *xx_deg, *yy_deg, *svel, *m11, *m12, *m22;
    const double *evlo, *evla;
    const int *iper, *rec_ptr, *rec_idx;
    const double *stlo, *stla, *tt_obs, *weight;
    int calc_adj;
    double* syn;
    int *fwd_iters, *adj_iters;
    bool kden;    // is_kden: the kernel-density adjoint as well
};

// One event of preproc::forward_for_event (src/preproc.cpp:79-143) plus
// accumulate_kernels (src/preproc.cpp:19-34).  Returns 0.5*sum(w r^2).
// With R.kden, the kernel-density adjoint (:128-137): source -w at every
// receiver, the field NOT masked (the reference masks adj_field a second
// time instead), accumulated into kden_acc with svel^-3.
double run_event(const EventRange& R, int ie, double* adj_acc, double* kden_acc) {
    const int nx = R.nx, ny = R.ny, n = nx * ny;
    const int ip = R.iper[ie];
    const double* svel = R.svel + static_cast<size_t>(ip) * n;
    const double* m11 = R.m11 + static_cast<size_t>(ip) * n;
    const double* m12 = R.m12 + static_cast<size_t>(ip) * n;
    const double* m22 = R.m22 + static_cast<size_t>(ip) * n;
    std::vector<double> fun(n), sphc(n), T(n);
    for (int k = 0; k < n; k++) {
        fun[k] = (1.0 / svel[k]) * 1.0;   // cwiseInverse() * _1_CR, :97-98
        sphc[k] = -m12[k];
    }
    int it = 0;
    orc_eik_fwd(nx, ny, R.xx_deg, R.yy_deg, m11, m22, sphc.data(), fun.data(),
                R.evlo[ie], R.evla[ie], T.data(), &it);
    if (R.fwd_iters) R.fwd_iters[ie] = it;

    const int r0 = R.rec_ptr[ie], nr = R.rec_ptr[ie + 1] - r0;
    std::vector<double> xr(nr), yr(nr), ttsyn(nr);
    for (int i = 0; i < nr; i++) {
        xr[i] = R.stlo[R.rec_idx[r0 + i]];
        yr[i] = R.stla[R.rec_idx[r0 + i]];
    }
    orc_interp2d(nx, ny, R.xx_deg, R.yy_deg, T.data(), nr, xr.data(), yr.data(), ttsyn.data());
    for (int i = 0; i < nr; i++) R.syn[r0 + i] = ttsyn[i];
    if (!R.calc_adj) return 0.0;

    std::vector<double> sadj(nr), Ta(n);
    for (int i = 0; i < nr; i++) sadj[i] = R.weight[r0 + i] * (ttsyn[i] - R.tt_obs[r0 + i]);
    orc_eik_adj(nx, ny, R.xx_deg, R.yy_deg, m11, m22, sphc.data(), T.data(), nr, xr.data(),
                yr.data(), sadj.data(), Ta.data(), &it);
    if (R.adj_iters) R.adj_iters[ie] = it;
    orc_mask_uniform_grid(nx, ny, R.xx_deg, R.yy_deg, Ta.data(), R.evlo[ie], R.evla[ie]);
    double* acc = adj_acc + static_cast<size_t>(ip) * n;
    for (int k = 0; k < n; k++) acc[k] += Ta[k] * om::pow_m3(svel[k]);   // pow(svel, -3)
    if (R.kden && kden_acc) {
        std::vector<double> sk(nr), Tk(n);
        for (int i = 0; i < nr; i++) sk[i] = -R.weight[r0 + i] * 1.0;
        orc_eik_adj(nx, ny, R.xx_deg, R.yy_deg, m11, m22, sphc.data(), T.data(), nr, xr.data(),
                    yr.data(), sk.data(), Tk.data(), &it);
        double* kacc = kden_acc + static_cast<size_t>(ip) * n;
        for (int k = 0; k < n; k++) kacc[k] += Tk[k] * om::pow_m3(svel[k]);
    }
    double s = 0.0;
    for (int i = 0; i < nr; i++) {
        const double r = ttsyn[i] - R.tt_obs[r0 + i];
        s += R.weight[r0 + i] * (r * r);
    }
    return 0.5 * s;
}

}  // namespace

extern "C" int orc_forward_for_events(int nx, int ny, int nper, const double* xx_deg,
                                      const double* yy_deg, const double* svel,
                                      const double* m11, const double* m12, const double* m22,
                                      int ne, const double* evlo, const double* evla,
                                      const int* iper, const int* rec_ptr, const int* rec_idx,
                                      const double* stlo, const double* stla,
                                      const double* tt_obs, const double* weight,
                                      int calc_adj, double* syn, double* adj_s, double* chi,
                                      int* fwd_iters, int* adj_iters, int nthreads,
                                      double* kden_s) {
    EventRange R{nx, ny, nper, xx_deg, yy_deg, svel, m11, m12, m22, evlo, evla, iper,
                 rec_ptr, rec_idx, stlo, stla, tt_obs, weight, calc_adj, syn,
                 fwd_iters, adj_iters, kden_s != nullptr};
    const size_t plane = static_cast<size_t>(nx) * ny * nper;
    if (nthreads <= 1) {
        double c = 0.0;
        for (int ie = 0; ie < ne; ie++) c += run_event(R, ie, adj_s, kden_s);
        if (chi) *chi = c;
        return 0;
    }
    // Round-robin event ownership, one private accumulator per worker, summed
    // in worker order afterwards (the allreduce of src/preproc.cpp:146, :238).
    std::vector<std::vector<double>> acc(nthreads), kacc(nthreads);
    std::vector<double> chis(nthreads, 0.0);
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++) {
        pool.emplace_back([&, t]() {
            if (calc_adj) acc[t].assign(plane, 0.0);
            if (calc_adj && kden_s) kacc[t].assign(plane, 0.0);
            double c = 0.0;
            for (int ie = t; ie < ne; ie += nthreads)
                c += run_event(R, ie, calc_adj ? acc[t].data() : nullptr,
                               calc_adj && kden_s ? kacc[t].data() : nullptr);
            chis[t] = c;
        });
    }
    for (auto& th : pool) th.join();
    double c = 0.0;
    for (int t = 0; t < nthreads; t++) {
        c += chis[t];
        if (calc_adj)
            for (size_t k = 0; k < plane; k++) adj_s[k] += acc[t][k];
        if (calc_adj && kden_s)
            for (size_t k = 0; k < plane; k++) kden_s[k] += kacc[t][k];
    }
    if (chi) *chi = c;
    return 0;
}

// postproc::kernel_precondition (src/postproc.cpp:487-517): with the kernel
// density normalised by its largest magnitude, ker *= 1/norm where norm >
// VERYTINY (1e-12, include/config.h:71), unchanged elsewhere; nothing when
// the density itself is below VERYTINY.
extern "C" void orc_kernel_precondition(size_t n, const double* ker_den, double* ker) {
    double L_inf = 0.0;
    for (size_t i = 0; i < n; i++) L_inf = std::max(L_inf, std::abs(ker_den[i]));
    if (L_inf < 1e-12) return;
    for (size_t i = 0; i < n; i++) {
        const double norm = ker_den[i] / L_inf;
        const double h = norm > 1e-12 ? 1.0 / norm : 1.0;
        ker[i] = ker[i] * h;
    }
}

// src/preproc.cpp:276-304 (vs-only parametrisation, is_kden = false).
extern "C" void orc_combine_kernels_vs(int nx, int ny, int nz, int nper, const double* adj_s,
                                       const double* vs3d, const double* vp3d,
                                       const double* sen_vs, const double* sen_vp,
                                       const double* sen_rho, double* ker_vs) {
    const size_t n3 = static_cast<size_t>(nx) * ny * nz;
    for (size_t i = 0; i < n3; i++) ker_vs[i] = 0.0;
    for (int ip = 0; ip < nper; ++ip) {
        const double* adj_tt = adj_s + static_cast<size_t>(ip) * nx * ny;
        for (int ix = 0; ix < nx; ++ix) {
            for (int iy = 0; iy < ny; ++iy) {
                const double att = adj_tt[ix + nx * iy];
                for (int k = 0; k < nz; ++k) {
                    const size_t i3 = (static_cast<size_t>(ix) * ny + iy) * nz + k;
                    const size_t i4 = i3 * nper + ip;
                    const double vs = vs3d[i3];
                    const double vp = vp3d[i3];
                    const double dab = orc_dalpha_dbeta(vs);
                    const double dra = orc_drho_dalpha(vp);
                    ker_vs[i3] -= att * (sen_vs[i4] + sen_vp[i4] * dab + sen_rho[i4] * dra * dab);
                }
            }
        }
    }
}
