// CPU oracle: per-column dispersion and depth-kernel drivers.
// TEST INFRASTRUCTURE ONLY (see oracle.h).
#include "oracle.h"

#include <thread>
#include <vector>

namespace {

// surfker::build_disp_req / refine_request (src/surfdisp.cpp:60-108) followed
// by the float cast of the model (src/surfdisp.cpp:434-444).
void build_layers(int nz, const double* dep, const double* vs, std::vector<float>& thk,
                  std::vector<float>& vp, std::vector<float>& vsf, std::vector<float>& rho) {
    const int mmax = nz + 1;
    std::vector<double> t(mmax, 0.0), a(mmax, 0.0), b(mmax, 0.0), r(mmax, 0.0);
    for (int kk = 0; kk < nz; ++kk) {
        b[kk] = vs[kk];
        a[kk] = orc_vs2vp(vs[kk]);          // src/surf_grid.cpp:223-224
        r[kk] = orc_vp2rho(a[kk]);
        if (kk == nz - 1) t[kk] = (nz > 1) ? t[kk - 1] : 0.0;
        else t[kk] = dep[kk + 1] - dep[kk];
    }
    t[mmax - 1] = 0.0;
    a[mmax - 1] = a[nz - 1];
    b[mmax - 1] = b[nz - 1];
    r[mmax - 1] = r[nz - 1];
    thk.resize(mmax);
    vp.resize(mmax);
    vsf.resize(mmax);
    rho.resize(mmax);
    for (int i = 0; i < mmax; i++) {
        thk[i] = static_cast<float>(t[i]);
        vp[i] = static_cast<float>(a[i]);
        vsf[i] = static_cast<float>(b[i]);
        rho[i] = static_cast<float>(r[i]);
    }
}

template <class F>
void for_columns(int ncol, int nthreads, F&& f) {
    if (nthreads <= 1) {
        for (int c = 0; c < ncol; c++) f(c);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++)
        pool.emplace_back([&, t]() {
            for (int c = t; c < ncol; c += nthreads) f(c);
        });
    for (auto& th : pool) th.join();
}

}  // namespace

// SurfGrid::fwdsurf (src/surf_grid.cpp:194-245); column c = ix*ny + iy.
extern "C" int orc_fwdsurf(int nx, int ny, int nz, const double* zgrid, const double* vs3d,
                           int nper, const double* periods, int iwave, int igr, double* svel,
                           int* status, int nthreads) {
    const int ncol = nx * ny;
    for_columns(ncol, nthreads, [&](int col) {
        const int ix = col / ny, iy = col % ny;
        std::vector<float> thk, vp, vs, rho;
        build_layers(nz, zgrid, vs3d + static_cast<size_t>(col) * nz, thk, vp, vs, rho);
        std::vector<double> cg(nper, 0.0);
        const int st = orc_surfdisp96(thk.data(), vp.data(), vs.data(), rho.data(), nz + 1,
                                      1, iwave, 1, igr, nper, periods, cg.data());
        if (status) status[ix + nx * iy] = st;
        for (int ip = 0; ip < nper; ip++)
            svel[static_cast<size_t>(ip) * nx * ny + ix + nx * iy] = cg[ip];
    });
    return 0;
}

// SurfGrid::compute_dispersion_kernel -> surfker::depthkernelHTI1d
// (src/surf_grid.cpp:247-305, src/surfdisp.cpp:481-547).
extern "C" int orc_depthkernel_hti(int nx, int ny, int nz, const double* zgrid,
                                   const double* vs3d, int nper, const double* periods,
                                   double* sen_vs, double* sen_vp, double* sen_rho,
                                   int* status, int nthreads) {
    const int ncol = nx * ny;
    const int mmax = nz + 1;
    for_columns(ncol, nthreads, [&](int col) {
        const int ix = col / ny, iy = col % ny;
        std::vector<float> thk, vp, vs, rho;
        build_layers(nz, zgrid, vs3d + static_cast<size_t>(col) * nz, thk, vp, vs, rho);
        std::vector<double> cp(nper, 0.0);
        const int st = orc_surfdisp96(thk.data(), vp.data(), vs.data(), rho.data(), mmax, 1, 2,
                                      1, 0, nper, periods, cp.data());
        if (status) status[ix + nx * iy] = st;
        std::vector<double> du(mmax), dw(mmax), su(mmax), sw(mmax), da(mmax), db(mmax),
            dh(mmax), dr(mmax), dgc(mmax), dgs(mmax);
        double cg = 0.0;
        for (int ip = 0; ip < nper; ip++) {
            double t_val = periods[ip];
            double cp_val = cp[ip];
            orc_sregn96_hti(thk.data(), vp.data(), vs.data(), rho.data(), mmax, &t_val, &cp_val,
                            &cg, du.data(), dw.data(), su.data(), sw.data(), da.data(), db.data(),
                            dh.data(), dr.data(), dgc.data(), dgs.data(), 1);
            for (int k = 0; k < nz; k++) {
                const size_t i4 = ((static_cast<size_t>(col)) * nz + k) * nper + ip;
                sen_vs[i4] = db[k];
                sen_vp[i4] = da[k];
                sen_rho[i4] = dr[k];
            }
        }
    });
    return 0;
}

// surfker::depthkernel_rayleigh_group (src/surfdisp.cpp:203-285) per column:
// phase velocities at t, t(1 + 0.005) and t(1 - 0.005), then sregnpu.
extern "C" int orc_depthkernel_group(int nx, int ny, int nz, const double* zgrid,
                                     const double* vs3d, int nper, const double* periods,
                                     double* sen_vs, double* sen_vp, double* sen_rho,
                                     int* status, int nthreads) {
    const int ncol = nx * ny;
    const int mmax = nz + 1;
    const double dt = 0.01;
    std::vector<double> t1(nper), t2(nper);
    for (int i = 0; i < nper; ++i) {
        t1[i] = periods[i] * (1.0 + 0.5 * dt);
        t2[i] = periods[i] * (1.0 - 0.5 * dt);
    }
    for_columns(ncol, nthreads, [&](int col) {
        const int ix = col / ny, iy = col % ny;
        std::vector<float> thk, vp, vs, rho;
        build_layers(nz, zgrid, vs3d + static_cast<size_t>(col) * nz, thk, vp, vs, rho);
        std::vector<double> cp(nper, 0.0), cp1(nper, 0.0), cp2(nper, 0.0);
        int st = orc_surfdisp96(thk.data(), vp.data(), vs.data(), rho.data(), mmax, 1, 2, 1, 0,
                                nper, periods, cp.data());
        st |= orc_surfdisp96(thk.data(), vp.data(), vs.data(), rho.data(), mmax, 1, 2, 1, 0,
                             nper, t1.data(), cp1.data());
        st |= orc_surfdisp96(thk.data(), vp.data(), vs.data(), rho.data(), mmax, 1, 2, 1, 0,
                             nper, t2.data(), cp2.data());
        if (status) status[ix + nx * iy] = st;
        std::vector<double> ua(mmax), ub(mmax), uh(mmax), ur(mmax), ca(mmax), cb(mmax),
            ch(mmax), cr(mmax);
        for (int ip = 0; ip < nper; ip++) {
            double cg = 0.0;
            orc_sregnpu(thk.data(), vp.data(), vs.data(), rho.data(), mmax, periods[ip], cp[ip],
                        t1[ip], cp1[ip], t2[ip], cp2[ip], &cg, ua.data(), ub.data(), uh.data(),
                        ur.data(), ca.data(), cb.data(), ch.data(), cr.data(), 1);
            for (int k = 0; k < nz; k++) {
                const size_t i4 = ((static_cast<size_t>(col)) * nz + k) * nper + ip;
                sen_vs[i4] = ub[k];
                sen_vp[i4] = ua[k];
                sen_rho[i4] = ur[k];
            }
        }
    });
    return 0;
}

// surfker::depthkernel_love_phase (src/surfdisp.cpp:295-349, igr 0) and
// depthkernel_love_group (:351-426, igr 1) per column: Love phase
// velocities (surfdisp96, iwave 1) at t (and t(1 +- 0.005)), then slegn96 /
// slegnpu; sen_vs, sen_rho (nx, ny, nz, nper) the first nz layers.
extern "C" int orc_depthkernel_love(int nx, int ny, int nz, const double* zgrid,
                                    const double* vs3d, int nper, const double* periods,
                                    int igr, double* sen_vs, double* sen_rho, int* status,
                                    int nthreads) {
    const int ncol = nx * ny;
    const int mmax = nz + 1;
    const double dt = 0.01;
    std::vector<double> t1(nper), t2(nper);
    for (int i = 0; i < nper; ++i) {
        t1[i] = periods[i] * (1.0 + 0.5 * dt);
        t2[i] = periods[i] * (1.0 - 0.5 * dt);
    }
    for_columns(ncol, nthreads, [&](int col) {
        const int ix = col / ny, iy = col % ny;
        std::vector<float> thk, vp, vs, rho;
        build_layers(nz, zgrid, vs3d + static_cast<size_t>(col) * nz, thk, vp, vs, rho);
        std::vector<double> cp(nper, 0.0), cp1(nper, 0.0), cp2(nper, 0.0);
        int st = orc_surfdisp96(thk.data(), vp.data(), vs.data(), rho.data(), mmax, 1, 1, 1, 0,
                                nper, periods, cp.data());
        if (igr) {
            st |= orc_surfdisp96(thk.data(), vp.data(), vs.data(), rho.data(), mmax, 1, 1, 1, 0,
                                 nper, t1.data(), cp1.data());
            st |= orc_surfdisp96(thk.data(), vp.data(), vs.data(), rho.data(), mmax, 1, 1, 1, 0,
                                 nper, t2.data(), cp2.data());
        }
        if (status) status[ix + nx * iy] = st;
        std::vector<double> kb(mmax), kr(mmax);
        for (int ip = 0; ip < nper; ip++) {
            double cg = 0.0;
            if (igr)
                orc_slegnpu(thk.data(), vs.data(), rho.data(), mmax, periods[ip], cp[ip], t1[ip],
                            cp1[ip], t2[ip], cp2[ip], &cg, kb.data(), kr.data(), 1);
            else
                orc_slegn96(thk.data(), vs.data(), rho.data(), mmax, periods[ip], cp[ip], &cg,
                            kb.data(), kr.data(), 1);
            for (int k = 0; k < nz; k++) {
                const size_t i4 = ((static_cast<size_t>(col)) * nz + k) * nper + ip;
                sen_vs[i4] = kb[k];
                sen_rho[i4] = kr[k];
            }
        }
    });
    return 0;
}
