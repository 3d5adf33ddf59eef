// CPU oracle: L-BFGS direction, strong-Wolfe step control, descent angle,
// gradient normalisation and the multiplicative vs update.  TEST
// INFRASTRUCTURE ONLY (see oracle.h).  vs-only parametrisation (one active
// parameter); inner products are sequential sums in index order.
#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

namespace {
constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double RAD2DEG = 180.0 / PI;                 // include/config.h:69
constexpr double REAL_EPS = DBL_EPSILON;               // include/config.h:30

double dot(const double* a, const double* b, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}
}  // namespace

// optimize::lbfgs_direction (src/optimize.cpp:150-255) for one parameter.
// models[h], grads[h] for h = 0 .. nhist (nhist + 1 consecutive iterates,
// the last being the current one); returns r = H g in dir.
extern "C" void orc_lbfgs_direction(size_t n, int nhist, const double* const* models,
                                    const double* const* grads, double* dir) {
    std::vector<double> q(grads[nhist], grads[nhist] + n);
    std::vector<std::vector<double>> s(nhist, std::vector<double>(n)), y(nhist, std::vector<double>(n));
    std::vector<double> rho(nhist, 0.0), alpha(nhist, 0.0);
    for (int h = 0; h < nhist; ++h) {
        for (size_t i = 0; i < n; i++) {
            s[h][i] = std::log(models[h + 1][i]) - std::log(models[h][i]);   // :190-191
            y[h][i] = grads[h + 1][i] - grads[h][i];                         // :197
        }
        const double sy = dot(s[h].data(), y[h].data(), n);
        rho[h] = (sy > 0.0) ? (1.0 / sy) : 0.0;                              // :203
    }
    for (int h = nhist - 1; h >= 0; --h) {                                   // :209-214
        alpha[h] = rho[h] * dot(s[h].data(), q.data(), n);
        for (size_t i = 0; i < n; i++) q[i] = q[i] - alpha[h] * y[h][i];
    }
    std::vector<double> r = q;                                               // :219-228
    if (nhist > 0) {
        const int last = nhist - 1;
        const double yy = dot(y[last].data(), y[last].data(), n);
        const double sy = dot(s[last].data(), y[last].data(), n);
        const double gamma = (sy > 0.0 && yy > 0.0) ? (sy / yy) : 1.0;
        for (size_t i = 0; i < n; i++) r[i] = gamma * r[i];
    }
    for (int h = 0; h < nhist; ++h) {                                        // :231-236
        const double beta = rho[h] * dot(y[h].data(), r.data(), n);
        for (size_t i = 0; i < n; i++) r[i] = r[i] + (alpha[h] - beta) * s[h][i];
    }
    std::copy(r.begin(), r.end(), dir);
}

// Inversion::grad_normalization (src/inversion.cpp:302-323), one parameter.
extern "C" double orc_grad_normalization(size_t n, double* g) {
    double m = 0.0;
    for (size_t i = 0; i < n; i++) m = std::max(m, std::abs(g[i]));
    if (m < REAL_EPS) return m;
    for (size_t i = 0; i < n; i++) g[i] = g[i] / m;
    return m;
}

// optimize::calc_descent_angle (src/optimize.cpp:33-57).
extern "C" double orc_descent_angle(size_t n, const double* dir, const double* grad) {
    const double d = dot(grad, dir, n);
    const double gn = std::sqrt(dot(grad, grad, n));
    const double dn = std::sqrt(dot(dir, dir, n));
    if (gn < REAL_EPS || dn < REAL_EPS) return 90.0;
    double c = d / (gn * dn);
    c = std::max(-1.0, std::min(1.0, c));
    return std::acos(c) * RAD2DEG;
}

// optimize::wolfe_condition (src/optimize.cpp:74-145) from the two inner
// products gd = grad . dir and kd = ker_next . dir.  Returns 0 ACCEPT, 1 TRY,
// 2 FAIL; next_alpha and the bracket are updated as in the reference.
extern "C" int orc_wolfe_condition(double gd, double kd, double alpha, double* alpha_L,
                                   double* alpha_R, double f0, double f1, int subiter, double c1,
                                   double c2, int max_sub_niter, double alpha_init,
                                   double* next_alpha) {
    const double q = -gd;
    const double q1 = -kd;
    const bool cond_armijo = f1 <= f0 + alpha * c1 * q;
    const bool cond_curvature = q1 >= c2 * q;
    int status;
    if (cond_armijo && cond_curvature) {
        status = 0;
        *next_alpha = alpha;
    } else if (!cond_armijo) {
        *alpha_R = alpha;
        *next_alpha = (*alpha_L + *alpha_R) * 0.5;
        status = 1;
    } else {
        *alpha_L = alpha;
        const double candidate = (*alpha_R > 0.0) ? (*alpha_L + *alpha_R) * 0.5 : alpha * 2.0;
        if (candidate > alpha_init) {
            *next_alpha = alpha_init;
            status = 0;
        } else {
            *next_alpha = candidate;
            status = 1;
        }
    }
    if (status == 1 && subiter == max_sub_niter - 1) {
        status = 2;
        *next_alpha = alpha;
    }
    return status;
}

// Inversion::model_update, vs-only (src/inversion.cpp:465-490):
// vs *= (1 - alpha*dir); vp = vs2vp(vs); rho = vp2rho(vp).
extern "C" void orc_model_update_vs(size_t n, const double* vs, const double* dir, double alpha,
                                    double* vs_out, double* vp_out, double* rho_out) {
    for (size_t i = 0; i < n; i++) {
        const double v = vs[i] * (1 - alpha * dir[i]);
        vs_out[i] = v;
        const double vp = orc_vs2vp(v);
        vp_out[i] = vp;
        rho_out[i] = orc_vp2rho(vp);
    }
}
