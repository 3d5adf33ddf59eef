// Converged state of the oracle's factored-eikonal forward solve, for the
// discrete adjoint (eikonal_discrete.cpp).  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <vector>

struct EikState {
    int nx = 0, ny = 0;
    double dx = 0, dy = 0;           // grid spacing (radians)
    double fun0 = 0;                 // slowness at the source (bilinear)
    int idx0 = 0, idy0 = 0;          // source cell and its bilinear weights
    double r1 = 0, r2 = 0;
    std::vector<double> a, b, c;     // metric (src/eikonal_solver.cpp:55-65)
    std::vector<double> T0, T0x, T0y;
    std::vector<double> G, Gx, Gy;   // T0 = G fun0, T0x = Gx fun0, T0y = Gy fun0
    std::vector<double> tau;
    std::vector<unsigned char> ischange;
};

// The forward solve (src/eikonal_solver.cpp:22-318); tol > 0 stops as the
// reference, tol == 0 at a fixed point.  Fills *st when given.
int eik_fwd_core(int nx, int ny, const double* xx_deg, const double* yy_deg,
                 const double* spha, const double* sphb, const double* sphc, const double* fun,
                 double x0_deg, double y0_deg, double tol, int maxiter, double* T_out,
                 int* niter, EikState* st);
