// Shared device-side types and constants for the SurfATT B200 engine.
//
// Field layout in HBM: every 2-D surface field is a row-major [iy][ix] plane
// (ix fastest), i.e. the reference's Eigen column-major nx x ny matrix
// (index ix + nx*iy).  Per-period fields are stacked planes [iper][iy][ix];
// per-source geometry planes are [isrc][iy][ix].
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sa {

constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double R_EARTH = 6371.0;
constexpr double DEG2RAD = PI / 180.0;

// Status codes written per event (device) and returned by the C ABI (host).
enum Status : int {
    ST_OK = 0,
    ST_NOCONV = 3,        // sweep iteration cap reached (reference only warns)
    ST_NONFINITE = 5,     // NaN/Inf in a travel-time or adjoint field
    ST_TEAM = 7,          // a cooperative sweep's wait gave up (FP32 tail teams)
};

// Surface grid (device pointers).  Trigonometric row tables are produced on
// the host with the C library so that they match a CPU evaluation exactly.
struct Grid {
    int nx, ny;
    const double* xx_deg;   // [nx] degrees (receiver interpolation, source mask)
    const double* yy_deg;   // [ny]
    const double* xx;       // [nx] radians = xx_deg * DEG2RAD
    const double* yy;       // [ny]
    const double* cosy;     // [ny] cos(yy)
    const double* siny;     // [ny] sin(yy)
    double dx, dy;          // radians, xx[1]-xx[0], yy[1]-yy[0]
};

// Per-period media.  In isotropic mode (flat surface, m11 = m22 = 1,
// m12 = 0) the metric depends on the row only: forward a = 1/(R^2 cos^2),
// adjoint a = 1/((R^2 cos) cos), b = 1/R^2, c = -0.0.
template <class T>
struct Media {
    int nper;
    int iso;
    const T* fun;         // [nper][ny][nx] slowness (1/svel)*1
    const double* inv_svel3;  // [nper][ny][nx] svel^-3 (FP64 accumulation)
    const T* a_f_row;     // [ny]  (iso)
    const T* a_a_row;     // [ny]  (iso)
    T b_iso;
    const T* a_f;         // [nper][ny][nx] (general)
    const T* b_p;
    const T* c_f;
    const T* a_a;
    const T* c_a;
};

// Per-source great-circle geometry: T0 = G*fun0, T0x = Gx*fun0, T0y = Gy*fun0.
template <class T>
struct Geometry {
    const T* G;
    const T* Gx;
    const T* Gy;
};

struct Events {
    int ne;
    const int* src;         // [ne] unique-source index (geometry plane)
    const int* iper;        // [ne]
    const double* evlo;     // [ne] degrees
    const double* evla;
    const int* rec_ptr;     // [ne+1]
    const int* rec_idx;     // [npair] station index
    const double* stlo;     // [nsta] degrees
    const double* stla;
    const double* cos_stla; // [nsta] cos(stla*DEG2RAD) (host C library)
    const double* tt_obs;   // [npair]
    const double* weight;   // [npair]
    const double* sadj;     // [npair] explicit adjoint sources (mode ADJ_ONLY; in
                            // FWD_ADJ they replace w*(Tsyn - Tobs)) or null
    const double* T_in;     // [ne][ny][nx] forward field input (mode ADJ_ONLY) or null
};

struct Outputs {
    double* syn;        // [npair] synthetic times (may be null in ADJ_ONLY)
    double* chi_ev;     // [ne] 0.5*sum(w r^2) per event (may be null)
    double* adj_s;      // [nper][ny][nx] accumulated Ta*svel^-3 (may be null)
    int* fwd_iters;     // [ne] (may be null)
    int* adj_iters;     // [ne] (may be null)
    int* status;        // [ne] (may be null)
    double* T_out;      // [ne][ny][nx] optional full forward field
    double* Ta_out;     // [ne][ny][nx] optional full adjoint field (unmasked)
    // deterministic accumulation: instead of adding into adj_s, each event
    // writes its masked Ta * svel^-3 plane to contrib[(e - contrib_e0)*n]
    // and an ordered reduction sums them in event order (may be null)
    double* contrib;
    int contrib_e0;
    // is_kden: [nper][ny][nx] accumulated kernel-density adjoint (may be null)
    double* kden_s;
};

enum Mode : int { MODE_FWD = 0, MODE_FWD_ADJ = 1, MODE_ADJ_ONLY = 2 };

// Per-warp scratch slot.  Planes of nx*ny elements of type T (sweep fields)
// plus FP64 planes where the reference's arithmetic must stay FP64.
struct Scratch {
    int nslots;            // event slots in use
    int nwarps;            // FP32 kernel with tail teams: warps launched (all slots)
    size_t slot_bytes;
    unsigned char* base;
    unsigned int* queue;   // work-queue counter (reset to 0 before each launch)
    const int* order;      // queue position -> event (NULL: identity)
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace sa
