"""GPU parity: eikonal:: drop-ins (single solves) against the CPU oracle.

Bar: FP64 path <= 1e-12 relative on T and Ta with the oracle's iteration
count; FP32 path <= 1e-5 relative on these continent-scale test grids (their
travel times reach ~1000 s)."""
import numpy as np
import pytest

from conftest import lin

pytestmark = pytest.mark.gpu
PI = np.pi


def grid_121x91():
    # tests/eikonal_test/test_eikonal.cpp:447-463
    nx, ny = 121, 91
    xx, yy = lin(nx, -30.0, 30.0), lin(ny, -20.0, 20.0)
    lon, lat = np.meshgrid(xx * PI / 180.0, yy * PI / 180.0)
    spha = 1.0 + 0.10 * np.sin(2.0 * lon) * np.cos(lat)
    sphb = 1.0 + 0.08 * np.cos(1.5 * lon) * np.sin(lat)
    sphc = 0.03 * np.sin(lon + lat)
    fun = 1.0 / (3.2 + 0.3 * np.cos(lat))
    return xx, yy, spha, sphb, sphc, fun, 0.3, -0.4


def grid_161x121():
    # tests/eikonal_test/test_eikonal.cpp:540-577
    nx, ny = 161, 121
    xx, yy = lin(nx, -35.0, 35.0), lin(ny, -25.0, 25.0)
    lon, lat = np.meshgrid(xx, yy)
    lonr, latr = lon * PI / 180.0, lat * PI / 180.0
    g1 = np.exp(-((lon - 10.0) ** 2 / (2.0 * 8.0 * 8.0) + (lat + 6.0) ** 2 / (2.0 * 5.0 * 5.0)))
    g2 = np.exp(-((lon + 14.0) ** 2 / (2.0 * 10.0 * 10.0) + (lat - 8.0) ** 2 / (2.0 * 7.0 * 7.0)))
    checker = np.sin(3.0 * lonr) * np.cos(2.5 * latr)
    vel = 3.35 + 0.10 * np.cos(1.7 * latr) + 0.08 * np.sin(1.3 * lonr) + 0.14 * g1 - 0.12 * g2 \
        + 0.05 * checker
    vel = np.clip(vel, 2.8, 4.2)
    spha = 1.0 + 0.12 * np.sin(2.0 * lonr) * np.cos(latr) + 0.03 * g1
    sphb = 1.0 + 0.10 * np.cos(1.5 * lonr) * np.sin(latr) - 0.02 * g2
    sphc = 0.04 * np.sin(lonr + latr) + 0.01 * checker
    return xx, yy, spha, sphb, sphc, 1.0 / vel, 1.2, -2.4


def homogeneous_61x41():
    xx, yy = lin(61, -30, 30), lin(41, -20, 20)
    o = np.ones((41, 61))
    return xx, yy, o, o, np.zeros_like(o), o / 3.0, 0.0, 0.0


def aniso_31():
    xx = lin(31, -15, 15)
    o = np.ones((31, 31))
    return xx, xx.copy(), o * 1.2, o * 0.9, o * 0.1, o / 3.0, 0.0, 0.0


def c1_like():
    # 0.05 deg grid, smooth velocity, off-node source
    xx, yy = 102.0 + 0.05 * np.arange(41), 24.0 + 0.05 * np.arange(41)
    X, Y = np.meshgrid(xx, yy)
    v = 3.2 + 0.2 * np.sin(X * 3) * np.cos(Y * 2)
    o = np.ones((41, 41))
    return xx, yy, o, o, np.zeros_like(o), 1.0 / v, 103.013, 24.987


CASES = {"121x91": grid_121x91, "161x121": grid_161x121, "homog": homogeneous_61x41,
         "aniso31": aniso_31, "c1like": c1_like}


def rel_err(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


@pytest.mark.parametrize("name", list(CASES))
def test_forward_fp64_matches_oracle(orc, gpu, name):
    from surfattpp_b200 import eikonal
    args = CASES[name]()
    T_ref, it_ref = orc.eik_fwd(*args)
    T, it = eikonal.FSM_UW_PS_lonlat_2d(*args, precision="fp64", return_iters=True)
    assert it == it_ref
    m = T_ref > 0
    assert rel_err(T[m], T_ref[m]) <= 1e-12
    assert np.all(T[~m] == T_ref[~m])


@pytest.mark.parametrize("name", list(CASES))
def test_forward_fp32_close_to_oracle(orc, gpu, name):
    from surfattpp_b200 import eikonal
    args = CASES[name]()
    T_ref, _ = orc.eik_fwd(*args)
    T = eikonal.FSM_UW_PS_lonlat_2d(*args, precision="fp32")
    m = T_ref > 1e-6
    assert rel_err(T[m], T_ref[m]) <= 1e-5


def _adj_case(orc, n=31):
    xx = lin(n, -10.0, 10.0)
    o = np.ones((n, n))
    z = np.zeros((n, n))
    T, _ = orc.eik_fwd(xx, xx, o, o, z, o / 3.0, 0.0, 0.0)
    return xx, o, z, T


@pytest.mark.parametrize("recs", [([5.0], [0.0], [1.0]),
                                  ([5.0, -5.0, 2.3], [0.0, 3.0, -7.7], [2.0, -1.5, 0.4])])
def test_adjoint_fp64_matches_oracle(orc, gpu, recs):
    from surfattpp_b200 import eikonal
    xx, o, z, T = _adj_case(orc)
    Ta_ref, it_ref = orc.eik_adj(xx, xx, o, o, z, T, *recs)
    Ta, it = eikonal.FSM_O1_JSE_lonlat_2d(xx, xx, o, o, z, T, *recs, precision="fp64",
                                          return_iters=True)
    assert it == it_ref
    scale = np.abs(Ta_ref).max()
    assert np.abs(Ta - Ta_ref).max() <= 1e-12 * scale
    # reference assertions (test_eikonal.cpp:384-400)
    assert np.isfinite(Ta).all()
    assert max(np.abs(Ta[0]).max(), np.abs(Ta[-1]).max(), np.abs(Ta[:, 0]).max(),
               np.abs(Ta[:, -1]).max()) < 1e-14


def test_adjoint_anisotropic_fp64(orc, gpu):
    from surfattpp_b200 import eikonal
    xx, yy, spha, sphb, sphc, fun, x0, y0 = grid_121x91()
    T, _ = orc.eik_fwd(xx, yy, spha, sphb, sphc, fun, x0, y0)
    rec = ([10.0, -12.5, 3.3], [5.0, -8.0, 12.0], [1.0, 0.5, -2.0])
    Ta_ref, it_ref = orc.eik_adj(xx, yy, spha, sphb, sphc, T, *rec)
    Ta, it = eikonal.FSM_O1_JSE_lonlat_2d(xx, yy, spha, sphb, sphc, T, *rec, precision="fp64",
                                          return_iters=True)
    assert it == it_ref
    assert np.abs(Ta - Ta_ref).max() <= 1e-12 * np.abs(Ta_ref).max()


def test_adjoint_zero_source_and_linearity(gpu, orc):
    from surfattpp_b200 import eikonal
    xx, o, z, T = _adj_case(orc, 21)
    Ta0 = eikonal.FSM_O1_JSE_lonlat_2d(xx, xx, o, o, z, T, [], [], [])
    assert np.abs(Ta0).max() < 1e-8
    a = eikonal.FSM_O1_JSE_lonlat_2d(xx, xx, o, o, z, T, [5.0], [0.0], [2.0])
    b = eikonal.FSM_O1_JSE_lonlat_2d(xx, xx, o, o, z, T, [-5.0], [3.0], [-1.5])
    ab = eikonal.FSM_O1_JSE_lonlat_2d(xx, xx, o, o, z, T, [5.0, -5.0], [0.0, 3.0], [2.0, -1.5])
    assert np.abs(a + b - ab).max() < 1e-8


def test_small_grid_raises(gpu):
    from surfattpp_b200 import eikonal
    o = np.ones((2, 5))
    with pytest.raises(ValueError):
        eikonal.FSM_UW_PS_lonlat_2d(lin(5, 0, 1), lin(2, 0, 1), o, o, o * 0, o, 0.5, 0.5)
