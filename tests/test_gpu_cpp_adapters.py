"""The C++ side of the drop-in boundary: tests/cpp/adapters_test.cpp, plain
C++20 compiled against include/surfatt_gpu.h and linked to
libsurfatt_gpu.so (tests/cpp/Makefile), holds adapters in the reference's
layouts -- SurfGrid::svel [(ix*ny + iy)*nper + iper], SrcRec::events_local
as a std::map, column-major nx x ny planes -- for SurfGrid::fwdsurf,
preproc::forward_for_event, Inversion::run_forward_adjoint and
eikonal::FSM_UW_PS_lonlat_2d, and loads the reference's example table
through sa_srcrec_load.  Run on the checkerboard case (FP64) and checked
against the oracle: phase velocities bit-identical; travel times, misfit
and the single solve 1e-12 relative; adj_s within the batch tests' error
bound; ker_vs 1e-12 of its maximum."""
import os
import subprocess

import numpy as np
import pytest

from test_gpu_batch import adj_bound, assert_within

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_build", "adapters_test")


def _binary():
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "cpp")], check=True)
    return BIN


def _write(path, header, arrays):
    with open(path, "wb") as f:
        for v in header:
            f.write(np.int64(v).tobytes())
        for a, dt in arrays:
            a = np.ascontiguousarray(a, dtype=dt).ravel()
            f.write(np.int64(a.size).tobytes())
            f.write(a.tobytes())


def _read(path, count):
    out = []
    with open(path, "rb") as f:
        for _ in range(count):
            n = int(np.frombuffer(f.read(8), np.int64)[0])
            out.append(np.frombuffer(f.read(8 * n), np.float64).copy())
    return out


def test_cpp_adapters_against_oracle(gpu, orc, tmp_path):
    from surfattpp_b200 import workloads as W
    w = W.config1()
    m11, m12, m22 = w.media()
    ev = w.events()
    sv_true, _ = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8)
    ev["tt_obs"] = orc.forward_for_events(w.xx_deg, w.yy_deg, sv_true, m11, m12, m22, ev,
                                          calc_adj=False, nthreads=8)["syn"].copy()
    vs0 = w.meta["vs_start"]
    nx, ny, nz = vs0.shape
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    _write(inp, (nx, ny, nz),
           [(w.xx_deg, np.float64), (w.yy_deg, np.float64), (w.zgrid, np.float64),
            (w.periods, np.float64), (vs0, np.float64), (ev["evlo"], np.float64),
            (ev["evla"], np.float64), (ev["iper"], np.int32), (ev["rec_ptr"], np.int32),
            (ev["rec_idx"], np.int32), (ev["stlo"], np.float64), (ev["stla"], np.float64),
            (ev["tt_obs"], np.float64), (ev["weight"], np.float64)])
    csv = os.path.join(HERE, "golden", "src_rec_file_ph.csv")
    r = subprocess.run([_binary(), str(inp), str(outp), csv], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    assert "table 4800 observations 16 periods 384 events first MX00_0 last MX23_9" in r.stdout
    svel, syn, adj, chis, ker, T = _read(outp, 6)
    # oracle chain
    sv0, _ = orc.fwdsurf(w.zgrid, vs0, w.periods, nthreads=8)
    ref = orc.forward_for_events(w.xx_deg, w.yy_deg, sv0, m11, m12, m22, ev, calc_adj=True,
                                 nthreads=8)
    assert np.array_equal(svel.reshape(nx, ny, w.nper).transpose(2, 1, 0), sv0)
    assert np.max(np.abs(syn - ref["syn"]) / np.abs(ref["syn"])) <= 1e-12
    for c in chis:
        assert abs(c - ref["chi"]) <= 1e-12 * abs(ref["chi"])
    bound = adj_bound(orc, w, sv0, ev, ref, syn)
    assert_within(adj.reshape(w.nper, ny, nx), ref["adj_s"], 2.0 * bound + 1e-300)
    sen = orc.depthkernel_hti(w.zgrid, vs0, w.periods, nthreads=8)
    vp0 = np.vectorize(orc.vs2vp)(vs0)
    kref = orc.combine_kernels_vs(ref["adj_s"], vs0, vp0, *sen[:3])
    assert np.abs(ker.reshape(nx, ny, nz) - kref).max() <= 1e-12 * np.abs(kref).max()
    ip = int(ev["iper"][0])
    one, zero = np.ones((ny, nx)), np.zeros((ny, nx))
    Tref, _ = orc.eik_fwd(w.xx_deg, w.yy_deg, one, one, zero, 1.0 / sv0[ip], ev["evlo"][0],
                          ev["evla"][0])
    T = T.reshape(ny, nx)
    m = Tref > 0
    assert np.max(np.abs(T[m] - Tref[m]) / Tref[m]) <= 1e-12
