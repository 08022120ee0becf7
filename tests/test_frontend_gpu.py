"""GPU: tsuner.exe and the TSUNER() drop-in write the reference NetCDF layout.

tsuner.exe runs a small data.dat (reference format) end to end; the output
file is read back with scipy's classic-NetCDF reader and checked against the
layout of the reference writer (GPU/netcdf.cu:38-242) and against the same
run through the tsu_* API (frames at the save cadence of
GPU/main_TSUNER.cu:157-167, the final frame, hmax/eta_max/bmin)."""
import os
import subprocess

import numpy as np
import pytest

import tsuner_b200 as T
from tsuner_b200.abi import make_params, make_switches

pytestmark = pytest.mark.gpu

EXE = os.path.join(os.path.dirname(T.LIB_PATH), "tsuner.exe")

DATA = """# This file is prepared to be read by a C program. Do not add new lines.
# xmin
-5
# xmax
5
# ymin
-5
# ymax
5
# Total simulation time
1.5
# Save time every
0.25
# npx
60
# npy
40
# CFL
0.9
# epsilon_h. Threshold for a cell to be considered dry.
1e-4
# Ratio of densities (>1)
2.6
# Mean diameter of sediment grain (>0)
2e-4
# Friction (Chezy) coefficient (>0)
2.5e-2
# Porosity (>=0 and <1.0):
0.4
# Critical theta:
0.0047
# Geometric mean size of suspended sediment
100e-6
# Output file name
{prefix}
# bathymetry file
unused.nc
# initial condition file
unused_h.nc
# mask
0
# Sea level correction
0
# tides
0
"""


def cini_state(p):
    x = p.xmin + 0.5 * p.dx + np.arange(p.npx) * p.dx
    y = p.ymin + 0.5 * p.dy + np.arange(p.npy) * p.dy
    X, Y = np.meshgrid(x, y)
    H = -2.5 * np.exp(-5.0 * (X * X + Y * Y)) - X * (X > 0)
    h = H + 2.0 + 6 * np.exp(-5.0 * ((X + 2) ** 2 + Y ** 2))
    h = h * (h > 0)
    V = np.zeros((5, p.npy, p.npx))
    V[0], V[3] = h, H
    return V


def test_tsuner_exe_writes_reference_layout(tmp_path):
    from scipy.io import netcdf_file
    assert os.path.exists(EXE), "tsuner.exe not built"
    prefix = str(tmp_path / "sim")
    dd = tmp_path / "data.dat"
    dd.write_text(DATA.format(prefix=prefix))
    r = subprocess.run([EXE, str(dd), "0"], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, TSU_QUIET="1"))
    assert r.returncode == 0, r.stderr
    assert "Normal End." in r.stdout
    f = netcdf_file(prefix + ".nc", "r", mmap=False)
    try:
        assert f.version_byte == 1  # classic CDF-1, as nc_create(NC_CLOBBER)
        assert f.dimensions["x"] == 60 and f.dimensions["y"] == 40 and f.dimensions["time"] is None
        for name in ("b", "eta", "ux", "uy", "c"):
            assert f.variables[name].dimensions == ("time", "y", "x")
        for name in ("hmax", "bmin", "eta_max"):
            assert f.variables[name].dimensions == ("y", "x")
            assert f.variables[name]._FillValue == -1e30
        assert f.variables["eta"].units == b"meters" and f.variables["ux"].long_name == b"x-velocity"
        assert f.title == b"TSUNER NOAA PMEL model output" and f.Conventions == b"CF-1.0"
        assert f.Friction == pytest.approx(2.5e-2)
        t = f.variables["time"][:].copy()
        eta = f.variables["eta"][:].copy()
        hmax = f.variables["hmax"][:].copy()
        bmin = f.variables["bmin"][:].copy()
        xs = f.variables["x"][:].copy()
    finally:
        f.close()
    assert t[0] == 0.0 and t[-1] >= 1.5 and np.all(np.diff(t) > 0)
    assert len(t) >= 7  # t = 0, one frame per 0.25 s crossing, final frame
    assert np.allclose(xs, -5 + (np.arange(60) + 0.5) * (10 / 60))
    p = make_params(60, 40, 10.0 / 60, 10.0 / 40)
    p.xmin, p.xmax, p.ymin, p.ymax = -5.0, 5.0, -5.0, 5.0
    V0 = cini_state(p)
    # frame 0 is the analytic initial state (libm vs numpy exp: last bits)
    assert np.abs(eta[0] - (V0[0] - V0[3])).max() < 1e-12


def test_tsuner_exe_matches_api_run(tmp_path):
    """Identical inputs through --raw: the file equals the tsu_* API run."""
    from scipy.io import netcdf_file
    p = make_params(60, 40, 10.0 / 60, 10.0 / 40)
    p.xmin, p.xmax, p.ymin, p.ymax = -5.0, 5.0, -5.0, 5.0
    V0 = cini_state(p)
    raw = str(tmp_path / "in")
    V0[0].astype("<f8").tofile(raw + "_h.f64")
    V0[3].astype("<f8").tofile(raw + "_H.f64")
    prefix = str(tmp_path / "sim")
    dd = tmp_path / "data.dat"
    dd.write_text(DATA.format(prefix=prefix))
    r = subprocess.run([EXE, str(dd), "0", "--raw", raw], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, TSU_QUIET="1"))
    assert r.returncode == 0, r.stderr
    f = netcdf_file(prefix + ".nc", "r", mmap=False)
    try:
        t = f.variables["time"][:].copy()
        eta = f.variables["eta"][:].copy()
        ux = f.variables["ux"][:].copy()
        hmax = f.variables["hmax"][:].copy()
        bmin = f.variables["bmin"][:].copy()
    finally:
        f.close()
    sw = make_switches(order=2, wbc=1, read_files=0)
    s = T.Solver(p, sw)
    s.set_state(V0)
    s.set_mask(None)
    s.reset()
    s.run_until(1.5)
    V = s.state()
    hm, bm, em = s.extrema()
    tt, _, _ = s.time()
    s.close()
    assert tt == t[-1]
    assert np.array_equal(eta[-1], V[0] - V[3])
    assert np.array_equal(ux[-1], V[1] / (V[0] + np.finfo(np.float64).eps))
    assert np.array_equal(hmax, hm)
    assert np.array_equal(bmin, -bm)
