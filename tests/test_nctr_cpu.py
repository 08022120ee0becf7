"""CPU: the input pipeline (tsuner_b200/csrc/nctr.cpp: the arithmetic of the
reference's Read_files == 1 loader, Problem_loader.cxx:355-625 with
interpolations.cxx and tides.cxx) against the reference's own functions.

The reference functions are compiled unmodified from the reference checkout
into oracle/_ref/interp/libref_interp.so, with an in-memory netCDF stand-in
serving the grids its file reads ask for (oracle/ref_build/fake_netcdf.c).
Every step must agree value for value on seeded synthetic grids shaped like
the reference's example files: the grid interpolation, the fill-value fix of
the free surface, the boundary series CC (with fill values in the NCTR
grids), the sphere metrics, the Cartesian mappings of fields and of CC, the
whole loader chain (tsu_nctr_prepare), and the tide boundary values.  The
golden fixture tests/golden/nctr_pipeline.npz (written from the reference
functions by tests/golden/make_golden_nctr.py) pins the chain when the
reference build is absent."""
import ctypes as C
import os

import numpy as np
import pytest

import tsuner_b200 as T
from nctr_cases import REF_SO, Ref, grids, p

need_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref/interp not built")
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nctr_pipeline.npz")


def product_prepare(g):
    L = T.lib()
    npx, npy, nt = g["npx"], g["npy"], len(g["tgrid"])
    n = npx * npy
    sp = T.SimParams()
    h, H = np.zeros(n), np.zeros(n)
    hu = np.zeros(2 * n)
    fixH = np.zeros(n, np.int32)
    CC = np.zeros(nt * (2 * npx + 2 * npy) * 4)
    tCC = np.zeros(nt)
    rc = L.tsu_nctr_prepare(len(g["xb"]), len(g["yb"]), p(g["xb"]), p(g["yb"]), p(g["bathy"]), len(g["xf"]),
                            len(g["yf"]), p(g["xf"]), p(g["yf"]), p(g["fix"]), len(g["xc"]), len(g["yc"]), p(g["xc"]),
                            p(g["yc"]), nt, p(g["tgrid"]), p(g["ha"]), p(g["ua"]), p(g["va"]), npx, npy, g["slr"],
                            C.byref(sp), p(h), p(hu), p(H), p(fixH), p(CC), p(tCC))
    assert rc == 0
    box = np.array([sp.xmin, sp.xmax, sp.ymin, sp.ymax, sp.dx, sp.dy])
    assert (sp.npx, sp.npy, sp.nvol) == (npx, npy, n)
    return {"h": h, "H": H, "fixH": fixH, "CC": CC, "tCC": tCC, "box": box, "hu": hu}


@need_ref
def test_loader_chain_equals_the_reference():
    g = grids()
    ref, _ = Ref().loader(g)
    new = product_prepare(g)
    for k in ("h", "H", "fixH", "CC", "tCC", "box"):
        assert np.array_equal(new[k], ref[k]), k
    assert not new["hu"].any()
    assert (new["fixH"] == 0).any() and (new["fixH"] == 1).any()


@need_ref
def test_each_step_equals_the_reference():
    g = grids(seed=9, npx=53, npy=41)
    R = Ref()
    _, st = R.loader(g)
    L = T.lib()
    npx, npy, nt = g["npx"], g["npy"], len(g["tgrid"])
    xb, yb = g["xb"], g["yb"]
    dxg = (xb[-1] - xb[0]) / (len(xb) - 1)
    dyg = (yb[-1] - yb[0]) / (len(yb) - 1)
    xmin, xmax, ymin, ymax = xb[0] - 0.5 * dxg, xb[-1] + 0.5 * dxg, yb[0] - 0.5 * dyg, yb[-1] + 0.5 * dyg
    Hs = np.zeros(npx * npy)
    assert L.tsu_nctr_interp_grid(xmin, xmax, ymin, ymax, xmin, ymin, len(xb), len(yb), dxg, dyg, npx, npy,
                                  p(g["bathy"]), p(Hs)) == 0
    assert np.array_equal(Hs, st["H_geo"])
    xc, yc = g["xc"], g["yc"]
    dxc, dyc = (xc[-1] - xc[0]) / len(xc), (yc[-1] - yc[0]) / len(yc)
    es = np.zeros(npx * npy)
    L.tsu_nctr_interp_grid(xmin, xmax, ymin, ymax, xc[0], yc[0], len(xc), len(yc), dxc, dyc, npx, npy,
                           p(np.ascontiguousarray(g["ha"][0])), p(es))
    assert L.tsu_nctr_fix_eta(p(es), p(Hs), npx, npy, g["slr"]) == 0
    assert np.array_equal(es, st["eta_geo"])
    CC = np.zeros(nt * (2 * npx + 2 * npy) * 4)
    assert L.tsu_nctr_boundary_series(p(g["ha"]), p(g["ua"]), p(g["va"]), nt, len(xc), len(yc), xc[0], yc[0], dxc,
                                      dyc, npx, npy, xmin, xmax, ymin, ymax, p(Hs), g["slr"], p(CC)) == 0
    assert np.array_equal(CC, st["CC_geo"])
    dxE = np.zeros(npy)
    dmax, dyu = C.c_double(), C.c_double()
    dx, dy = (xmax - xmin) / npx, (ymax - ymin) / npy
    assert L.tsu_nctr_sphere_metrics(ymin, dy, npy, xmax, xmin, dx, p(dxE), C.byref(dyu), C.byref(dmax)) == 0
    assert np.array_equal(dxE, st["dxE"]) and dmax.value == st["dmax"] and dyu.value == st["dy_unit"]
    xm, xM, ym, yM = 0.0, dmax.value, 0.0, dyu.value * (ymax - ymin)
    Hc = np.zeros(npx * npy)
    assert L.tsu_nctr_to_cartesian(xm, xM, ym, yM, p(dxE), dy * dyu.value, npx, npy, p(Hs), p(Hc)) == 0
    assert np.array_equal(Hc, st["H_cart"])
    assert L.tsu_nctr_to_cartesian_series(xm, xM, ym, yM, p(dxE), dy * dyu.value, npx, npy, nt, p(CC)) == 0
    ref, _ = R.loader(g)
    assert np.array_equal(CC, ref["CC"])


@need_ref
def test_tides_equal_the_reference():
    rng = np.random.default_rng(3)
    nxt, nyt, npt, npx, npy = 20, 16, 6, 33, 27
    tides = rng.normal(0, 0.5, (npt, nyt, nxt))
    tides[2, 0, 3] = 3e5  # above the 1e5 limit: zeroed on the boundary
    xp = np.linspace(-124.4, -123.6, nxt)
    yp = np.linspace(46.6, 47.2, nyt)
    R = Ref()
    R.dataset("tides.nc", [("lon", nxt), ("lat", nyt), ("time", npt)],
              [("lon", xp), ("lat", yp), ("time", np.arange(npt) * 600.0), ("tides", tides)])
    box = (-124.5, -123.5, 46.5, 47.3)
    nseg = 2 * npx + 2 * npy
    ref = np.zeros(npt * nseg)
    eta = np.zeros(nxt * nyt)
    assert R.L.ref_tides_prep(p(eta), b"tides.nc", npx, npy, *box, p(ref), ref.size) == npt
    new = np.zeros(npt * nseg)
    assert T.lib().tsu_nctr_tides(p(tides), nxt, nyt, npt, p(xp), npx, npy, *box, p(new)) == 0
    assert np.array_equal(new, ref)


def test_loader_chain_equals_the_golden_fixture():
    if not os.path.exists(GOLDEN):
        pytest.skip("golden fixture not written (tests/golden/make_golden_nctr.py)")
    d = np.load(GOLDEN)
    g = {k: d["in_" + k] for k in ("xb", "yb", "bathy", "xf", "yf", "fix", "xc", "yc", "tgrid", "ha", "ua", "va")}
    g.update(npx=int(d["npx"]), npy=int(d["npy"]), slr=float(d["slr"]))
    new = product_prepare(g)
    for k in ("h", "H", "fixH", "CC", "tCC", "box"):
        assert np.array_equal(new[k], d[k]), k


def test_invalid_arguments_are_refused():
    L = T.lib()
    z = np.zeros(4)
    assert L.tsu_nctr_interp_grid(0, 1, 0, 1, 0, 0, 2, 2, 0.5, 0.5, 0, 2, p(z), p(z)) == T.abi.TSU_ERR_INVALID
    assert L.tsu_nctr_fix_eta(None, p(z), 2, 2, 0.0) == T.abi.TSU_ERR_INVALID
