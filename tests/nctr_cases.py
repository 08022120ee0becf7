"""Seeded synthetic inputs of the input pipeline (the reference's
Read_files == 1 loader): a bathymetry grid, a non-erodible-bed grid and NCTR
free-surface / velocity grids in geographic coordinates, shaped like the
reference's example files (which are NetCDF4/HDF5 and cannot be read here),
plus the reference's own functions driven on them through
oracle/_ref/interp/libref_interp.so.  Shared by tests/test_nctr_cpu.py and
tests/golden/make_golden_nctr.py."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "interp", "libref_interp.so")


def grids(seed=5, nxb=60, nyb=50, nxf=40, nyf=30, nxc=30, nyc=25, ntime=8, npx=48, npy=36):
    rng = np.random.default_rng(seed)
    g = {"npx": npx, "npy": npy, "slr": 0.25}
    # bathymetry: lon -124.5 .. -123.5, lat 46.5 .. 47.3 (cell centres), depth below datum in metres
    g["xb"] = np.linspace(-124.5, -123.5, nxb)
    g["yb"] = np.linspace(46.5, 47.3, nyb)
    X, Y = np.meshgrid(g["xb"], g["yb"])
    g["bathy"] = 40.0 * (-123.6 - X) + 5.0 * np.sin(7 * Y) + rng.normal(0, 0.3, X.shape)
    # non-erodible blocks on a coarser, shifted grid
    g["xf"] = np.linspace(-124.45, -123.55, nxf)
    g["yf"] = np.linspace(46.55, 47.25, nyf)
    fix = np.ones((nyf, nxf))
    fix[5:12, 8:20] = 0.0
    fix[18:24, 25:33] = 0.0
    g["fix"] = fix
    # NCTR grids in centimetres, with fill values where the model is dry
    g["xc"] = np.linspace(-124.6, -123.4, nxc)
    g["yc"] = np.linspace(46.45, 47.35, nyc)
    g["tgrid"] = np.arange(ntime, dtype=np.float64) * 30.0
    t = g["tgrid"][:, None, None]
    Xc, Yc = np.meshgrid(g["xc"], g["yc"])
    ha = 80.0 * np.sin(0.01 * t + 3 * Xc) * np.cos(4 * Yc) + rng.normal(0, 1.0, (ntime, nyc, nxc))
    ua = 30.0 * np.cos(0.02 * t + 2 * Yc) + 0 * Xc
    va = 20.0 * np.sin(0.015 * t + 5 * Xc) + 0 * Yc
    dry = Xc > -123.5
    ha[:, dry] = -1.0e34
    ua[:, dry] = 1.0e35
    va[:, dry] = -1.0e35
    g["ha"], g["ua"], g["va"] = ha, ua, va
    return g


def p(a):
    return None if a is None else np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)


_KEEP = []  # arrays the in-memory netCDF datasets point at, alive for the process


class Ref:
    """The reference's own functions (oracle/_ref/interp, test infrastructure).
    The in-memory netCDF registry is process-wide; registering a path again
    replaces its dataset."""

    def __init__(self):
        L = C.CDLL(REF_SO)
        d, i, vp = C.c_double, C.c_int, C.c_void_p
        L.ref_interpolate_spherics.argtypes = [d] * 6 + [i] * 2 + [d] * 2 + [i] * 2 + [vp, vp]
        L.ref_fix_eta.argtypes = [vp, vp, i, i, d]
        L.ref_interpolate_CC.argtypes = [C.c_char_p, vp, vp, i, i] + [d] * 6 + [C.c_ulong, d, d, vp, i, d]
        L.ref_spheric2cartesian.argtypes = [d] * 4 + [vp, d, i, i, vp, vp]
        L.ref_spheric2cartesian_CC.argtypes = [d] * 4 + [vp, d, i, i, i, vp]
        L.ref_transforms.argtypes = [d, d, i, d, d, vp, d, C.POINTER(d), C.POINTER(d)]
        L.ref_tides_prep.argtypes = [vp, C.c_char_p, i, i, d, d, d, d, vp, C.c_size_t]
        L.ref_tides_prep.restype = C.c_int
        L.fake_nc_dataset.argtypes = [C.c_char_p]
        L.fake_nc_dataset.restype = C.c_int
        L.fake_nc_dim.argtypes = [i, C.c_char_p, C.c_size_t]
        L.fake_nc_var.argtypes = [i, C.c_char_p, vp, C.c_size_t]
        L.fake_nc_set_boundaries.argtypes = [i, i]
        self.L = L

    def dataset(self, path, dims, variables):
        """Registers an in-memory netCDF file; returns its ncid (index + 1)."""
        ds = self.L.fake_nc_dataset(path.encode())
        for name, n in dims:
            self.L.fake_nc_dim(ds, name.encode(), n)
        for name, arr in variables:
            a = np.ascontiguousarray(arr, np.float64)
            _KEEP.append(a)
            self.L.fake_nc_var(ds, name.encode(), p(a), a.size)
        return ds + 1

    def loader(self, g):
        """The reference's Read_files == 1 loader steps (Problem_loader.cxx:
        396-605, SPL = 0) on the grids g, with the reference functions."""
        L, npx, npy, slr = self.L, g["npx"], g["npy"], g["slr"]
        xb, yb = g["xb"], g["yb"]
        nxb, nyb = len(xb), len(yb)
        dxg = (xb[-1] - xb[0]) / (nxb - 1)
        dyg = (yb[-1] - yb[0]) / (nyb - 1)
        xmin, xmax = xb[0] - 0.5 * dxg, xb[-1] + 0.5 * dxg
        ymin, ymax = yb[0] - 0.5 * dyg, yb[-1] + 0.5 * dyg
        n = npx * npy
        Hs, fs, es = np.zeros(n), np.zeros(n), np.zeros(n)
        bat = np.ascontiguousarray(g["bathy"], np.float64)
        L.ref_interpolate_spherics(xmin, xmax, ymin, ymax, xmin, ymin, nxb, nyb, dxg, dyg, npx, npy, p(bat), p(Hs))
        xf, yf = g["xf"], g["yf"]
        dxf = (xf[-1] - xf[0]) / (len(xf) - 1)
        dyf = (yf[-1] - yf[0]) / (len(yf) - 1)
        fx = np.ascontiguousarray(g["fix"], np.float64)
        L.ref_interpolate_spherics(xmin, xmax, ymin, ymax, xf[0], yf[0], len(xf), len(yf), dxf, dyf, npx, npy, p(fx),
                                   p(fs))
        xc, yc = g["xc"], g["yc"]
        nxc, nyc, nt = len(xc), len(yc), len(g["tgrid"])
        dxc = (xc[-1] - xc[0]) / nxc
        dyc = (yc[-1] - yc[0]) / nyc
        ha0 = np.ascontiguousarray(g["ha"][0], np.float64)
        L.ref_interpolate_spherics(xmin, xmax, ymin, ymax, xc[0], yc[0], nxc, nyc, dxc, dyc, npx, npy, p(ha0), p(es))
        L.ref_fix_eta(p(es), p(Hs), npx, npy, slr)
        dims = [("lat", nyc), ("lon", nxc), ("time", nt)]
        hid = self.dataset("nctr_h.nc", dims, [("ha", g["ha"])])
        self.dataset("nctr_u.nc", dims, [("time", g["tgrid"]), ("ua", g["ua"])])
        self.dataset("nctr_v.nc", dims, [("va", g["va"])])
        CC = np.zeros(nt * (2 * npx + 2 * npy) * 4)
        tCC = np.zeros(nt)
        L.ref_interpolate_CC(b"nctr_h.nc", p(CC), p(tCC), npx, npy, xmin, xmax, ymin, ymax, xc[0], yc[0], nt, dxc, dyc,
                             p(Hs), hid, slr)
        stage = {"H_geo": Hs.copy(), "fix_geo": fs.copy(), "eta_geo": es.copy(), "CC_geo": CC.copy(), "tCC": tCC}
        dx = (xmax - xmin) / npx
        dy = (ymax - ymin) / npy
        dxE = np.zeros(npy)
        dmax, dyu = C.c_double(), C.c_double()
        L.ref_transforms(ymin, dy, npy, xmax, xmin, p(dxE), dx, C.byref(dmax), C.byref(dyu))
        xmin, xmax = 0.0, dmax.value
        ymax, ymin = dyu.value * (ymax - ymin), 0.0
        dyE = dy * dyu.value
        Hc, fc, ec = np.zeros(n), np.zeros(n), np.zeros(n)
        L.ref_spheric2cartesian(xmin, xmax, ymin, ymax, p(dxE), dyE, npx, npy, p(Hs), p(Hc))
        L.ref_spheric2cartesian(xmin, xmax, ymin, ymax, p(dxE), dyE, npx, npy, p(fs), p(fc))
        L.ref_spheric2cartesian(xmin, xmax, ymin, ymax, p(dxE), dyE, npx, npy, p(es), p(ec))
        L.ref_spheric2cartesian_CC(xmin, xmax, ymin, ymax, p(dxE), dyE, npx, npy, nt, p(CC))
        # the value assignment of Problem_loader.cxx:576-605, restated
        H = Hc.copy()
        h = ec * 0.01 + H + slr
        h = h * (h >= 0.0)
        fixH = (fc >= 0.5).astype(np.int32)
        stage.update(dxE=dxE, dmax=dmax.value, dy_unit=dyu.value, H_cart=Hc, eta_cart=ec, fix_cart=fc)
        out = {"h": h, "H": H, "fixH": fixH, "CC": CC, "tCC": tCC,
               "box": np.array([xmin, xmax, ymin, ymax, (xmax - xmin) / npx, (ymax - ymin) / npy])}
        return out, stage
