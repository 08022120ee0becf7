"""ctypes mirror of include/tsuner_b200.h (types and status codes).

The layouts here must match the C header field for field; tests check the
struct sizes against the values the library reports.
"""
import ctypes as C

TSU_OK = 0
TSU_ERR_GPU_OOM = 1
TSU_ERR_HOST_OOM = 2
TSU_ERR_INVALID = 3
TSU_ERR_CUDA = 4
TSU_ERR_NO_DEVICE = 5
TSU_ERR_NONFINITE = 6
TSU_ERR_IO = 7


class SimParams(C.Structure):
    """Layout-identical to `struct SimParams` (TSUNER.h:10-30)."""
    _fields_ = [
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("total_time", C.c_double), ("save_time", C.c_double),
        ("npx", C.c_int), ("npy", C.c_int), ("nvol", C.c_int),
        ("CFL", C.c_double), ("Q", C.c_double), ("R", C.c_double), ("porosity", C.c_double),
        ("DS", C.c_double), ("FR", C.c_double), ("Opar", C.c_double), ("OC", C.c_double),
        ("Dsg", C.c_double), ("HQB", C.c_double), ("vmax", C.c_double), ("epsilon_h", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double),
    ]


class TsuSwitches(C.Structure):
    _fields_ = [
        ("order", C.c_int), ("rk", C.c_int), ("wbc", C.c_int), ("bedload", C.c_int),
        ("suspension", C.c_int), ("read_files", C.c_int), ("bedload_law", C.c_int),
        ("precision", C.c_int), ("grass_ag", C.c_double), ("eta0", C.c_double),
        ("manning", C.c_int), ("reserved", C.c_int),
    ]


class TsuConsts(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("vs", "Rp", "A_er", "sqrt_FR", "VP", "K_dep", "sqrt_OC", "DS5")]


G = 9.81


def derive_params(p, friction_datdat):
    """Problem_loader.cxx:337-342: FR /= 8 (Chezy), HQB, Q, Opar."""
    p.FR = friction_datdat / 8.0
    p.HQB = 5.0 * p.DS
    p.Q = p.DS * (G * (p.R - 1.0) * p.DS) ** 0.5 / (1.0 - p.porosity)
    p.Opar = p.FR / ((p.R - 1.0) * G * p.DS)
    return p


def make_params(npx, npy, dx, dy, *, CFL=0.9, epsilon_h=1e-4, R=2.6, DS=2e-4, friction=2.5e-2,
                porosity=0.4, OC=0.0047, Dsg=100e-6, total_time=1e30, save_time=-1.0):
    """SimParams for an npx x npy Cartesian box [0, npx*dx] x [0, npy*dy] with
    the sediment values of the reference data.dat (data.dat:21-33)."""
    p = SimParams()
    p.xmin, p.xmax, p.ymin, p.ymax = 0.0, npx * dx, 0.0, npy * dy
    p.total_time, p.save_time = total_time, save_time
    p.npx, p.npy, p.nvol = npx, npy, npx * npy
    p.CFL, p.R, p.porosity, p.DS, p.OC, p.Dsg = CFL, R, porosity, DS, OC, Dsg
    p.vmax = 10.0
    p.epsilon_h = epsilon_h
    p.dx, p.dy = dx, dy
    derive_params(p, friction)
    return p


def make_switches(order=2, wbc=1, bedload=1, suspension=1, read_files=0, bedload_law=0,
                  precision=0, grass_ag=1e-3, rk=1, eta0=0.0, manning=0):
    s = TsuSwitches()
    s.eta0 = eta0
    s.manning = manning
    s.order, s.rk, s.wbc, s.bedload, s.suspension = order, rk, wbc, bedload, suspension
    s.read_files, s.bedload_law, s.precision, s.grass_ag = read_files, bedload_law, precision, grass_ag
    return s
