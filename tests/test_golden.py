"""CPU: the oracle against golden fixtures produced by the reference's own
CUDA kernels (tests/golden/make_golden.py, run on a B200).  This pins the
oracle to the reference without a GPU: the outputs of the -nolto build must
be reproduced value for value (state, running extrema, simulated time and
next dt); the reference makefile recipe build (-dlto) within 1e-12 relative
per field with identical wet/dry flags."""
import glob
import os

import numpy as np
import pytest

import oracle
from tsuner_b200.abi import SimParams, TsuConsts, TsuSwitches

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# the time-step fixtures (nctr_*.npz pin the input pipeline: tests/test_nctr_cpu.py)
FIXTURES = sorted(f for f in glob.glob(os.path.join(HERE, "*.npz")) if not os.path.basename(f).startswith("nctr_"))
PFIELDS = ["xmin", "xmax", "ymin", "ymax", "total_time", "save_time", "npx", "npy", "nvol", "CFL", "Q", "R",
           "porosity", "DS", "FR", "Opar", "OC", "Dsg", "HQB", "vmax", "epsilon_h", "dx", "dy"]
# fixtures written before the Manning switch existed carry the first nine
SFIELDS = ["order", "rk", "wbc", "bedload", "suspension", "read_files", "bedload_law", "precision", "grass_ag",
           "manning"]
KFIELDS = ["vs", "Rp", "A_er", "sqrt_FR", "VP", "K_dep", "sqrt_OC", "DS5"]


def _struct(cls, fields, vals):
    s = cls()
    for f, v in zip(fields, vals):
        t = dict(cls._fields_)[f]
        setattr(s, f, int(v) if t.__name__ in ("c_int", "c_long") else float(v))
    return s


def test_fixtures_present():
    assert len(FIXTURES) >= 6, "golden fixtures missing (tests/golden/make_golden.py)"


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_reproduces_reference_build(path):
    d = np.load(path)
    p = _struct(SimParams, PFIELDS, d["params"])
    sw = _struct(TsuSwitches, SFIELDS, d["switches"])
    k = _struct(TsuConsts, KFIELDS, d["consts"])
    CC = d["CC"] if d["CC"].size else None
    tCC = d["tCC"] if d["tCC"].size else None
    r = oracle.OracleRun(p, sw, d["V_in"], d["mask"], CC, tCC, kconsts=k)
    r.run(int(d["steps"]))
    shp = (p.npy, p.npx)
    if sw.manning:
        # the Manning branch calls pow() per cell (GPU/Reconstructor.cu:48):
        # libm's and the device's may differ in the last bit, so this fixture
        # is held to 1e-12 relative per field instead of value for value
        for f in range(5):
            assert np.abs(r.V[f] - d["V_out"][f]).max() <= 1e-12 * max(np.abs(d["V_out"][f]).max(), 1e-300)
        assert np.array_equal(r.V[0] > p.epsilon_h, d["V_out"][0] > p.epsilon_h)
        assert abs(r.t.value - float(d["t"])) <= 1e-12 * float(d["t"])
        return
    assert np.array_equal(r.V, d["V_out"])
    assert np.array_equal(r.hmax.reshape(shp), d["hmax"])
    assert np.array_equal(r.bmin.reshape(shp), d["bmin"])
    assert np.array_equal(r.eta_max.reshape(shp), d["eta_max"])
    assert r.t.value == float(d["t"]) and r.dt.value == float(d["dt"])
    rec = d["V_out_recipe"]
    assert np.array_equal(r.V[0] > p.epsilon_h, rec[0] > p.epsilon_h)
    for f in range(5):
        assert np.abs(r.V[f] - rec[f]).max() <= 1e-12 * max(np.abs(rec[f]).max(), 1e-300)
    assert abs(r.t.value - float(d["t_recipe"])) <= 1e-12 * float(d["t_recipe"])


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_libm_constants_close_to_device(path):
    """libm pow() vs device pow(): the two per-run constants agree to a few ulp."""
    d = np.load(path)
    p = _struct(SimParams, PFIELDS, d["params"])
    k = oracle.consts(p)
    dev = dict(zip(KFIELDS, d["consts"]))
    for f in KFIELDS:
        assert abs(getattr(k, f) - dev[f]) <= 4 * np.spacing(abs(dev[f])), f
