"""CPU tests of the C ABI: the product library loads, exports every function
include/tsuner_b200.h declares, agrees with the Python struct mirror, and
its host-only entry points (status strings, data.dat parser, device probe)
behave.  No kernel is launched here."""
import ctypes as C
import os
import re

import pytest

import tsuner_b200
from tsuner_b200.abi import SimParams, TsuConsts, TsuSwitches

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "tsuner_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src))
    return sorted(n for n in names if n.startswith("tsu_") or n in ("TSUNER", "checkCUDAsupport", "initializeGPU"))


def test_every_declared_symbol_is_exported(product_lib):
    decl = declared_functions()
    assert "TSUNER" in decl and "tsu_step" in decl
    missing = [n for n in decl if not hasattr(product_lib, n)]
    assert not missing, missing
    assert set(decl) == set(tsuner_b200.EXPORTS)


def test_struct_layouts_match(product_lib):
    out = (C.c_size_t * 3)()
    assert product_lib.tsu_struct_sizes(out) == 0
    assert list(out) == [C.sizeof(SimParams), C.sizeof(TsuSwitches), C.sizeof(TsuConsts)]
    # TSUNER.h:10-30 layout: 6 doubles, 3 ints (+pad), 14 doubles
    assert C.sizeof(SimParams) == 176
    assert SimParams.CFL.offset == 64 and SimParams.dy.offset == 168


def test_default_switches_are_the_reference_defaults(product_lib):
    sw = TsuSwitches()
    assert product_lib.tsu_switches_default(C.byref(sw)) == 0
    # Sim_parameters.hxx:45-54
    assert (sw.order, sw.rk, sw.wbc, sw.bedload, sw.suspension, sw.read_files) == (2, 1, 1, 1, 1, 1)
    assert sw.precision == 0 and sw.bedload_law == 0


def test_strerror(product_lib):
    assert product_lib.tsu_strerror(0) == b"ok"
    assert product_lib.tsu_strerror(1) == b"not enough GPU memory"
    assert product_lib.tsu_strerror(2) == b"not enough CPU memory"


DATA_DAT = """# This file is read by a C program.
# xmin
-5
# xmax
5
# ymin
-5
# ymax
5
# Total simulation time
7200
# Save time every
20
# npx
100
# npy
80
# CFL
0.9
# epsilon_h
1e-4
# Ratio of densities (>1)
2.6
# Mean diameter of sediment grain (>0)
2e-4
# Friction (Chezy) coefficient (>0)
2.5e-2
# Porosity
0.4
# Critical theta
0.0047
# Geometric mean size of suspended sediment
100e-6
# Output file name
sim
# bathymetry file
./bathy.nc
# IC file
./ic_h.nc
# mask file
0
# sea level correction
0.5
# tides file
0
"""


def test_parse_data_dat(product_lib, tmp_path):
    f = tmp_path / "data.dat"
    f.write_text(DATA_DAT)
    p = SimParams()
    bufs = [C.create_string_buffer(256) for _ in range(5)]
    slr = C.c_double()
    rc = product_lib.tsu_parse_data_dat(str(f).encode(), C.byref(p), bufs[0], bufs[1], bufs[2], bufs[3],
                                        C.byref(slr), bufs[4], 256)
    assert rc == 0
    assert (p.npx, p.npy, p.nvol) == (100, 80, 8000)
    assert p.total_time == 7200 and p.save_time == 20 and p.CFL == 0.9
    assert p.FR == 2.5e-2 / 8.0  # Problem_loader.cxx:338
    assert p.HQB == 5.0 * 2e-4
    assert p.Q == 2e-4 * (9.81 * 1.6 * 2e-4) ** 0.5 / 0.6
    assert p.dx == 10.0 / 100 and p.dy == 10.0 / 80
    assert bufs[0].value == b"sim" and bufs[1].value == b"./bathy.nc" and bufs[3].value == b"0"
    assert slr.value == 0.5
    f.write_text(DATA_DAT.split("# Output")[0])
    assert product_lib.tsu_parse_data_dat(str(f).encode(), C.byref(p), None, None, None, None, None, None, 0) == 3


def test_device_probe_contract(product_lib):
    rc = product_lib.checkCUDAsupport(0)
    assert rc in (0, 1, 2, 3)
    if rc == 1:  # no GPU here: creating a solver fails cleanly with a status
        h = C.c_void_p()
        p = tsuner_b200.make_params(8, 8, 1.0, 1.0)
        sw = tsuner_b200.make_switches()
        assert product_lib.tsu_create(C.byref(h), C.byref(p), C.byref(sw), 0) == 5
