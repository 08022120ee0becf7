"""Generates the golden fixtures tests/golden/*.npz from the reference's own
CUDA build (oracle/_ref/<variant>/libtsuner_ref.so: the unmodified reference
kernels driven step by step).  Needs a GPU; run on the B200 box:

    python tests/golden/make_golden.py [output_dir]

Each fixture stores the inputs (state, mask, boundary series, SimParams,
switches), the step count, the outputs of the -nolto build of the reference
kernels (state, running extrema, t, next dt), the state and t of the
reference makefile recipe build (-dlto), and the per-run sediment constants as the device evaluates them
(TsuConsts from the product's constants kernel: device pow(), the same
function the reference kernels call per cell).  tests/test_golden.py replays
them through the CPU oracle without a GPU.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
import tsuner_b200 as T  # noqa: E402
from tsuner_b200 import workloads as W  # noqa: E402
from tsuner_b200.abi import make_switches  # noqa: E402

# name -> (variant, workload factory, switches, steps)
CASES = {
    "walls_hump_40x30": ("default", lambda: W.hump(40, 30, 10.0, sigma=70.0),
                         dict(order=2, wbc=1, read_files=0), 40),
    "nwave_48x36": ("default", lambda: W.nwave_shelf(48, 36, 40.0, slr=0.5, amp=2.0, period=200.0, t_series=150.0),
                    dict(order=2, wbc=1, read_files=1), 60),
    "nwave_expiring_44x32": ("default", lambda: W.nwave_shelf(44, 32, 40.0, slr=0.5, amp=2.0, period=200.0,
                                                              t_series=8.0), dict(order=2, wbc=1, read_files=1), 60),
    "free_36x28": ("rf0_wbc0", lambda: W.hump(36, 28, 10.0, sigma=60.0), dict(order=2, wbc=0, read_files=0), 40),
    "periodic_32x24": ("rf0_wbc2", lambda: W.hump(32, 24, 10.0, sigma=60.0), dict(order=2, wbc=2, read_files=0), 40),
    "order1_40x24": ("order1", lambda: W.nwave_shelf(40, 24, 40.0, slr=0.5, amp=2.0, period=200.0, t_series=150.0),
                     dict(order=1, wbc=1, read_files=1), 50),
    "nosed_40x24": ("nosed", lambda: W.nwave_shelf(40, 24, 40.0, slr=0.5, amp=2.0, period=200.0, t_series=150.0),
                    dict(order=2, wbc=1, read_files=1, bedload=0, suspension=0), 50),
    "above4096_72x64": ("default", lambda: W.hump(72, 64, 10.0, sigma=120.0), dict(order=2, wbc=1, read_files=0), 30),
    "hancock_nwave_48x36": ("rk0", lambda: W.nwave_shelf(48, 36, 40.0, slr=0.5, amp=2.0, period=200.0,
                                                         t_series=150.0), dict(order=2, wbc=1, read_files=1, rk=0), 60),
    "hancock_o1_40x24": ("rk0_order1", lambda: W.nwave_shelf(40, 24, 40.0, slr=0.5, amp=2.0, period=200.0,
                                                             t_series=150.0), dict(order=1, wbc=1, read_files=1, rk=0),
                         50),
    "manning_hump_40x30": ("manning_rf0", lambda: W.hump(40, 30, 10.0, sigma=70.0),
                           dict(order=2, wbc=1, read_files=0, manning=1), 40),
}

PFIELDS = ["xmin", "xmax", "ymin", "ymax", "total_time", "save_time", "npx", "npy", "nvol", "CFL", "Q", "R",
           "porosity", "DS", "FR", "Opar", "OC", "Dsg", "HQB", "vmax", "epsilon_h", "dx", "dy"]
SFIELDS = ["order", "rk", "wbc", "bedload", "suspension", "read_files", "bedload_law", "precision", "grass_ag",
           "manning"]
KFIELDS = ["vs", "Rp", "A_er", "sqrt_FR", "VP", "K_dep", "sqrt_OC", "DS5"]


def main(out=HERE):
    os.makedirs(out, exist_ok=True)
    for name, (variant, make, swd, steps) in CASES.items():
        w = make()
        sw = make_switches(**swd)
        if swd.get("read_files"):
            CC, tCC = w.CC, w.tCC
        else:
            CC, tCC = W.expired_series(w.p.npx, w.p.npy) if variant == "default" else (None, None)
        if not (oracle.ref_available(variant) and oracle.ref_available(variant + "-nolto")):
            print("skip", name, "(variant %s not built)" % variant)
            continue
        r = oracle.ref_run(variant + "-nolto", w.p, w.V, w.mask, CC, tCC, steps)
        rl = oracle.ref_run(variant, w.p, w.V, w.mask, CC, tCC, steps)
        with T.Solver(w.p, sw) as s:
            k = s.consts()
        np.savez_compressed(
            os.path.join(out, name + ".npz"),
            variant=variant, steps=steps, V_in=w.V, mask=w.mask,
            CC=(w.CC if swd.get("read_files") else np.zeros(0)),
            tCC=(w.tCC if swd.get("read_files") else np.zeros(0)),
            params=np.array([float(getattr(w.p, f)) for f in PFIELDS]),
            switches=np.array([float(getattr(sw, f)) for f in SFIELDS]),
            consts=np.array([getattr(k, f) for f in KFIELDS]),
            V_out=r["V"], hmax=r["hmax"], bmin=r["bmin"], eta_max=r["eta_max"], t=r["t"], dt=r["dt"],
            V_out_recipe=rl["V"], t_recipe=rl["t"])
        print("wrote", name, "t=%.6f" % r["t"])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
