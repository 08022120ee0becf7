"""Writes tests/golden/nctr_pipeline.npz: the inputs and the outputs of the
reference's Read_files == 1 loader chain (its own interpolation functions,
oracle/_ref/interp/libref_interp.so, built by oracle/build_ref.py from the
reference checkout) on the seeded synthetic grids of tests/nctr_cases.py.
Runs on the CPU:

    python tests/golden/make_golden_nctr.py [output_dir]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from nctr_cases import Ref, grids  # noqa: E402


def main(out=HERE):
    g = grids()
    ref, _ = Ref().loader(g)
    arrays = {"in_" + k: g[k] for k in ("xb", "yb", "bathy", "xf", "yf", "fix", "xc", "yc", "tgrid", "ha", "ua", "va")}
    arrays.update(npx=g["npx"], npy=g["npy"], slr=g["slr"], **ref)
    path = os.path.join(out, "nctr_pipeline.npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
