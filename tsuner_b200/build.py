"""Builds the in-tree product library tsuner_b200/libtsuner_b200.so (sm_100a).

  python -m tsuner_b200.build [--force]

Every .cu/.cpp under csrc/ is compiled separately (the FP64 plain-form units
with -fmad=false, matching the reference build, GPU/makefile:10, so that no
multiply-add is contracted) and linked into one shared library exporting the
C ABI of include/tsuner_b200.h.  Objects go to tsuner_b200/_build/.
"""
import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libtsuner_b200.so")
EXE = os.path.join(PKG, "tsuner.exe")
INC = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# per-unit extra flags
UNIT_FLAGS = {
    "stage64.cu": ["-fmad=false"],
    "solver.cu": ["-fmad=false"],
    "noalloc.cu": ["-fmad=false"],
    # FP32 precision form: single precision may contract and use the hardware
    # approximations; its FP64 islands are unaffected by this flag.
    "stage32.cu": ["-use_fast_math"],
    # host restatement of the reference's input interpolation: no contraction,
    # like the reference's host build
    "nctr.cpp": ["-Xcompiler", "-ffp-contract=off"],
}
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INC, "-I" + CSRC]


def _headers():
    hs = [os.path.join(INC, f) for f in os.listdir(INC)]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build failed: " + os.path.basename(cmd[-3] if len(cmd) > 3 else cmd[0]))
    return r


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))
    hdrs = _headers() + [os.path.abspath(__file__)]
    objs = []
    for f in srcs:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            cmd = [NVCC] + ARCH + COMMON + UNIT_FLAGS.get(f, []) + ["-c", src, "-o", obj]
            if f.endswith(".cpp"):
                cmd = [NVCC] + COMMON + UNIT_FLAGS.get(f, []) + ["-x", "c++", "-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            r = _run(cmd)
            if verbose:
                sys.stdout.write(r.stderr)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    # tsuner.exe front end, linked against the library (rpath = its folder)
    app = os.path.join(PKG, "app", "tsuner_main.cpp")
    if force or _stale(EXE, [app, LIB] + hdrs):
        _run(["g++", "-O2", "-std=c++17", "-I" + INC, "-I/usr/local/cuda/include", app, "-o", EXE,
              "-L" + PKG, "-ltsuner_b200", "-Wl,-rpath,$ORIGIN", "-L/usr/local/cuda/lib64", "-lcudart"])
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose))


if __name__ == "__main__":
    main()
