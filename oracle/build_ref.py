"""Build recipe for the reference checker (oracle/_ref/).

TEST INFRASTRUCTURE ONLY.  Compiles the reference TSUNER CUDA sources,
unmodified, where they lie under the reference checkout, together with
oracle/ref_build/ref_harness.cu into one shared library per compile-time
switch variant:  oracle/_ref/<variant>/libtsuner_ref.so

The reference selects its scheme with #defines in Sim_parameters.hxx
(order, RK, WBC, BEDLOAD, SUSPENSION, Read_files; Sim_parameters.hxx:45-54).
A variant is built without copying or editing any reference file: a small
generated header is force-included (-include) that first includes the
reference Sim_parameters.hxx (which is `#pragma once`) and then re-#defines
the switches, so the later `#include "Sim_parameters.hxx"` of TSUNER.h is a
no-op and the kernels see the variant's values.

Flags follow GPU/makefile:10 (-O2 -fmad=false -rdc=true -dlto) with
-arch=native replaced by sm_100a (this container has no GPU to query).
Every variant is also built as "<variant>-nolto": the same sources and flags
without -dlto.  Link-time optimisation generates the device code at the
device-link step, and there the reference build's arithmetic differs from a
strict -fmad=false compile in the last bits (measured: 1e-16..3e-15 relative
after 2000 steps); the -nolto build is the bit-for-bit pin of the oracle and
of the product, the recipe build is the reference as its makefile makes it.

Usage:  python oracle/build_ref.py [--ref PATH] [variant ...]
The built .so files travel to the GPU box; the reference tree is only read
here, at build time.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference checkout: TSUNER_REF_DIR, else where this container mounts it
DEFAULT_REF = os.environ.get("TSUNER_REF_DIR", "/root/reference")

# name -> switch overrides (unset keys keep the reference defaults:
# order 2, RK 1, WBC 1, BEDLOAD 1, SUSPENSION 1, Read_files 1)
VARIANTS = {
    "default": {},
    "rf0_wbc1": {"Read_files": 0, "WBC": 1},
    "rf0_wbc0": {"Read_files": 0, "WBC": 0},
    "rf0_wbc2": {"Read_files": 0, "WBC": 2},
    "order1": {"order": 1},
    "nosed": {"BEDLOAD": 0, "SUSPENSION": 0},
    # MUSCL-Hancock (GPU/Reconstructor.cu:280-342, one stage per step)
    "rk0": {"RK": 0},
    "rk0_order1": {"RK": 0, "order": 1},
    # the unfinished Manning friction branch (GPU/Reconstructor.cu:47-50)
    "manning_rf0": {"Manning": 1, "Read_files": 0},
}

KERNEL_SOURCES = [
    "GPU/Reconstructor.cu",
    "GPU/VolumeSolver.cu",
    "GPU/Volume_kernel.cu",
    "GPU/Reduction_kernel_min.cu",
]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O2", "-arch=sm_100a", "-fmad=false", "-rdc=true", "-dlto",
         "-Xcompiler", "-fPIC", "-w"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("reference build step failed")


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build_variant(name, ref=DEFAULT_REF, force=False):
    lto = not name.endswith("-nolto")
    sw = VARIANTS[name[:-6] if not lto else name]
    flags = FLAGS if lto else [f for f in FLAGS if f != "-dlto"]
    vdir = os.path.join(OUT, name)
    os.makedirs(vdir, exist_ok=True)
    so = os.path.join(vdir, "libtsuner_ref.so")
    srcs = [os.path.join(ref, s) for s in KERNEL_SOURCES]
    deps = srcs + [os.path.join(HERE, "ref_build", "ref_harness.cu"), __file__,
                   os.path.join(ref, "Sim_parameters.hxx"), os.path.join(ref, "GPU", "SedFlux.cuh")]
    if not force and _newer(so, deps):
        return so
    ov = os.path.join(vdir, "switches.h")
    with open(ov, "w") as f:
        f.write("/* generated by oracle/build_ref.py: variant %s */\n" % name)
        f.write('#include "%s"\n' % os.path.join(ref, "Sim_parameters.hxx"))
        for k, v in sw.items():
            f.write("#undef %s\n#define %s %d\n" % (k, k, v))
    inc = ["-include", ov, "-I" + os.path.join(ref, "GPU"), "-I" + ref,
           "-I" + os.path.join(HERE, "ref_build")]
    objs = []
    for s in srcs + [os.path.join(HERE, "ref_build", "ref_harness.cu")]:
        o = os.path.join(vdir, os.path.basename(s).replace(".cu", ".o"))
        _run([NVCC] + flags + inc + ["-c", s, "-o", o])
        objs.append(o)
    dl = os.path.join(vdir, "dlink.o")
    # GPU/makefile:27-28 passes the full NVCCFLAGS (incl. -fmad=false) to the
    # device link; with -dlto that is where device code is generated.
    _run([NVCC] + flags + ["-dlink"] + objs + ["-o", dl])
    _run(["g++", "-shared", "-o", so] + objs + [dl, "-L/usr/local/cuda/lib64", "-lcudart"])
    for o in objs + [dl]:
        os.remove(o)
    return so


def build_interp(ref=DEFAULT_REF, force=False):
    """oracle/_ref/interp/libref_interp.so: the reference's host input
    interpolation (interpolations.cxx, tides.cxx, unmodified, g++ -O2 as the
    reference makefile builds its host code) with ref_build/ref_interp_shim.cpp
    and the in-memory netCDF stand-in ref_build/fake_netcdf.c."""
    vdir = os.path.join(OUT, "interp")
    os.makedirs(vdir, exist_ok=True)
    so = os.path.join(vdir, "libref_interp.so")
    rb = os.path.join(HERE, "ref_build")
    srcs = [os.path.join(ref, "interpolations.cxx"), os.path.join(ref, "tides.cxx"),
            os.path.join(rb, "ref_interp_shim.cpp")]
    fake = os.path.join(rb, "fake_netcdf.c")
    deps = srcs + [fake, os.path.join(rb, "netcdf.h"), __file__, os.path.join(ref, "TSUNER.h"),
                   os.path.join(ref, "Sim_parameters.hxx")]
    if not force and _newer(so, deps):
        return so
    inc = ["-I" + ref, "-I" + rb, "-I/usr/local/cuda/include"]
    objs = []
    for s in srcs:
        o = os.path.join(vdir, os.path.basename(s) + ".o")
        _run(["g++", "-O2", "-fPIC", "-w"] + inc + ["-c", s, "-o", o])
        objs.append(o)
    o = os.path.join(vdir, "fake_netcdf.o")
    _run(["gcc", "-O2", "-fPIC", "-I" + rb, "-c", fake, "-o", o])
    objs.append(o)
    _run(["g++", "-shared", "-o", so] + objs)
    for o in objs:
        os.remove(o)
    return so


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("variants", nargs="*", help="kernel variants (and/or 'interp'); default: all")
    a = ap.parse_args(argv)
    if not os.path.isdir(a.ref):
        print("reference tree not present; keeping prebuilt oracle/_ref")
        return 0
    names = a.variants or [v + sfx for v in VARIANTS for sfx in ("", "-nolto")] + ["interp"]
    for v in names:
        print(build_interp(a.ref, a.force) if v == "interp" else build_variant(v, a.ref, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
