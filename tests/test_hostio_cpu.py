"""CPU: the host worker pool behind the library's bulk host <-> device
copies (tsu::host_parallel in hostio.cpp).  A C++ driver linked against the
built libtsuner_b200.so checks that every index runs exactly once per call
over thousands of calls, from four caller threads at once, and in a forked
child.  No GPU is touched."""
import os
import subprocess

import pytest

import tsuner_b200 as T

HERE = os.path.dirname(os.path.abspath(__file__))
CUDA_LIB = "/usr/local/cuda/lib64"


def test_host_pool(tmp_path):
    lib_dir = os.path.dirname(T.LIB_PATH)
    if not os.path.exists(T.LIB_PATH):
        pytest.fail("libtsuner_b200.so is not built")
    exe = str(tmp_path / "pool_check")
    subprocess.run(["g++", "-O2", "-std=c++17", os.path.join(HERE, "hostio_pool_check.cpp"), "-o", exe,
                    "-L" + lib_dir, "-ltsuner_b200", "-Wl,-rpath," + lib_dir, "-Wl,-rpath," + CUDA_LIB,
                    "-L" + CUDA_LIB, "-lcudart", "-pthread"], check=True)
    env = dict(os.environ, TSU_HOST_THREADS="6")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=180, env=env)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "threads 6" in r.stdout and "ok" in r.stdout


def test_host_threads_symbol():
    n = T.lib().tsu_host_threads()
    assert 1 <= n <= 256
