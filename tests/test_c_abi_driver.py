"""The C ABI from a C host: tests/c_abi/driver.c (plain C99, no Python types) is built
with gcc against include/raven_b200.h and libravenb200.so.  On the CPU the program must
compile and link; on a B200 it runs its checks (free stream, conservation of 10
LSRK(5,4) steps through the host-buffer entry point, bit-equality with the device entry
point, status codes) and exits 0."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "raven.jl_b200")
CUDA = "/usr/local/cuda"


def _build(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not found")
    if not os.path.exists(os.path.join(LIBDIR, "libravenb200.so")):
        pytest.skip("libravenb200.so is not built")
    exe = str(tmp_path / "rb200_c_driver")
    cmd = ["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-D_DEFAULT_SOURCE",
           os.path.join(ROOT, "tests", "c_abi", "driver.c"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), "-L", LIBDIR, "-lravenb200", "-Wl,-rpath," + LIBDIR,
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-lm",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_driver_compiles_and_links(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_c_driver_runs(tmp_path, cuda_ok):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failure(s)" in r.stdout
