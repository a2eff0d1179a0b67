"""The C ABI driven from C, the way the Fortran host binds it."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_driver", "abi_driver.c")
LIBDIR = os.path.join(ROOT, "simp_b200")


def _compile(out, link=True):
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    cmd = [cc, "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o", out]
    if link:
        cmd += ["-L", LIBDIR, "-lsimp_gpu", f"-Wl,-rpath,{LIBDIR}", "-lm"]
    else:
        cmd = cmd[:-2] + ["-c", "-o", out]
    subprocess.run(cmd, check=True)


def test_header_compiles_as_c99(tmp_path):
    _compile(str(tmp_path / "abi_driver.o"), link=False)


@pytest.mark.gpu
def test_c_driver_runs(gpu_lib, tmp_path):
    exe = str(tmp_path / "abi_driver")
    _compile(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "abi_driver ok" in r.stdout
