"""The C ABI from a compiled C program (tests/c_abi/cholqr2_from_c.c), the
way a `ccall` binding reaches it: plain pointers, sizes and statuses, no
Python in between. Without a GPU the program checks the statuses of bad
arguments; on a B200 it also orthonormalizes a matrix through fb_zcholqr2
and fb_zcholqr2_staged and checks both against each other and the accuracy
targets."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "c_abi", "cholqr2_from_c.c")
LIBDIR = os.path.join(ROOT, "funicular.jl_b200")


def build(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = str(tmp_path / "cholqr2_from_c")
    subprocess.run([cc, "-O2", "-std=c11", "-Wall", "-I", os.path.join(ROOT, "include"), SRC, "-L", LIBDIR,
                    "-lfunicular_b200", f"-Wl,-rpath,{LIBDIR}", "-lm", "-o", exe], check=True)
    return exe


def test_c_program_gets_the_statuses_without_a_device(fb, tmp_path):
    if fb._lib.device_count() > 0:
        pytest.skip("covered by the device run")
    r = subprocess.run([build(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "statuses ok" in r.stdout


@pytest.mark.gpu
def test_c_program_orthonormalizes_through_the_abi(backend, tmp_path):
    r = subprocess.run([build(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("info 0 passes 2")
