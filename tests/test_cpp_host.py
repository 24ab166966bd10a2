"""The header-only C++14 mirror of bld::bld_mult_cuda: it must compile with
-std=c++14 -Wall -pedantic here, and (GPU) pass the reference's own
test_bld_mult_cuda.cpp cases re-expressed in tests/cpp/."""

import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
SRC = os.path.join(ROOT, "tests", "cpp", "test_bld_mult_cuda.cpp")


def compile_test(out_path, bldm):
    lib_dir = os.path.dirname(bldm.LIB_PATH)
    cmd = [CXX, "-std=c++14", "-Wall", "-Wextra", "-pedantic", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "bnmf-algs_b200", "cpp"),
           SRC, "-L", lib_dir, "-lbldm", f"-Wl,-rpath,{lib_dir}", "-o", out_path]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_header_compiles(tmp_path, bldm):
    compile_test(str(tmp_path / "t"), bldm)


@pytest.mark.gpu
def test_cpp_reference_cases_on_gpu(tmp_path, bldm, kat, oracle):
    exe = str(tmp_path / "t")
    compile_test(exe, bldm)
    xp = tmp_path / "X.txt"
    np.savetxt(xp, kat["X"])
    outs = [str(tmp_path / "S_legacy.txt"), str(tmp_path / "S_appr.txt")]
    r = subprocess.run([exe, str(xp)] + outs, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    x, y = kat["X"].shape
    z = kat["z"]
    for path in outs:
        S = np.loadtxt(path).reshape(x, y, z)
        lm = oracle.log_marginal_S(S, np.ones(x), np.ones(z), kat["a"], kat["b"])
        assert lm >= kat["log_marginal_min"]
        assert oracle.sparseness(S) >= kat["sparseness_min"]
