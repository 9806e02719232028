"""The C++ Operator facade (cubismup_3d_b200/cpp/cubismup3d.hpp) compiled
against the C ABI: compile check on CPU, trajectory parity on the GPU."""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO, rel_l2

SRC = os.path.join(REPO, "tests", "cpp", "tg_driver.cpp")


def build_driver(out_dir):
    exe = os.path.join(out_dir, "tg_driver")
    lib_dir = os.path.join(REPO, "cubismup_3d_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(REPO, "include"), "-I", os.path.join(lib_dir, "cpp"),
           SRC, "-o", exe, "-L", lib_dir, "-lcup_b200", f"-Wl,-rpath,{lib_dir}"]
    subprocess.run(cmd, check=True)
    return exe


def test_facade_compiles_and_links(tmp_path):
    exe = build_driver(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [0, 1])
def test_facade_operator_pipeline_matches_oracle(tmp_path, oracle, scheme):
    exe = build_driver(str(tmp_path))
    n, nsteps = 32, 8
    out = os.path.join(str(tmp_path), "out.bin")
    subprocess.run([exe, str(n), str(nsteps), str(scheme), out], check=True, timeout=300)
    raw = np.fromfile(out, dtype=np.float64)
    fields = raw[:3 * n ** 3].reshape(3, n, n, n)
    dts = raw[3 * n ** 3:]
    from cubismup_3d_b200 import initial_conditions as ic
    orc = oracle.OracleSim(n, n, n, 2 * np.pi, nu=0.01, CFL=0.5, rampup=3, DLM=0.0, lambda_=1.0,
                           scheme=["ref", "upwind3_rk2"][scheme])
    orc.set_velocity(*ic.taylor_green((n, n, n), 2 * np.pi / n))
    odts = orc.run(nsteps)
    assert np.allclose(dts, odts, rtol=1e-12, atol=0)
    for a, b in zip(fields, orc.velocity()):
        assert rel_l2(a, b) < 1e-10
