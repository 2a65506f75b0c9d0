"""The drop-in as a DAPHNE tree would link it: the reference harness's own
main (src/CPU/common/main.cpp, compiled from the reference's source with its
own flags) linked with the front ends' kernel.cpp (oracle/Makefile target
`harness`, the recipe of the integration notes).  main.cpp calls init / run /
check_output through the vtable of the front end's `myKernel`
(src/CPU/common/main.cpp:72-80), so these tests fail if the front end's
`kernel` class is not layout-identical to src/CPU/include/benchmark.h:11-55.

The executables are built by build() where the reference tree is present and
travel with the other built files; the tests skip when they are absent."""
import os
import pathlib
import subprocess

import pytest

from test_harness import _dataset
from test_harness_ec import _write

ROOT = pathlib.Path(__file__).resolve().parents[1]
HARNESS = ROOT / "oracle" / "_ref" / "harness"
NDT_EXE = HARNESS / "ndt_kernel"
EC_EXE = HARNESS / "ec_kernel"


def _need(exe):
    if not exe.exists():
        pytest.skip("reference harness link not built (needs the reference tree at build time)")
    return exe


@pytest.mark.parametrize("exe,env_in,message", [
    (NDT_EXE, "NDT_INPUT", "Error opening the testcase file"),
    (EC_EXE, "EC_INPUT", "Error opening the input data file"),
])
def test_reference_main_reaches_init(tmp_path, exe, env_in, message):
    """The reference main calls the front end's init() (which prints "init")
    and the front end stops at the missing data file with the reference's
    exit(-3)."""
    exe = _need(exe)
    env = dict(os.environ, **{env_in: str(tmp_path / "none.dat")})
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, cwd=tmp_path, timeout=60)
    assert r.stdout.startswith("init\n"), r.stdout + r.stderr
    assert message in r.stderr
    assert r.returncode == 253  # exit(-3)


@pytest.mark.parametrize("exe", [NDT_EXE, EC_EXE])
@pytest.mark.parametrize("args,code", [(["-p"], 2), (["-x", "3"], 3), (["-p", "0"], 4)])
def test_reference_main_usage(exe, args, code):
    exe = _need(exe)
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=60)
    assert r.returncode == code and "Usage" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("p", [1, 4])
def test_reference_main_runs_ndt_data(pkg, oracle, binding_mod, tmp_path, p):
    exe = _need(NDT_EXE)
    _dataset(pkg, oracle, binding_mod, tmp_path)
    env = dict(os.environ, NDT_INPUT=str(tmp_path / "ndt_input.dat"), NDT_OUTPUT=str(tmp_path / "ndt_output.dat"))
    r = subprocess.run([str(exe), "-p", str(p)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "result ok" in r.stdout and "average time per testcase (#7)" in r.stdout


@pytest.mark.gpu
def test_reference_main_runs_ec_data(tmp_path):
    exe = _need(EC_EXE)
    env = _write(tmp_path)
    r = subprocess.run([str(exe), "-p", "3"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "result ok" in r.stdout and "average time per testcase (#5)" in r.stdout
