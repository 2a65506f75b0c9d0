"""The DAPHNE harness front end (daphne-benchmark_b200/daphne/kernel): the
reference's CLI, data files and acceptance rule, on the GPU library."""
import os
import pathlib
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
HARNESS = ROOT / "daphne-benchmark_b200" / "daphne"


@pytest.fixture(scope="module")
def kernel_exe():
    subprocess.run(["make", "-C", str(HARNESS)], check=True, stdout=subprocess.DEVNULL)
    return HARNESS / "kernel"


@pytest.mark.parametrize("args,code", [(["-p"], 2), (["-x", "3"], 3), (["-p", "0"], 4), (["-p", "abc"], 4)])
def test_usage_exit_codes(kernel_exe, args, code):
    r = subprocess.run([str(kernel_exe), *args], capture_output=True, text=True)
    assert r.returncode == code and "Usage" in r.stdout


def test_missing_data_file(kernel_exe, tmp_path):
    env = dict(os.environ, NDT_INPUT=str(tmp_path / "none.dat"), NDT_OUTPUT=str(tmp_path / "none2.dat"))
    r = subprocess.run([str(kernel_exe)], capture_output=True, text=True, env=env)
    assert r.returncode != 0 and "Error opening the testcase file" in r.stderr


def _dataset(pkg, oracle, binding_mod, tmp_path):
    cfg = pkg.synth.small_config("h", 8000, 30.0, 10, 500, seed=11)
    scene = pkg.synth.make_scene(cfg)
    cfg2 = pkg.synth.small_config("h2", 6000, 25.0, 8, 400, seed=12)
    scene2 = pkg.synth.make_scene(cfg2)
    cases = []
    for i in range(5):  # shared map: one grid build for these
        a = pkg.synth.make_alignment(cfg, scene, i)
        cases.append((a.guess, a.scan, scene.map))
    for i in range(2):  # a second map
        a = pkg.synth.make_alignment(cfg2, scene2, i)
        cases.append((a.guess, a.scan, scene2.map))
    prm = binding_mod.reference_params()
    outs, convs = [], []
    for g, s, m in cases:
        o, c, _, _ = oracle.align(prm, s, g, m)
        outs.append(o)
        convs.append(c)
    pkg.datfile.write_input(tmp_path / "ndt_input.dat", cases)
    pkg.datfile.write_output(tmp_path / "ndt_output.dat", outs, convs)
    return np.array(outs), np.array(convs)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [1, 3, 7])
def test_harness_runs_reference_data(pkg, oracle, binding_mod, kernel_exe, tmp_path, p):
    outs, convs = _dataset(pkg, oracle, binding_mod, tmp_path)
    env = dict(os.environ, NDT_INPUT=str(tmp_path / "ndt_input.dat"), NDT_OUTPUT=str(tmp_path / "ndt_output.dat"),
               NDT_DATAGEN_OUT=str(tmp_path / "dategen.dat"))
    r = subprocess.run([str(kernel_exe), "-p", str(p)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "result ok" in r.stdout and "average time per testcase (#7)" in r.stdout
    got = pkg.datfile.read_output(tmp_path / "dategen.dat")
    assert got["converged"].tolist() == convs.tolist()
    T = got["T"].reshape(-1, 4, 4)
    R = outs.reshape(-1, 4, 4)
    assert np.array_equal(T[:, :, 3].view(np.uint32), R[:, :, 3].view(np.uint32))
    assert np.max(np.abs(T[:, :3, :3] - R[:, :3, :3])) <= 2e-3


@pytest.mark.gpu
def test_harness_detects_wrong_reference(pkg, oracle, binding_mod, kernel_exe, tmp_path):
    outs, convs = _dataset(pkg, oracle, binding_mod, tmp_path)
    bad = outs.copy().reshape(-1, 4, 4)
    bad[3, 0, 3] += 0.5  # translation beyond MAX_TRANSLATION_EPS
    pkg.datfile.write_output(tmp_path / "ndt_output.dat", bad.reshape(-1, 16), convs)
    env = dict(os.environ, NDT_INPUT=str(tmp_path / "ndt_input.dat"), NDT_OUTPUT=str(tmp_path / "ndt_output.dat"))
    r = subprocess.run([str(kernel_exe)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 1 and "error: wrong result" in r.stdout
