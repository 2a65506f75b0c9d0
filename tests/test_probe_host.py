"""The exact parts of the derivative pass's neighbour search
(daphne-benchmark_b200/csrc/probe.cuh) compiled as host code and checked
against the reference's probe loop and distance test on the CPU
(tests/native/probe_check.cpp): 800k probe axes (box edges, cell
boundaries, four resolutions incl. a non-power of two) and 4M point/mean
pairs within a few ulps of the radius, at coordinates up to 1e5 m."""
import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
CUDA_INC = pathlib.Path("/usr/local/cuda/include")


@pytest.mark.skipif(not (shutil.which("g++") and CUDA_INC.is_dir()), reason="needs g++ and the CUDA headers")
def test_probe_exact_parts_on_host(tmp_path):
    exe = tmp_path / "probe_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{CUDA_INC}",
                    f"-I{ROOT / 'daphne-benchmark_b200' / 'csrc'}", str(ROOT / "tests" / "native" / "probe_check.cpp"),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "axes 800000 bad 0" in r.stdout and "window disagreements 0" in r.stdout and "bad 0\n" in r.stdout
