"""The tensor-core descriptor encoders of csrc/umma_desc.h, checked bit for
bit against CUTLASS's CuTe descriptor types (CuTe's make_instr_desc and its
SmemDescriptor bitfields, filled as its make_umma_desc fills them for a
no-swizzle K-major operand).  Host code only: compiled with nvcc, no GPU."""
import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _cute_include():
    """CUTLASS/CuTe headers vendored in the flashinfer package, located without importing it."""
    import importlib.util

    spec = importlib.util.find_spec("flashinfer")
    if spec is None or not spec.submodule_search_locations:
        return None
    p = pathlib.Path(list(spec.submodule_search_locations)[0]) / "data" / "cutlass" / "include"
    return p if (p / "cute" / "arch" / "mma_sm100_desc.hpp").exists() else None


def test_descriptors_match_cute(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    inc = _cute_include()
    if inc is None or not pathlib.Path(nvcc).exists():
        pytest.skip("CUTLASS headers or nvcc not available")
    exe = tmp_path / "umma_desc_check"
    subprocess.run([nvcc, "-std=c++17", "-O1", "-I", str(inc), "-I", str(ROOT / "daphne-benchmark_b200" / "csrc"),
                    str(ROOT / "tests" / "native" / "umma_desc_check.cu"), "-o", str(exe)], check=True,
                   capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert r.stdout.strip().endswith("OK")
