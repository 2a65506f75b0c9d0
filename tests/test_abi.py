"""The C ABI library loads here (no GPU) and exports every entry point that
include/ndt_b200.h declares; calls that need a device fail loudly."""
import ctypes
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "ndt_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"NDT_API\s+[\w\s\*]*?\b(ndt_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for name in ("ndt_create", "ndt_set_map", "ndt_align", "ndt_align_with_map", "ndt_align_batch",
                 "ndt_align_batch_device", "ndt_align_batch_packed", "ndt_destroy"):
        assert name in syms


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.ndt.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_param_presets(pkg):
    r = pkg.ndt.reference_params()
    assert (r.resolution, r.outlier_ratio, r.step_size, r.transformation_epsilon, r.max_iterations, r.compat) == \
        (1.0, 0.55, 0.1, 0.1, 0, 1)
    c = pkg.ndt.corrected_params()
    assert (c.compat, c.transformation_epsilon, c.max_iterations, c.min_points_per_voxel, c.eigen_ratio) == \
        (0, 0.01, 30, 6, 0.01)
    assert ctypes.sizeof(pkg.ndt.Params) == 64


def test_kernel_variants_listed(pkg):
    v = pkg.ndt.kernel_variants()
    assert len(v) >= 2 and all(t in (128, 256) and b >= 1 for t, b in v)


def test_bad_arguments_rejected(pkg):
    L = pkg.ndt.lib()
    h = ctypes.c_void_p()
    p = pkg.ndt.reference_params()
    p.resolution = -1.0
    assert L.ndt_create(ctypes.byref(p), 0, ctypes.byref(h)) == -1  # NDT_E_ARG
    p = pkg.ndt.reference_params()
    p.precision = 7
    assert L.ndt_create(ctypes.byref(p), 0, ctypes.byref(h)) == -1
    # context setters reject a null context before touching a device
    assert L.ndt_set_chunk_tiles(None, 8) == -1
    assert L.ndt_get_chunk_tiles(None) == -1
    assert L.ndt_set_kernel_variant(None, 0) == -1


def test_no_cpu_fallback_without_device(pkg):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(pkg.ndt.NdtError):
        pkg.ndt.Context(pkg.ndt.reference_params())


def _c_layout(tmp_path, struct, fields):
    """sizeof and offsetof of each field of an include/ndt_b200.h struct, from the C compiler."""
    import shutil
    import subprocess

    if not shutil.which("gcc"):
        pytest.skip("needs gcc")
    src = tmp_path / f"{struct}.c"
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "ndt_b200.h"', "int main(void) {",
             f'  printf("%zu\\n", sizeof({struct}));']
    lines += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / struct
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    out = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    return out[0], out[1:]


@pytest.mark.parametrize("mirror", ["ndt.Params", "ndt.Counters", "binding.NdtParams"])
def test_struct_mirrors_match_the_header(pkg, binding_mod, tmp_path, mirror):
    """Every ctypes mirror of a header struct has the C compiler's size and field offsets."""
    mod, name = mirror.split(".")
    cls = getattr(pkg.ndt if mod == "ndt" else binding_mod, name)
    struct = "ndt_counters" if name == "Counters" else "ndt_params"
    fields = [f[0] for f in cls._fields_]
    size, offsets = _c_layout(tmp_path, struct, fields)
    assert ctypes.sizeof(cls) == size
    assert [getattr(cls, f).offset for f in fields] == offsets
