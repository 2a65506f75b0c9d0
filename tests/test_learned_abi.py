"""The learned-init pipeline driven from C++ through the C ABI
(tests/native/learned_abi.cpp: host buffers only, linked against
libndt_b200.so): it builds here without a GPU; on a GPU its results equal
the Python-side LearnedBatch (ndt_align_batch_learned_device) bit for bit."""
import pathlib
import shutil
import struct
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "learned_abi.cpp"
LIBDIR = ROOT / "daphne-benchmark_b200" / "_build"


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    gxx = shutil.which("g++")
    if not gxx or not (LIBDIR / "libndt_b200.so").exists():
        pytest.skip("needs g++ and the built library")
    out = tmp_path_factory.mktemp("abi") / "learned_abi"
    subprocess.run([gxx, "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(SRC), "-o", str(out), f"-L{LIBDIR}",
                    "-lndt_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return out


def test_builds_against_the_header(exe):
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_cpp_learned_batch_equals_python(pkg, exe, tmp_path):
    torch = pytest.importorskip("torch")
    L, PN, ndt, synth = pkg.learned, pkg.posenet, pkg.ndt, pkg.synth
    cfg = synth.small_config("abi_l", 30000, 50.0, 20, 3000, seed=71, dt=1.0, dyaw_deg=5.0)
    scene = synth.make_scene(cfg)
    aligns = [synth.make_alignment(cfg, scene, i) for i in range(48)]
    spec = L.refinement_levels(cfg.resolution)
    levels = L.level_contexts(ndt, scene.map, cfg.resolution, levels=spec)
    net = PN.PoseNet(center=(0.0, 0.0, 0.0), scale=4.0)
    w = PN.init_weights(5)
    net.set_weights(w)
    dev = L.DeviceScans(torch, [a.scan for a in aligns])
    pts, offs, total = dev.batch(np.arange(len(aligns)))
    guesses = np.stack([a.guess for a in aligns]).astype(np.float32)
    lb = L.LearnedBatch(levels, net, torch, pts, offs, total, guesses, PN.learned_params())  # the C defaults
    lb.run()
    out, conv, fit, st, choice, start = lb.results()
    B = len(aligns)
    offsets = np.zeros(B + 1, np.int32)
    offsets[1:] = np.cumsum([len(a.scan) for a in aligns])
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(struct.pack("<i", len(scene.map)) + np.ascontiguousarray(scene.map, np.float32).tobytes())
        lv = [[lvl["resolution"], lvl["step_size"], lvl["max_iterations"], lvl["transformation_epsilon"]] for lvl in spec]
        f.write(struct.pack("<i", len(spec)) + np.asarray(lv, np.float64).tobytes())
        f.write(struct.pack("<i", len(w)) + w.tobytes())
        f.write(np.zeros(3, np.float32).tobytes() + struct.pack("<f", 4.0) + PN.DELTA_SCALE.tobytes())
        f.write(struct.pack("<i", B) + offsets.tobytes())
        f.write(np.concatenate([a.scan for a in aligns]).astype(np.float32).tobytes() + guesses.tobytes())
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = (tmp_path / "out.bin").read_bytes()
    o = np.frombuffer(raw, np.float32, 16 * B).reshape(B, 16)
    pos = 64 * B
    c = np.frombuffer(raw, np.int32, B, pos)
    pos += 4 * B
    fi = np.frombuffer(raw, np.float64, B, pos)
    pos += 8 * B
    s = np.frombuffer(raw, np.int32, B, pos)
    pos += 4 * B
    ch = np.frombuffer(raw, np.int32, B, pos)
    pos += 4 * B
    stt = np.frombuffer(raw, np.float32, 16 * B, pos).reshape(B, 16)
    assert np.array_equal(o.view(np.uint32), out.view(np.uint32))
    assert np.array_equal(c, conv) and np.array_equal(fi.view(np.uint64), fit.view(np.uint64))
    assert np.array_equal(s, st) and np.array_equal(ch, choice)
    assert np.array_equal(stt.view(np.uint32), start.view(np.uint32))
    net.close()
    for ctx in levels:
        ctx.close()
