"""The DAPHNE euclidean_cluster front end (daphne-benchmark_b200/daphne_ec/
kernel): the reference's CLI, data files (ec_input.dat, ec_output.dat) and
acceptance rule, clustering on the GPU library.  The data files are written
from the reference's own results (tests/golden/ec_cases.npz)."""
import os
import pathlib
import struct
import subprocess

import numpy as np
import pytest

import ec_ref

ROOT = pathlib.Path(__file__).resolve().parents[1]
HARNESS = ROOT / "daphne-benchmark_b200" / "daphne_ec"
GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "ec_cases.npz"


def _rings(xyz):
    x, y = xyz[:, 0], xyz[:, 1]
    d = np.sqrt(x * x + y * y)
    r = np.where(d < 15, 0, np.where(d < 30, 1, np.where(d < 45, 2, np.where(d < 60, 3, 4))))
    return [xyz[r == k] for k in range(5)]


@pytest.fixture(scope="module")
def ec_exe():
    subprocess.run(["make", "-C", str(HARNESS)], check=True, stdout=subprocess.DEVNULL)
    return HARNESS / "kernel"


def _write(tmp_path, reorder=False, bad_centroid=None):
    """ec_input.dat (int32 T; per case int32 n + n x float32[3]) and ec_output.dat (per case the
    coloured cloud, the 8-column boxes and the centroids), as the reference's files are laid out."""
    gold = np.load(GOLDEN)
    T = int(gold["cases"])
    rng = np.random.default_rng(3)
    with open(tmp_path / "ec_input.dat", "wb") as fi, open(tmp_path / "ec_output.dat", "wb") as fo:
        fi.write(struct.pack("<i", T))
        for i in range(T):
            xyz = np.ascontiguousarray(gold[f"in{i}"], np.float32)
            fi.write(struct.pack("<i", len(xyz)) + xyz.tobytes())
            pts = np.concatenate([ring[gold[f"idx{i}_{k}"].astype(np.int64)] for k, ring in enumerate(_rings(xyz))])
            boxes = ec_ref.boxes10_to_8(gold[f"boxes{i}"]).copy()
            cen = gold[f"centroids{i}"].copy()
            if reorder:  # the rule sorts both sides: any order of the reference's entries is accepted
                pts, boxes, cen = pts[rng.permutation(len(pts))], boxes[rng.permutation(len(boxes))], cen[::-1]
            if bad_centroid is not None and i == 2:
                cen[5, 1] += bad_centroid
            rec = np.zeros(len(pts), np.dtype([("xyz", "<f4", (3,)), ("rgb", "u1", (3,))]))
            rec["xyz"], rec["rgb"] = pts, (10, 20, 30)
            fo.write(struct.pack("<i", len(pts)) + rec.tobytes())
            fo.write(struct.pack("<i", len(boxes)) + np.ascontiguousarray(boxes, "<f8").tobytes())
            fo.write(struct.pack("<i", len(cen)) + np.ascontiguousarray(cen, "<f8").tobytes())
    return dict(os.environ, EC_INPUT=str(tmp_path / "ec_input.dat"), EC_OUTPUT=str(tmp_path / "ec_output.dat"))


@pytest.mark.parametrize("args,code", [(["-p"], 2), (["-x", "3"], 3), (["-p", "0"], 4)])
def test_usage_exit_codes(ec_exe, args, code):
    r = subprocess.run([str(ec_exe), *args], capture_output=True, text=True)
    assert r.returncode == code and "Usage" in r.stdout


def test_missing_data_file(ec_exe, tmp_path):
    env = dict(os.environ, EC_INPUT=str(tmp_path / "none.dat"), EC_OUTPUT=str(tmp_path / "none2.dat"))
    r = subprocess.run([str(ec_exe)], capture_output=True, text=True, env=env)
    assert r.returncode != 0 and "Error opening the input data file" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("p,reorder", [(1, False), (3, True), (8, False)])
def test_harness_runs_reference_data(ec_exe, tmp_path, p, reorder):
    env = _write(tmp_path, reorder=reorder)
    r = subprocess.run([str(ec_exe), "-p", str(p)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "result ok" in r.stdout and "max delta: 0\n" in r.stdout
    assert "average time per testcase (#5)" in r.stdout


@pytest.mark.gpu
def test_harness_detects_wrong_reference(ec_exe, tmp_path):
    env = _write(tmp_path, bad_centroid=0.01)  # beyond the rule's 0.001
    r = subprocess.run([str(ec_exe), "-p", "2"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 1 and "error: wrong result" in r.stdout
