"""Golden fixtures of the euclidean-clustering parity tests, from the
reference itself.  Run here, where the reference tree exists and oracle/_ref
is built (make -C oracle ref):

    python tests/golden/make_ec_fixtures.py

Reads the reference's own data files data/ec_input.dat.gz and
data/ec_output.dat.gz, checks that the UNMODIFIED reference kernel
(oracle/_ref/libref_ec.so) reproduces the shipped output under its own
acceptance rule (the oracle pin), and writes ec_cases.npz: per test case the
input cloud, the reference's clusters of each distance ring (extract()'s
output: sizes and point indices into the ring's cloud, in its order), and the
reference's segmentByDistance boxes and centroids, and per kept box the yaw
quaternion (z, w) of the reference's pose estimate computed with the hull's
own length (oracle/ec_shim.cpp ref_ec_box_yaw: the reference's
minAreaRectAngle reads past the end of the hull, so its own yaw is not
reproducible).
"""
from __future__ import annotations

import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1] / "oracle"))

import binding  # noqa: E402
import ec_ref  # noqa: E402

REF_DATA = binding.reference_dir() / "data"
RING_TOL = (0.5, 1.1, 1.6, 2.3, np.float32(2.6).item())


def rings(xyz):
    """The cloud split of segmentByDistance (kernel.cpp:781-805), by float distance from the origin."""
    x, y = xyz[:, 0], xyz[:, 1]
    d = np.sqrt(x * x + y * y)  # float32 products, sum and square root
    r = np.where(d < 15, 0, np.where(d < 30, 1, np.where(d < 45, 2, np.where(d < 60, 3, 4))))
    return [xyz[r == k] for k in range(5)]


def kept(pts):
    """clusterAndColor's box filter (kernel.cpp:747-749) on a cluster's float extents."""
    lo, hi = pts.min(0), pts.max(0)
    d = hi - lo
    return bool(d[0] > 0 and d[1] > 0 and d[2] > 0 and d[0] < 15 and d[1] < 15 and hi[2] > -1.5 and lo[2] > -1.5
                and lo[2] < 1.0)


def main():
    ins = ec_ref.read_input(REF_DATA / "ec_input.dat.gz")
    outs = ec_ref.read_output(REF_DATA / "ec_output.dat.gz", len(ins))
    ref = ec_ref.Reference()
    arrays = {"cases": np.array(len(ins))}
    for i, (xyz, out) in enumerate(zip(ins, outs)):
        pts, b10, cen = ref.segment(xyz)
        ok, d = ec_ref.check(pts, ec_ref.boxes10_to_8(b10), cen, out[0], out[2], out[3])
        assert ok, f"case {i}: the reference does not reproduce its shipped output (max delta {d})"
        arrays[f"in{i}"] = xyz
        arrays[f"boxes{i}"] = b10
        arrays[f"centroids{i}"] = cen
        arrays[f"npts{i}"] = np.array(len(pts))
        yaw = []
        for k, cloud in enumerate(rings(xyz)):
            cl = ref.extract(cloud, RING_TOL[k])
            arrays[f"sizes{i}_{k}"] = np.array([len(c) for c in cl], np.int32)
            arrays[f"idx{i}_{k}"] = (np.concatenate(cl) if cl else np.zeros(0)).astype(np.uint16)
            for c in cl:
                if kept(cloud[c]):
                    yaw.append(ref.box_yaw(cloud[c])[1:])
        assert len(yaw) == len(b10)
        arrays[f"yaw{i}"] = np.array(yaw, np.float64).reshape(-1, 2)
    np.savez_compressed(HERE / "ec_cases.npz", **arrays)
    print("wrote", HERE / "ec_cases.npz")


if __name__ == "__main__":
    main()
