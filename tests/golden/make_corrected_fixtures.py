"""Golden fixtures of the corrected NDT (the FP64 oracle's corrected mode).

    python tests/golden/make_corrected_fixtures.py

The corrected mode has no reference code to pin it to; it is checked by
finite differences (tests/test_oracle_fd.py) and by reaching the synthetic
ground truth.  This file freezes its results on the seeded cases of
make_fixtures.py so that any later change to it shows: per case the final
transform (uint32 bit patterns), converged, the fitness (uint64 bits), the
number of derivative evaluations, one evaluation at the guess (score,
gradient, Hessian bits) and the pose error against the ground truth.
Writes corrected_cases.json.
"""
from __future__ import annotations

import json
import math
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "daphne-benchmark_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(HERE))

import binding  # noqa: E402
import make_fixtures  # noqa: E402
import synth  # noqa: E402


def pose_error(T, truth):
    """Translation (m) and rotation (degrees) between a 4x4 result and the truth."""
    T = np.asarray(T, np.float64).reshape(4, 4)
    dt = float(np.linalg.norm(T[:3, 3] - truth[:3, 3]))
    R = T[:3, :3] @ truth[:3, :3].T
    c = max(-1.0, min(1.0, (np.trace(R) - 1.0) / 2.0))
    return dt, math.degrees(math.acos(c))


def main():
    orc = binding.Oracle()
    get_scene = make_fixtures.scene_cache()
    records = []
    for name, cfg, idx in make_fixtures.cases():
        scene = get_scene(cfg)
        a = synth.make_alignment(cfg, scene, idx)
        prm = binding.corrected_params(cfg.resolution)
        out, conv, fit, evals = orc.align(prm, a.scan, a.guess, scene.map)
        p6 = orc.pose_vector(0, a.guess)
        trans = orc.transform(a.scan, orc.build_tm(0, p6))
        s, g, H, pairs = orc.derivatives(prm, scene.map, a.scan, trans, p6)
        dt, dr = pose_error(out, a.truth)
        records.append({
            "name": name,
            "index": idx,
            "input_sha256": synth.digest(a.scan, a.guess, scene.map),
            "out_bits": out.view(np.uint32).tolist(),
            "converged": int(conv),
            "fitness_bits": int(np.array(fit).view(np.uint64)),
            "evaluations": int(evals),
            "guess_eval": {"p6_bits": p6.view(np.uint64).tolist(), "score_bits": int(np.array(s).view(np.uint64)),
                           "gradient_bits": g.view(np.uint64).tolist(),
                           "hessian_bits": H.reshape(36).view(np.uint64).tolist(), "pairs": int(pairs)},
            "truth_error": {"translation_m": dt, "rotation_deg": dr},
        })
        print(f"{name:10s} conv {conv} evals {evals:3d} error {dt:.4f} m {dr:.4f} deg")
    (HERE / "corrected_cases.json").write_text(json.dumps({"cases": records}, indent=1))


if __name__ == "__main__":
    main()
