"""Generate the golden fixtures of tests/golden/ from the compiled reference.

Run here, where the reference sources exist (oracle/_ref built by
`make -C oracle ref`):

    python tests/golden/make_fixtures.py

Writes
  * reference_cases.json -- seeded synthetic cases (inputs are regenerated from
    the seed by daphne-benchmark_b200/synth.py, whose output is checked by the
    stored sha256) with the UNMODIFIED reference kernel's results:
    partial_points_callback output (16 floats as uint32 bit patterns, converged),
    the grid bbox/dims/occupied-cell checksum, and one computeDerivatives
    evaluation (score, gradient, Hessian) at the guess.
  * reference_ndt_output.json -- the 5 records of the reference's own golden file
    data/ndt_output.dat.gz (its matching input file is not distributed).
"""
from __future__ import annotations

import hashlib
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "daphne-benchmark_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import binding  # noqa: E402
import datfile  # noqa: E402
import synth  # noqa: E402

REF_DIR = binding.reference_dir()


def cases():
    """(name, config, alignment index, scan-override) tuples; small enough for CPU tests."""
    small = synth.small_config("s8k", 8000, 30.0, 10, 500, seed=11)
    mid = synth.small_config("s20k", 20000, 40.0, 16, 1000, seed=12)
    half = synth.small_config("s20k_r05", 20000, 30.0, 12, 800, seed=13, resolution=0.5)
    far = synth.small_config("s8k_far", 8000, 30.0, 10, 400, seed=14, dt=3.0, dyaw_deg=15.0)
    c1 = synth.CONFIGS["c1"]
    out = []
    for i in range(3):
        out.append((f"small_{i}", small, i))
    for i in range(2):
        out.append((f"mid_{i}", mid, i))
    out.append(("res05_0", half, 0))
    out.append(("far_0", far, 0))
    out.append(("far_1", far, 1))
    for i in range(2):
        out.append((f"c1_{i}", c1, i))
    return out


def scene_cache():
    cache = {}

    def get(cfg):
        key = (cfg.seed, cfg.map_points, cfg.area, cfg.walls)
        if key not in cache:
            cache[key] = synth.make_scene(cfg)
        return cache[key]

    return get


def grid_summary(ref, cloud):
    bbox, dims, cells = ref.grid(cloud)
    occ = np.nonzero(cells[:, 12] > 0)[0]
    h = hashlib.sha256(np.ascontiguousarray(cells[occ]).tobytes()).hexdigest()
    return {
        "bbox_bits": bbox.view(np.uint32).tolist(),
        "dims": dims.tolist(),
        "occupied": int(occ.size),
        "occupied_sha256": h,
    }


def main():
    if not binding.Reference.available("serial"):
        binding.build(quiet=False)
    ref = binding.Reference("serial")
    orc = binding.Oracle()
    get_scene = scene_cache()
    records = []
    for name, cfg, idx in cases():
        scene = get_scene(cfg)
        a = synth.make_alignment(cfg, scene, idx)
        prm = binding.reference_params(cfg.resolution)
        if cfg.resolution != 1.0:
            # the reference hard-codes resolution 1.0 (kernel.cpp:38); other
            # resolutions are pinned through the oracle only
            out, conv, _, _ = orc.align(prm, a.scan, a.guess, scene.map)
            source = "oracle"
            deriv = None
            grid = None
        else:
            out, conv = ref.align(a.scan, a.guess, scene.map)
            source = "reference"
            d1, d2 = orc.gauss(prm)
            trans = ref.transform(a.scan, a.guess)
            p6 = np.zeros(6)
            p6[:3] = a.guess.reshape(4, 4)[:3, 3]
            p6[3:] = ref.euler(a.guess)
            s, g, H = ref.derivatives(scene.map, a.scan, trans, p6, d1, d2)
            deriv = {"p6": p6.tolist(), "score": s, "gradient": g.tolist(), "hessian": H.reshape(36).tolist()}
            grid = grid_summary(ref, scene.map)
        records.append({
            "name": name,
            "source": source,
            "config": {k: getattr(cfg, k) for k in ("name", "map_points", "area", "walls", "resolution",
                                                     "scan_min", "dt", "dyaw_deg", "radius", "seed")},
            "index": idx,
            "input_sha256": synth.digest(a.scan, a.guess, scene.map),
            "out_bits": out.view(np.uint32).tolist(),
            "out": [float(v) for v in out],
            "converged": int(conv),
            "derivatives": deriv,
            "grid": grid,
        })
        print(name, source, conv, out.reshape(4, 4)[0])
    (HERE / "reference_cases.json").write_text(json.dumps({"cases": records}, indent=1))

    gold = REF_DIR / "data" / "ndt_output.dat.gz"
    if gold.exists():
        recs = datfile.read_output(gold)
        (HERE / "reference_ndt_output.json").write_text(json.dumps({
            "source": "data/ndt_output.dat.gz of the reference (5 records, 73 bytes each)",
            "records": [{"T_bits": r["T"].view(np.uint32).tolist(), "T": [float(v) for v in r["T"]],
                         "fitness_bits": int(np.array(r["fitness"]).view(np.uint64)),
                         "converged": int(r["converged"])} for r in recs],
        }, indent=1))


if __name__ == "__main__":
    main()
