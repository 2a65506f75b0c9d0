"""The corrected NDT (FP64 oracle, corrected mode) reproduces its frozen
results bit for bit (tests/golden/corrected_cases.json, made by
tests/golden/make_corrected_fixtures.py): final transform, converged,
fitness, evaluation count, and one evaluation at the guess.  Cases whose
guess is within the basin (not the far ones) end within 6 cm / 0.15 deg of
the synthetic ground truth."""
import json
import pathlib
import sys

import numpy as np
import pytest

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))

import make_fixtures  # noqa: E402
import make_corrected_fixtures as mcf  # noqa: E402

CASES = json.loads((GOLDEN / "corrected_cases.json").read_text())["cases"]
BY_NAME = {name: (cfg, idx) for name, cfg, idx in make_fixtures.cases()}
SCENES = make_fixtures.scene_cache()


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_corrected_oracle_frozen(pkg, oracle, binding_mod, case):
    cfg, idx = BY_NAME[case["name"]]
    scene = SCENES(cfg)
    a = pkg.synth.make_alignment(cfg, scene, idx)
    assert pkg.synth.digest(a.scan, a.guess, scene.map) == case["input_sha256"]
    prm = binding_mod.corrected_params(cfg.resolution)
    out, conv, fit, evals = oracle.align(prm, a.scan, a.guess, scene.map)
    assert out.view(np.uint32).tolist() == case["out_bits"]
    assert conv == case["converged"] and evals == case["evaluations"]
    assert int(np.array(fit).view(np.uint64)) == case["fitness_bits"]
    ge = case["guess_eval"]
    p6 = np.array(ge["p6_bits"], np.uint64).view(np.float64)
    trans = oracle.transform(a.scan, oracle.build_tm(0, p6))
    s, g, H, pairs = oracle.derivatives(prm, scene.map, a.scan, trans, p6)
    assert int(np.array(s).view(np.uint64)) == ge["score_bits"] and pairs == ge["pairs"]
    assert g.view(np.uint64).tolist() == ge["gradient_bits"]
    assert H.reshape(36).view(np.uint64).tolist() == ge["hessian_bits"]
    if not case["name"].startswith(("far", "res05", "mid_1")):
        dt, dr = mcf.pose_error(out, a.truth)
        assert dt < 0.06 and dr < 0.15, (dt, dr)
