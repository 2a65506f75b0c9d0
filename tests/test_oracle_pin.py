"""Pin the CPU oracle (oracle/ndt_oracle.cpp) to the reference.

1. Against the golden fixtures (tests/golden/reference_cases.json, produced by
   the compiled, unmodified reference kernel): full alignments, voxel grids
   and derivative evaluations agree bit for bit.
2. Against the compiled reference itself (oracle/_ref, when built here) on
   extra seeds and edge cases, and function by function (known-answer tests
   of buildTransformationMatrix, eulerAngles, solve, invertMatrix,
   transformPointCloud, trialValueSelectionMT, updateIntervalMT).
3. The reference's own golden output file (data/ndt_output.dat.gz, 5 records;
   its input file is not distributed): format and the structural facts the
   reference's code implies.
"""
import hashlib
import json
import math
import pathlib

import numpy as np
import pytest

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def _cases():
    return json.loads((GOLDEN / "reference_cases.json").read_text())["cases"]


def _inputs(pkg, c, cache={}):
    cfg = c["config"]
    conf = pkg.synth.Config(cfg["name"], cfg["map_points"], cfg["area"], cfg["walls"], cfg["resolution"], 1,
                            cfg["scan_min"], cfg["scan_min"], False, cfg["dt"], cfg["dyaw_deg"], radius=cfg["radius"],
                            seed=cfg["seed"])
    key = (conf.seed, conf.map_points, conf.area, conf.walls)
    if key not in cache:
        cache[key] = pkg.synth.make_scene(conf)
    scene = cache[key]
    a = pkg.synth.make_alignment(conf, scene, c["index"])
    assert pkg.synth.digest(a.scan, a.guess, scene.map) == c["input_sha256"]
    return conf, scene, a


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_oracle_matches_reference_fixture(pkg, oracle, binding_mod, case):
    conf, scene, a = _inputs(pkg, case)
    prm = binding_mod.reference_params(conf.resolution)
    out, conv, _, evals = oracle.align(prm, a.scan, a.guess, scene.map)
    assert out.view(np.uint32).tolist() == case["out_bits"]
    assert conv == case["converged"]
    assert evals <= 3  # Mode R: one evaluation at the guess + at most one per Newton iteration
    if case["grid"] is not None:
        bbox, dims, cells = oracle.grid(prm, scene.map)
        assert bbox.view(np.uint32).tolist() == case["grid"]["bbox_bits"]
        assert dims.tolist() == case["grid"]["dims"]
        occ = cells[cells[:, 12] > 0]
        assert occ.shape[0] == case["grid"]["occupied"]
        assert hashlib.sha256(np.ascontiguousarray(occ).tobytes()).hexdigest() == case["grid"]["occupied_sha256"]
    if case["derivatives"] is not None:
        d = case["derivatives"]
        trans = oracle.transform(a.scan, a.guess)
        s, g, H, pairs = oracle.derivatives(prm, scene.map, a.scan, trans, np.array(d["p6"]))
        assert s == d["score"]
        assert g.tolist() == d["gradient"]
        assert H.reshape(36).tolist() == d["hessian"]


def _edge_inputs(pkg):
    cfg = pkg.synth.small_config("edge", 8000, 30.0, 10, 500, seed=11)
    scene = pkg.synth.make_scene(cfg)
    a = pkg.synth.make_alignment(cfg, scene, 0)
    far = a.guess.copy()
    far[3] += 1000.0
    ident = np.eye(4, dtype=np.float32).reshape(16)
    return [
        ("regular", a.scan, a.guess, scene.map),
        ("no_overlap", a.scan, far, scene.map),
        ("map_1_point", a.scan, a.guess, scene.map[:1]),
        ("map_5_points", a.scan, a.guess, scene.map[:5]),
        ("map_duplicates", a.scan, a.guess, np.repeat(scene.map[:1], 50, axis=0)),
        ("scan_1_point", a.scan[:1], a.guess, scene.map),
        ("identity_guess", a.scan, ident, scene.map),
        ("map_100_points", a.scan, a.guess, scene.map[:100]),
    ]


def test_oracle_matches_compiled_reference_edges(pkg, oracle, reference, binding_mod):
    prm = binding_mod.reference_params()
    for name, scan, guess, cloud in _edge_inputs(pkg):
        r_out, r_conv = reference.align(scan, guess, cloud)
        o_out, o_conv, _, _ = oracle.align(prm, scan, guess, cloud)
        assert np.array_equal(r_out.view(np.uint32), o_out.view(np.uint32)), name
        assert r_conv == o_conv, name


@pytest.mark.slow
def test_oracle_matches_compiled_reference_seeds(pkg, oracle, reference, binding_mod):
    prm = binding_mod.reference_params()
    cfg = pkg.synth.CONFIGS["c1"]
    scene = pkg.synth.make_scene(cfg)
    for i in range(2, 8):
        a = pkg.synth.make_alignment(cfg, scene, i)
        r_out, r_conv = reference.align(a.scan, a.guess, scene.map)
        o_out, o_conv, _, _ = oracle.align(prm, a.scan, a.guess, scene.map)
        assert np.array_equal(r_out.view(np.uint32), o_out.view(np.uint32)), i
    rb, rcells = reference.grid(scene.map)[0], reference.grid(scene.map)[2]
    ob, _, ocells = oracle.grid(prm, scene.map)
    same = (rcells.view(np.uint64) == ocells.view(np.uint64)) | (np.isnan(rcells) & np.isnan(ocells))
    assert same.all() and np.array_equal(rb, ob)


def test_build_tm_known_answers(oracle, binding_mod):
    # buildTransformationMatrix(0) is diag(-1, 1, -1), not the identity
    # (permuted quaternion components, kernel.cpp:971-980)
    m = oracle.build_tm(1, np.zeros(6)).reshape(4, 4)
    assert np.array_equal(m[:3, :3], np.diag([-1.0, 1.0, -1.0]).astype(np.float32))
    # the translation column keeps its previous value (never written, kernel.cpp:1000-1012)
    base = np.eye(4, dtype=np.float32)
    base[:3, 3] = [1.5, -2.0, 3.25]
    m = oracle.build_tm(1, np.array([9.0, 9.0, 9.0, 0.1, -0.2, 0.3]), base.reshape(16)).reshape(4, 4)
    assert m[:3, 3].tolist() == [1.5, -2.0, 3.25]
    assert m[3].tolist() == [0.0, 0.0, 0.0, 1.0]
    # corrected build is Trans * Rx * Ry * Rz
    p = np.array([1.0, 2.0, 3.0, 0.1, -0.2, 0.3])
    m = oracle.build_tm(0, p).reshape(4, 4).astype(np.float64)
    a, b, c = p[3:]
    Rx = np.array([[1, 0, 0], [0, math.cos(a), -math.sin(a)], [0, math.sin(a), math.cos(a)]])
    Ry = np.array([[math.cos(b), 0, math.sin(b)], [0, 1, 0], [-math.sin(b), 0, math.cos(b)]])
    Rz = np.array([[math.cos(c), -math.sin(c), 0], [math.sin(c), math.cos(c), 0], [0, 0, 1]])
    assert np.allclose(m[:3, :3], Rx @ Ry @ Rz, atol=1e-6)
    assert np.allclose(m[:3, 3], p[:3])
    # and its pose vector inverts it
    assert np.allclose(oracle.pose_vector(0, m.astype(np.float32).reshape(16)), p, atol=1e-6)


def test_pose_helpers_match_reference(oracle, reference):
    rng = np.random.default_rng(7)
    for _ in range(50):
        p = rng.uniform(-3, 3, 6)
        base = rng.uniform(-5, 5, 16).astype(np.float32)
        assert np.array_equal(oracle.build_tm(1, p, base).view(np.uint32), reference.build_tm(p, base).view(np.uint32))
        m = reference.build_tm(p, base)
        assert np.array_equal(oracle.pose_vector(1, m)[3:], reference.euler(m))
    # yaw-only rotation: the reference's pose vector is (0, 0, yaw) negated twice -> (0, 0, psi)
    psi = 0.3
    m = np.eye(4, dtype=np.float32)
    m[0, 0], m[0, 1], m[1, 0], m[1, 1] = math.cos(psi), -math.sin(psi), math.sin(psi), math.cos(psi)
    e = reference.euler(m.reshape(16))
    assert abs(e[0]) < 1e-7 and abs(e[1]) < 1e-7 and abs(abs(e[2]) - psi) < 1e-6


def test_solve_invert_transform_match_reference(oracle, reference):
    rng = np.random.default_rng(3)
    for _ in range(20):
        A = rng.normal(size=(6, 6))
        b = rng.normal(size=6)
        assert np.array_equal(oracle.solve(A, b), reference.solve(A, b))
        m = rng.normal(size=9)
        assert np.array_equal(oracle.invert(m), reference.invert(m))
    # singular system: zero pivot replaced by 0.001 (kernel.cpp:317-320)
    A = np.zeros((6, 6))
    b = np.ones(6)
    x = oracle.solve(A, b)
    assert np.array_equal(x, reference.solve(A, b)) and np.allclose(x, 1000.0)
    # singular 3x3: inf / nan entries as the reference
    s = np.array([1.0, 2, 3, 2, 4, 6, 1, 1, 1])
    assert np.array_equal(np.isnan(oracle.invert(s)), np.isnan(reference.invert(s)))
    pts = rng.uniform(-50, 50, (100, 4)).astype(np.float32)
    T = rng.uniform(-2, 2, 16).astype(np.float32)
    assert np.array_equal(oracle.transform(pts, T)[:, :3], reference.transform(pts, T)[:, :3])


def test_more_thuente_helpers_match_reference(oracle, reference):
    rng = np.random.default_rng(5)
    for _ in range(200):
        args = rng.normal(size=9)
        args[0], args[3], args[6] = sorted(rng.uniform(0, 1, 3))
        a, b = oracle.trial_value(*args), reference.trial_value(*args)
        assert (a == b) or (math.isnan(a) and math.isnan(b))
        io = rng.normal(size=6)
        at, ft, gt = rng.normal(size=3)
        c1, o1 = oracle.update_interval(io, at, ft, gt)
        c2, o2 = reference.update_interval(io, at, ft, gt)
        assert c1 == c2 and np.array_equal(o1, o2)


def test_gauss_constants(oracle, binding_mod):
    d1, d2 = oracle.gauss(binding_mod.reference_params())
    # outlier 0.55, resolution 1 (kernel.cpp:1181-1185)
    c1, c2 = 10 * (1 - 0.55), 0.55
    d3 = -math.log(c2)
    e1 = -math.log(c1 + c2) - d3
    e2 = -2 * math.log((-math.log(c1 * math.exp(-0.5) + c2) - d3) / e1)
    assert d1 == e1 and d2 == e2


def test_reference_golden_output_file(pkg):
    """The 5 records of the reference's data/ndt_output.dat.gz."""
    d = json.loads((GOLDEN / "reference_ndt_output.json").read_text())
    recs = d["records"]
    assert len(recs) == 5
    raw = b""
    for r in recs:
        T = np.array(r["T_bits"], np.uint32).view(np.float32)
        raw += T.tobytes() + np.array([r["fitness_bits"]], np.uint64).tobytes() + bytes([r["converged"]])
    assert len(raw) == 5 * 73
    path = pathlib.Path(__import__("tempfile").mkdtemp()) / "ndt_output.dat"
    path.write_bytes(raw)
    parsed = pkg.datfile.read_output(path)
    for r, p in zip(recs, parsed):
        T = p["T"].reshape(4, 4).astype(np.float64)
        # converged is always true (two Newton iterations, kernel.cpp:1261)
        assert p["converged"] == 1 and r["converged"] == 1
        # row 3 is (0, 0, 0, 1) and the translation column is the guess's
        # (never written by buildTransformationMatrix; the golden guesses were at the origin)
        assert T[3].tolist() == [0.0, 0.0, 0.0, 1.0]
        assert T[:3, 3].tolist() == [0.0, 0.0, 0.0]
        # the rotation block is a proper rotation (float accuracy)
        R = T[:3, :3]
        assert np.allclose(R @ R.T, np.eye(3), atol=2e-5) and abs(np.linalg.det(R) - 1) < 2e-5


def test_radius_search_known_answers(oracle, reference, binding_mod):
    """voxelRadiusSearch (kernel.cpp:246-286): 27 float probes p + {-r, 0, r}^3, each skipped outside the
    bounding box; cells kept when the float distance to their mean is < r.  Oracle == reference (same cells,
    same order) at the box's corners, edges and faces, on cell boundaries, inside and far outside."""
    prm = binding_mod.reference_params()
    rng = np.random.default_rng(21)
    cloud = np.ones((3000, 4), np.float32)
    cloud[:, :3] = rng.uniform([0, 0, 0], [9.5, 7.25, 2.5], (3000, 3)).astype(np.float32)
    bbox = reference.grid(cloud, cells=False)[0]
    lo, hi = bbox[:3].astype(np.float64), bbox[3:].astype(np.float64)
    probes = []
    for cx in (lo[0], hi[0], (lo[0] + hi[0]) / 2):
        for cy in (lo[1], hi[1], (lo[1] + hi[1]) / 2):
            for cz in (lo[2], hi[2], (lo[2] + hi[2]) / 2):
                for d in (-0.6, -0.001, 0.0, 0.001, 0.6):
                    probes.append((cx + d, cy - d, cz + d))
    for k in range(1, 6):  # exactly on cell boundaries
        probes.append((lo[0] + k, lo[1] + k, lo[2] + 1))
    probes += [tuple(p) for p in rng.uniform(lo - 1.5, hi + 1.5, (200, 3))]
    probes.append((lo[0] - 50, lo[1], lo[2]))  # far outside: every probe skipped
    counts = []
    for p in probes:
        pt = np.array([p[0], p[1], p[2], 1.0], np.float32)
        r, o = reference.radius_search(cloud, pt), oracle.radius_search(prm, cloud, pt)
        assert np.array_equal(r.view(np.uint64), o.view(np.uint64)) or \
            (r.shape == o.shape and np.array_equal(np.isnan(r), np.isnan(o)) and np.array_equal(r[~np.isnan(r)], o[~np.isnan(o)])), p
        counts.append(len(o))
        assert len(o) <= 27
    assert counts[-1] == 0
    assert max(counts) >= 4  # cells count only when their mean is within r, so far fewer than 27


def test_update_derivatives_known_answers(oracle, reference, binding_mod):
    """updateDerivatives (kernel.cpp:438-493) pair by pair: oracle == reference bit for bit (score increment,
    gradient, Hessian; with and without the Hessian; near-zero angles take the reference's exact 0 / 1 branch),
    and the rejection branch: when d2 * exp(-d2 xCx / 2) leaves [0, 1] or is NaN the pair adds nothing."""
    prm = binding_mod.reference_params()
    d1, d2 = oracle.gauss(prm)
    rng = np.random.default_rng(17)
    for t in range(300):
        p = rng.uniform(-0.5, 0.5, 6)
        if t % 4 == 0:
            p[3:] = rng.uniform(-5e-5, 5e-5, 3)  # |angle| < 1e-4: cos 1, sin 0 (kernel.cpp:710-726)
        x = rng.uniform(-30, 30, 3)
        xt = rng.normal(0, 0.4, 3)
        A = rng.normal(size=(3, 3))
        icov = A @ A.T + 0.1 * np.eye(3)
        g0, H0 = rng.normal(size=6), rng.normal(size=36)
        for hess in (True, False):
            so, go, Ho = oracle.update_pair(prm, p, x, xt, icov, hess, g0, H0)
            sr, gr, Hr = reference.update_pair(p, x, xt, icov, d1, d2, hess, g0, H0)
            assert so == sr and np.array_equal(go, gr) and np.array_equal(Ho, Hr), (t, hess)
    # known answer of an accepted pair: score increment -d1 exp(-d2 xCx / 2)
    xt = np.array([0.1, -0.2, 0.05])
    s, g, H = oracle.update_pair(prm, np.zeros(6), np.ones(3), xt, np.eye(3))
    assert math.isclose(s, -d1 * math.exp(-d2 * float(xt @ xt) / 2), rel_tol=1e-15)
    # rejection: an indefinite inverse covariance makes xCx < 0, e * d2 > 1 -> nothing added
    g0, H0 = np.arange(6.0), np.arange(36.0)
    for icov, xt in ((-np.eye(3), np.array([2.0, 2.0, 2.0])), (np.eye(3), np.array([np.nan, 0.0, 0.0]))):
        so, go, Ho = oracle.update_pair(prm, np.full(6, 0.1), np.ones(3), xt, icov, True, g0, H0)
        sr, gr, Hr = reference.update_pair(np.full(6, 0.1), np.ones(3), xt, icov, d1, d2, True, g0, H0)
        assert so == 0.0 and sr == 0.0
        assert np.array_equal(go, g0) and np.array_equal(gr, g0)
        assert np.array_equal(Ho.reshape(36), H0) and np.array_equal(Hr.reshape(36), H0)
