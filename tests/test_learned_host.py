"""Host-side helpers of the learned pipeline (CPU): the subsample rule each
refinement level applies to a scan, the level parameters handed to the C
entry point, and the order of the starts."""
import numpy as np


def test_subsample_is_the_evenly_strided_rule(pkg):
    L = pkg.learned
    rng = np.random.default_rng(3)
    for n, cap in ((10, 4), (4097, 4096), (32000, 8192), (7, 7), (5, 9), (1000, 0)):
        scan = rng.normal(size=(n, 4)).astype(np.float32)
        sub = L.subsample(scan, cap)
        m = min(n, cap) if cap else n
        assert len(sub) == m
        # point (j n) / m for j < m, as the library's subsample_kernel reads it
        assert np.array_equal(sub, scan[(np.arange(m) * n) // m])
        assert sub.flags["C_CONTIGUOUS"]


def test_pipeline_params_carry_the_level_point_budgets(pkg):
    L = pkg.learned
    levels = L.refinement_levels(0.5)
    assert [lvl["resolution"] for lvl in levels] == [2.0, 1.0, 0.5]
    prm = L.pipeline_params(levels, judge_points=1024)
    assert list(prm.level_points[:3]) == [lvl["points_per_scan"] for lvl in levels] == [4096, 8192, 0]
    assert prm.judge_points == 1024 and prm.max_points == L.NET_POINTS
    # level_params sets the NDT fields and leaves out the point budget
    p = L.level_params(pkg.ndt.corrected_params(levels[0]["resolution"]), levels[0])
    assert abs(p.step_size - levels[0]["step_size"]) < 1e-12 and p.max_iterations == levels[0]["max_iterations"]


def test_start_offsets_grid(pkg):
    L = pkg.learned
    prm = pkg.posenet.learned_params(grid_xy=3, grid_yaw=1, step_xy=1.5)
    offs = L.start_offsets(prm)
    assert len(offs) == 9
    assert sorted({round(dx, 6) for dx, _, _ in offs}) == [-1.5, 0.0, 1.5]
    assert all(d == 0.0 for _, _, d in offs)
    prm = pkg.posenet.learned_params(grid_xy=2, grid_yaw=2, step_xy=0.5, step_yaw_deg=3.0)
    offs = L.start_offsets(prm)
    assert len(offs) == 8 and {round(np.degrees(d), 6) for _, _, d in offs} == {-1.5, 1.5}
