"""DAPHNE data file format (ndt_input.dat / ndt_output.dat) and the
reference's acceptance rule."""
import numpy as np


def test_input_round_trip(pkg, tmp_path):
    rng = np.random.default_rng(1)
    cases = [(rng.normal(size=16).astype(np.float32), rng.normal(size=(n, 4)).astype(np.float32),
              rng.normal(size=(m, 4)).astype(np.float32)) for n, m in ((5, 7), (0, 3), (11, 1))]
    p = tmp_path / "ndt_input.dat"
    pkg.datfile.write_input(p, cases)
    raw = p.read_bytes()
    assert len(raw) == 4 + sum(64 + 4 + 16 * s.shape[0] + 4 + 16 * m.shape[0] for _, s, m in cases)
    back = pkg.datfile.read_input(p)
    for (g, s, m), (g2, s2, m2) in zip(cases, back):
        assert np.array_equal(g, g2) and np.array_equal(s, s2) and np.array_equal(m, m2)


def test_output_round_trip(pkg, tmp_path):
    T = np.arange(32, dtype=np.float32).reshape(2, 16)
    p = tmp_path / "ndt_output.dat"
    pkg.datfile.write_output(p, T, [1, 0], [0.5, 1.5])
    assert len(p.read_bytes()) == 2 * 73
    r = pkg.datfile.read_output(p)
    assert np.array_equal(r["T"], T) and r["converged"].tolist() == [1, 0] and r["fitness"].tolist() == [0.5, 1.5]


def test_reference_check_rule(pkg):
    I = np.eye(4, dtype=np.float32).reshape(16)
    ok, d = pkg.datfile.reference_check(I, 1, I, 1)
    assert ok and d == 0.0
    T = I.copy().reshape(4, 4)
    T[0, 3] = 0.002  # translation beyond 0.001
    assert not pkg.datfile.reference_check(T, 1, I, 1)[0]
    assert not pkg.datfile.reference_check(I, 0, I, 1)[0]  # converged differs
    N = I.copy()
    N[5] = np.nan
    assert not pkg.datfile.reference_check(N, 1, I, 1)[0]  # NaN pattern differs
    R = np.diag([-1, 1, -1, 1]).astype(np.float32).reshape(16)  # rotation error < 2 per component passes
    assert pkg.datfile.reference_check(R, 1, I, 1)[0]
