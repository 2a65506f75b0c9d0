"""The euclidean-clustering checkers (no GPU): the brute-force labels agree
with the compiled reference kernel's clusters on small clouds, and the golden
fixture agrees with the reference where the reference tree exists here."""
import pathlib

import numpy as np
import pytest

import binding
import ec_ref

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "ec_cases.npz"


def _clusters_from_labels(lab, lo=20, hi=100000):
    # the reference's order: components by smallest index, sizes filtered, then a size sort.  Python's sort is
    # stable while the reference's std::sort is not, so compare as a multiset of (size, indices).
    groups = {}
    for i, l in enumerate(lab):
        groups.setdefault(int(l), []).append(i)
    return sorted((len(g), tuple(g)) for g in groups.values() if lo <= len(g) <= hi)


@pytest.mark.skipif(not ec_ref.Reference.available(), reason="compiled reference (oracle/_ref) not built here")
@pytest.mark.parametrize("tol", [0.5, 1.1])
def test_brute_labels_match_reference(tol):
    rng = np.random.default_rng(7)
    xyz = np.concatenate([rng.normal(c, 0.4, (60, 3)) for c in rng.uniform(-8, 8, (12, 3))]).astype(np.float32)
    ref = ec_ref.Reference().extract(xyz, tol)
    assert sorted((len(c), tuple(c)) for c in ref) == _clusters_from_labels(ec_ref.brute_labels(xyz, tol))


def test_fixture_shape():
    d = np.load(GOLDEN)
    T = int(d["cases"])
    assert T == 5
    for i in range(T):
        n = len(d[f"in{i}"])
        total = sum(int(d[f"sizes{i}_{k}"].sum()) for k in range(5))
        assert total == int(d[f"npts{i}"]) and total <= n
        assert len(d[f"boxes{i}"]) == len(d[f"centroids{i}"])


REF_DATA = binding.reference_dir() / "data"


@pytest.mark.skipif(not (ec_ref.Reference.available() and (REF_DATA / "ec_output.dat.gz").exists()),
                    reason="reference tree not present")
def test_reference_reproduces_its_shipped_output():
    ins = ec_ref.read_input(str(REF_DATA / "ec_input.dat.gz"))
    outs = ec_ref.read_output(str(REF_DATA / "ec_output.dat.gz"), len(ins))
    ref = ec_ref.Reference()
    for xyz, out in list(zip(ins, outs))[:2]:
        pts, b10, cen = ref.segment(xyz)
        ok, d = ec_ref.check(pts, ec_ref.boxes10_to_8(b10), cen, out[0], out[2], out[3])
        assert ok and d == 0.0
