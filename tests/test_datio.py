"""The input file's fast path (ndt_dat_open / _case / _map_relation): the
memory-mapped index agrees with the file's contents, map relations are found,
and malformed files are rejected with a message (no GPU needed)."""
import numpy as np
import pytest


def _cases(rng):
    A = rng.normal(0, 20, (3000, 4)).astype(np.float32)
    B = rng.normal(0, 20, (2000, 4)).astype(np.float32)
    grown = np.concatenate([A, rng.normal(0, 20, (500, 4)).astype(np.float32)])
    out = []
    for mp in (A, A, grown, B, B, A):
        out.append((rng.normal(0, 1, 16).astype(np.float32), rng.normal(0, 5, (int(rng.integers(0, 400)), 4))
                    .astype(np.float32), mp))
    return out


def test_index_and_relations(pkg, tmp_path):
    rng = np.random.default_rng(1)
    cases = _cases(rng)
    path = tmp_path / "ndt_input.dat"
    pkg.datfile.write_input(path, cases)
    with pkg.ndt.DatFile(path) as f:
        assert len(f) == len(cases)
        for i, (g, s, m) in enumerate(cases):
            g2, s2, m2 = f.case(i)
            assert np.array_equal(g2, g) and np.array_equal(s2, s) and np.array_equal(m2, m)
        D = pkg.ndt.DatFile
        assert [f.relation(i) for i in range(len(cases))] == [D.MAP_NEW, D.MAP_SAME, D.MAP_GROWN, D.MAP_NEW,
                                                              D.MAP_SAME, D.MAP_NEW]


def test_malformed_files(pkg, tmp_path):
    rng = np.random.default_rng(2)
    path = tmp_path / "ndt_input.dat"
    pkg.datfile.write_input(path, _cases(rng))
    data = path.read_bytes()
    short = tmp_path / "short.dat"
    short.write_bytes(data[:-100])
    with pytest.raises(pkg.ndt.NdtError, match="file ends inside test case 5"):
        pkg.ndt.DatFile(short)
    neg = tmp_path / "neg.dat"
    neg.write_bytes(data[:4 + 64] + np.int32(-3).tobytes() + data[4 + 64 + 4:])
    with pytest.raises(pkg.ndt.NdtError, match="negative point count"):
        pkg.ndt.DatFile(neg)
    with pytest.raises(pkg.ndt.NdtError, match="Error opening the testcase file"):
        pkg.ndt.DatFile(tmp_path / "missing.dat")
    empty = tmp_path / "empty.dat"
    empty.write_bytes(np.int32(0).tobytes())
    with pkg.ndt.DatFile(empty) as f:
        assert len(f) == 0
