"""DAPHNE ndt_mapping data files (little-endian, packed).

ndt_input.dat  (read by ndt_mapping::read_next_testcases, src/CPU/ndt_mapping/kernel.cpp:192-229):
    int32 T; then T times: float32[16] guess (row major, parseInitGuess :165),
    int32 N + N x float32[4] scan, int32 M + M x float32[4] map (parseFilteredScan :143).
ndt_output.dat (parseResult :178-190; written by the datagen variant's writeResult):
    T times 73 bytes: float32[16] final transformation, float64 fitness, uint8 converged.
"""
from __future__ import annotations

import gzip
import struct

import numpy as np

RECORD_DTYPE = np.dtype([("T", "<f4", (16,)), ("fitness", "<f8"), ("converged", "u1")])
assert RECORD_DTYPE.itemsize == 73


def write_input(path, cases):
    """cases: iterable of (guess16 float32, scan (N,4) float32, map (M,4) float32)."""
    cases = list(cases)
    with open(path, "wb") as f:
        f.write(struct.pack("<i", len(cases)))
        for guess, scan, cloud in cases:
            f.write(np.ascontiguousarray(guess, dtype="<f4").reshape(16).tobytes())
            for arr in (scan, cloud):
                arr = np.ascontiguousarray(arr, dtype="<f4").reshape(-1, 4)
                f.write(struct.pack("<i", arr.shape[0]))
                f.write(arr.tobytes())


def read_input(path):
    """List of (guess16, scan, map) from an ndt_input.dat (optionally .gz)."""
    opener = gzip.open if str(path).endswith(".gz") else open
    with opener(path, "rb") as f:
        data = f.read()
    (T,) = struct.unpack_from("<i", data, 0)
    off = 4
    out = []
    for _ in range(T):
        guess = np.frombuffer(data, "<f4", 16, off).copy()
        off += 64
        clouds = []
        for _k in range(2):
            (n,) = struct.unpack_from("<i", data, off)
            off += 4
            clouds.append(np.frombuffer(data, "<f4", 4 * n, off).reshape(n, 4).copy())
            off += 16 * n
        out.append((guess, clouds[0], clouds[1]))
    return out


def write_output(path, transforms, converged, fitness=None):
    T = np.asarray(transforms, dtype="<f4").reshape(-1, 16)
    rec = np.zeros(T.shape[0], dtype=RECORD_DTYPE)
    rec["T"] = T
    rec["converged"] = np.asarray(converged, dtype=np.uint8)
    if fitness is not None:
        rec["fitness"] = np.asarray(fitness, dtype="<f8")
    with open(path, "wb") as f:
        f.write(rec.tobytes())


def read_output(path):
    """Structured array of 73-byte records (T, fitness, converged)."""
    opener = gzip.open if str(path).endswith(".gz") else open
    with opener(path, "rb") as f:
        data = f.read()
    if len(data) % RECORD_DTYPE.itemsize:
        raise ValueError(f"{path}: {len(data)} bytes is not a whole number of 73-byte records")
    return np.frombuffer(data, RECORD_DTYPE).copy()


# check_next_outputs (kernel.cpp:1436-1496) thresholds
MAX_TRANSLATION_EPS = 0.001
MAX_EPS = 2.0
TEST_POINT = np.array([0.724, 0.447, 0.525, 1.0], dtype=np.float32)


def reference_check(result_T, result_conv, ref_T, ref_conv):
    """The reference's own acceptance rule for one record (kernel.cpp:1447-1494).

    Returns (ok, max_delta) where max_delta is the largest translation-column or
    transformed-test-point difference (float32 arithmetic as the reference).
    """
    a = np.asarray(result_T, dtype=np.float32).reshape(4, 4)
    b = np.asarray(ref_T, dtype=np.float32).reshape(4, 4)
    ok = bool(result_conv) == bool(ref_conv)
    if not np.array_equal(np.isnan(a), np.isnan(b)):
        ok = False
    with np.errstate(invalid="ignore"):
        dt = np.abs(a[:, 3] - b[:, 3])
        ra = np.zeros(4, np.float32)
        rb = np.zeros(4, np.float32)
        for h in range(4):
            for w in range(4):
                ra[h] = np.float32(ra[h] + np.float32(a[h, w] * TEST_POINT[w]))
                rb[h] = np.float32(rb[h] + np.float32(b[h, w] * TEST_POINT[w]))
        dp = np.abs(ra - rb)
    if np.any(dt > MAX_TRANSLATION_EPS) or np.any(dp > MAX_EPS):
        ok = False
    finite = np.concatenate([dt[np.isfinite(dt)], dp[np.isfinite(dp)]])
    return ok, float(finite.max()) if finite.size else 0.0
