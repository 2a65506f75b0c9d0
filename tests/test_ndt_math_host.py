"""The device-side NDT math (daphne-benchmark_b200/csrc/ndt_math.cuh: angle
terms, pose build, pose vector, 6x6 solve, More-Thuente trial value and interval update)
built as host code (tests/native/ndt_math_host.cpp) and compared bit for bit
with the reference's own routines (oracle/_ref) on many random inputs,
including singular systems and degenerate line-search states; the corrected
mode's pose build and pose vector, which the reference does not have, with
the FP64 oracle's.  The host
build uses the same libm as the reference, so this checks each expression's
operations and order; the device's own libm results are covered by the GPU
parity tests."""
import ctypes as C
import math
import pathlib
import shutil
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
CUDA_INC = pathlib.Path("/usr/local/cuda/include")
pytestmark = pytest.mark.skipif(not (shutil.which("g++") and CUDA_INC.is_dir()),
                                reason="needs g++ and the CUDA headers")


@pytest.fixture(scope="module")
def ndtm(tmp_path_factory):
    so = tmp_path_factory.mktemp("ndtm") / "libndtm.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", f"-I{CUDA_INC}",
                    f"-I{ROOT / 'daphne-benchmark_b200' / 'csrc'}", str(ROOT / "tests" / "native" / "ndt_math_host.cpp"),
                    "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    d, f = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"), np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    L.ndtm_angle_terms.argtypes = [d, C.c_int, d]
    L.ndtm_build_tm_compat.argtypes = [d, f]
    L.ndtm_build_tm_corrected.argtypes = [d, f]
    L.ndtm_pose_vector.argtypes = [C.c_int, f, d]
    L.ndtm_solve6.argtypes = [d, d, d]
    L.ndtm_trial_value.argtypes = [C.c_double] * 9
    L.ndtm_trial_value.restype = C.c_double
    L.ndtm_update_interval.argtypes = [d, C.c_double, C.c_double, C.c_double]
    L.ndtm_update_interval.restype = C.c_int
    return L


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.array_equal(a.view(np.uint64 if a.dtype == np.float64 else np.uint32),
                          b.view(np.uint64 if b.dtype == np.float64 else np.uint32)) or \
        (np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)]))


def test_pose_build_and_vector(ndtm, reference):
    rng = np.random.default_rng(1)
    for t in range(20000):
        p = rng.uniform(-4, 4, 6) if t % 5 else rng.uniform(-1e-4, 1e-4, 6)
        base = rng.uniform(-5, 5, 16).astype(np.float32)
        ours = base.copy()
        ndtm.ndtm_build_tm_compat(np.ascontiguousarray(p), ours)
        assert _same(ours, reference.build_tm(p, base)), p
        pv = np.zeros(6)
        ndtm.ndtm_pose_vector(1, ours, pv)
        assert _same(pv[3:], reference.euler(ours)), p


def test_solve6(ndtm, reference):
    rng = np.random.default_rng(2)
    for t in range(20000):
        A = rng.normal(size=(6, 6))
        if t % 4 == 1:
            A[:, rng.integers(0, 6)] = 0.0  # a zero pivot column: the reference's 0.001 fill
        if t % 4 == 2:
            A[rng.integers(0, 6)] = A[rng.integers(0, 6)] * 2.0  # dependent rows
        b = rng.normal(size=6)
        x = np.zeros(6)
        ndtm.ndtm_solve6(np.ascontiguousarray(A.reshape(36)), b, x)
        assert _same(x, reference.solve(A, b)), t


def test_more_thuente_helpers(ndtm, reference):
    rng = np.random.default_rng(3)
    for t in range(100000):
        v = rng.normal(size=9)
        v[0], v[3], v[6] = np.sort(rng.uniform(0, 1, 3)) if t % 2 else rng.uniform(0, 1, 3)
        if t % 11 == 0:
            v[8] = v[2]  # equal slopes: the interpolation's degenerate denominators
        if t % 13 == 0:
            v[7] = v[1]
        a = ndtm.ndtm_trial_value(*map(float, v))
        b = reference.trial_value(*map(float, v))
        assert a == b or (math.isnan(a) and math.isnan(b)), (t, v)
        io = rng.normal(size=6)
        at, ft, gt = rng.normal(size=3)
        if t % 7 == 0:
            gt = 0.0  # neither branch of the slope test: the interval is converged
        io_ours = np.ascontiguousarray(io.copy())
        c1 = ndtm.ndtm_update_interval(io_ours, at, ft, gt)
        c2, io_ref = reference.update_interval(io, at, ft, gt)
        assert c1 == c2 and _same(io_ours, io_ref), t


def test_angle_terms(ndtm, reference):
    """compat: the reference's computeAngleDerivatives bit for bit (incl. the exact 0 / 1 of |angle| < 1e-4);
    corrected: the same except h_ang_d1's z component, -sin(pitch) instead of +sin(pitch)."""
    rng = np.random.default_rng(4)
    for t in range(20000):
        p = rng.uniform(-3.5, 3.5, 6)
        if t % 3 == 0:
            p[3 + rng.integers(0, 3)] = rng.uniform(-2e-4, 2e-4)
        ref = reference.angle_terms(p)
        ours = np.zeros(69)
        ndtm.ndtm_angle_terms(np.ascontiguousarray(p), 1, ours)
        assert _same(ours, ref), p
        ndtm.ndtm_angle_terms(np.ascontiguousarray(p), 0, ours)
        d1z = 24 + 6 * 3 + 2  # h_ang d1, z
        assert ours[d1z] == -ref[d1z]
        ours[d1z] = ref[d1z]
        assert _same(ours, ref), p


def test_corrected_pose_build_and_vector_equal_the_oracle(ndtm, oracle):
    """The corrected mode's T = Trans * Rx * Ry * Rz and its inverse: the device code and the FP64 oracle agree
    bit for bit (host libm on both sides)."""
    rng = np.random.default_rng(5)
    for t in range(20000):
        p = rng.uniform(-3, 3, 6)
        if t % 4 == 0:
            p[3:] = rng.uniform(-1.5, 1.5, 3)
        ours = np.zeros(16, np.float32)
        ndtm.ndtm_build_tm_corrected(np.ascontiguousarray(p), ours)
        assert _same(ours, oracle.build_tm(0, p)), p
        pv = np.zeros(6)
        ndtm.ndtm_pose_vector(0, ours, pv)
        assert _same(pv, oracle.pose_vector(0, ours)), p
