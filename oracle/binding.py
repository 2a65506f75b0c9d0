"""ctypes bindings of the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Loaded only by tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg
and the reference arm).  Two libraries:
  * Oracle    -> oracle/_build/libndt_oracle.so (the FP64 restatement, Mode R / F)
  * Reference -> oracle/_ref/libref_ndt_{serial,omp}.so (the unmodified
                 reference kernel behind a C shim; present only where the
                 reference sources were available at build time)
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def reference_dir() -> pathlib.Path:
    """The reference source tree (read-only): $NDT_REFERENCE_DIR, else the
    directory `reference` beside this repository's checkout.  Only the
    recipes that compile the CPU checkers and the fixture generators read
    it; nothing run on a GPU machine needs it."""
    env = os.environ.get("NDT_REFERENCE_DIR")
    return pathlib.Path(env) if env else HERE.parents[1] / "reference"
ORACLE_SO = HERE / "_build" / "libndt_oracle.so"
REF_SO = {"serial": HERE / "_ref" / "libref_ndt_serial.so", "omp": HERE / "_ref" / "libref_ndt_omp.so"}

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class NdtParams(C.Structure):
    """Mirror of ndt_params (include/ndt_b200.h)."""

    _fields_ = [
        ("resolution", C.c_float),
        ("copy_groups", C.c_int32),
        ("outlier_ratio", C.c_double),
        ("step_size", C.c_double),
        ("transformation_epsilon", C.c_double),
        ("max_iterations", C.c_int32),
        ("compat", C.c_int32),
        ("min_points_per_voxel", C.c_int32),
        ("precision", C.c_int32),
        ("eigen_ratio", C.c_double),
        ("watchdog_evals", C.c_int32),
        ("dense_probe", C.c_int32),
    ]


def reference_params(resolution=1.0):
    """The values the reference kernel hard-codes (kernel.cpp:37-57)."""
    return NdtParams(resolution=resolution, outlier_ratio=0.55, step_size=0.1,
                     transformation_epsilon=0.1, max_iterations=0, compat=1,
                     min_points_per_voxel=0, precision=0, eigen_ratio=0.0, watchdog_evals=0)


def corrected_params(resolution=1.0):
    """Corrected NDT: trans_eps 0.01, 30 iterations, 6 points per voxel, 0.01 eigen floor."""
    return NdtParams(resolution=resolution, outlier_ratio=0.55, step_size=0.1,
                     transformation_epsilon=0.01, max_iterations=30, compat=0,
                     min_points_per_voxel=6, precision=0, eigen_ratio=0.01, watchdog_evals=0)


def build(quiet=True):
    """Compile the oracle (and the reference shims when the reference is present)."""
    targets = ["oracle"]
    if (reference_dir() / "src" / "CPU" / "ndt_mapping" / "kernel.cpp").exists():
        targets.append("ref")
    subprocess.run(["make", "-C", str(HERE), f"NDT_REFERENCE_DIR={reference_dir()}", *targets], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _ptr_array(arrays):
    ptrs = (C.c_void_p * len(arrays))()
    for i, a in enumerate(arrays):
        ptrs[i] = a.ctypes.data
    return ptrs


class Oracle:
    """FP64 restatement (oracle/ndt_oracle.cpp)."""

    def __init__(self, path=ORACLE_SO):
        if not pathlib.Path(path).exists():
            build()
        self.lib = L = C.CDLL(str(path))
        P = C.POINTER(NdtParams)
        L.oracle_gauss.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.oracle_align.argtypes = [P, _f32p, C.c_int, _f32p, _f32p, C.c_int, _f32p,
                                   C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.oracle_align.restype = C.c_int
        L.oracle_align_batch.argtypes = [P, C.c_int, C.c_void_p, _i32p, _f32p, _f32p, C.c_int,
                                         _f32p, _i32p, _f64p, _i32p, C.c_int]
        L.oracle_align_batch.restype = C.c_int
        L.oracle_grid.argtypes = [P, _f32p, C.c_int, _f32p, _i32p, C.c_void_p, C.c_longlong]
        L.oracle_grid.restype = C.c_longlong
        L.oracle_derivatives.argtypes = [P, _f32p, C.c_int, _f32p, _f32p, C.c_int, _f64p, C.c_int,
                                         _f64p, _f64p, C.POINTER(C.c_longlong)]
        L.oracle_derivatives.restype = C.c_double
        L.oracle_build_tm.argtypes = [C.c_int, _f64p, _f32p]
        L.oracle_pose_vector.argtypes = [C.c_int, _f32p, _f64p]
        L.oracle_solve.argtypes = [_f64p, _f64p, _f64p]
        L.oracle_invert.argtypes = [_f64p]
        L.oracle_transform.argtypes = [_f32p, C.c_int, _f32p, _f32p]
        L.oracle_trial_value.argtypes = [C.c_double] * 9
        L.oracle_trial_value.restype = C.c_double
        L.oracle_update_interval.argtypes = [_f64p, C.c_double, C.c_double, C.c_double]
        L.oracle_update_interval.restype = C.c_int
        L.oracle_radius_search.argtypes = [P, _f32p, C.c_int, _f32p, _f64p, C.c_int]
        L.oracle_radius_search.restype = C.c_int
        L.oracle_update_pair.argtypes = [P, _f64p, _f64p, _f64p, _f64p, C.c_int, _f64p, _f64p]
        L.oracle_update_pair.restype = C.c_double

    def update_pair(self, prm, p6, x, xt, icov, hessian=True, g=None, H=None):
        """One (point, cell) pair's derivative update (updateDerivatives, kernel.cpp:438-493).
        Returns (score increment, g, H) with g / H accumulated from the given ones (zeros by default)."""
        g = np.zeros(6) if g is None else np.array(g, np.float64)
        H = np.zeros(36) if H is None else np.array(H, np.float64).reshape(36)
        f = lambda a: np.ascontiguousarray(a, np.float64)  # noqa: E731
        s = self.lib.oracle_update_pair(C.byref(prm), f(p6), f(x), f(xt), f(np.reshape(icov, 9)), int(hessian), g, H)
        return s, g, H.reshape(6, 6)

    def radius_search(self, prm, cloud, pt):
        """Mode R voxelRadiusSearch (kernel.cpp:246-286): means of the neighbour cells of pt (x, y, z, w)."""
        cloud = np.ascontiguousarray(cloud, np.float32)
        means = np.zeros((64, 3))
        k = self.lib.oracle_radius_search(C.byref(prm), cloud, cloud.shape[0],
                                          np.ascontiguousarray(pt, np.float32).reshape(4), means, 64)
        if k < 0:
            raise RuntimeError(f"oracle_radius_search failed: {k}")
        return means[:k]

    def gauss(self, prm):
        d1, d2 = C.c_double(), C.c_double()
        self.lib.oracle_gauss(C.byref(prm), C.byref(d1), C.byref(d2))
        return d1.value, d2.value

    def align(self, prm, scan, guess, cloud):
        scan = np.ascontiguousarray(scan, np.float32)
        cloud = np.ascontiguousarray(cloud, np.float32)
        out = np.zeros(16, np.float32)
        conv, fit, ev = C.c_int(), C.c_double(), C.c_int()
        rc = self.lib.oracle_align(C.byref(prm), scan, scan.shape[0],
                                   np.ascontiguousarray(guess, np.float32).reshape(16), cloud,
                                   cloud.shape[0], out, C.byref(conv), C.byref(fit), C.byref(ev))
        if rc:
            raise RuntimeError(f"oracle_align failed: {rc}")
        return out, conv.value, fit.value, ev.value

    def align_batch(self, prm, scans, guesses, cloud, nthreads=None):
        scans = [np.ascontiguousarray(s, np.float32) for s in scans]
        B = len(scans)
        ns = np.array([s.shape[0] for s in scans], np.int32)
        g = np.ascontiguousarray(np.asarray(guesses, np.float32).reshape(B, 16))
        out = np.zeros((B, 16), np.float32)
        conv = np.zeros(B, np.int32)
        fit = np.zeros(B, np.float64)
        ev = np.zeros(B, np.int32)
        ptrs = _ptr_array(scans)
        cloud = np.ascontiguousarray(cloud, np.float32)
        rc = self.lib.oracle_align_batch(C.byref(prm), B, ptrs, ns, g, cloud, cloud.shape[0], out,
                                         conv, fit, ev, nthreads or os.cpu_count())
        if rc:
            raise RuntimeError(f"oracle_align_batch failed: {rc}")
        return out, conv, fit, ev

    def grid(self, prm, cloud, cells=True):
        cloud = np.ascontiguousarray(cloud, np.float32)
        bbox = np.zeros(6, np.float32)
        dims = np.zeros(3, np.int32)
        G = self.lib.oracle_grid(C.byref(prm), cloud, cloud.shape[0], bbox, dims, None, 0)
        if G < 0:
            raise RuntimeError(f"oracle_grid failed: {G}")
        arr = None
        if cells:
            arr = np.zeros((G, 13), np.float64)
            self.lib.oracle_grid(C.byref(prm), cloud, cloud.shape[0], bbox, dims, arr.ctypes.data, G)
        return bbox, dims, arr

    def derivatives(self, prm, cloud, scan, trans, p6, hessian=True):
        g = np.zeros(6)
        H = np.zeros(36)
        pairs = C.c_longlong()
        s = self.lib.oracle_derivatives(C.byref(prm), np.ascontiguousarray(cloud, np.float32),
                                        cloud.shape[0], np.ascontiguousarray(scan, np.float32),
                                        np.ascontiguousarray(trans, np.float32), scan.shape[0],
                                        np.ascontiguousarray(p6, np.float64), int(hessian), g, H,
                                        C.byref(pairs))
        return s, g, H.reshape(6, 6), pairs.value

    def build_tm(self, compat, p6, base=None):
        m = np.eye(4, dtype=np.float32).reshape(16).copy() if base is None else \
            np.ascontiguousarray(base, np.float32).reshape(16).copy()
        self.lib.oracle_build_tm(int(compat), np.ascontiguousarray(p6, np.float64), m)
        return m

    def pose_vector(self, compat, m16):
        p = np.zeros(6)
        self.lib.oracle_pose_vector(int(compat), np.ascontiguousarray(m16, np.float32).reshape(16), p)
        return p

    def solve(self, A, b):
        x = np.zeros(6)
        self.lib.oracle_solve(np.ascontiguousarray(A, np.float64).reshape(36),
                              np.ascontiguousarray(b, np.float64), x)
        return x

    def invert(self, m9):
        m = np.ascontiguousarray(m9, np.float64).reshape(9).copy()
        self.lib.oracle_invert(m)
        return m

    def transform(self, pts, m16):
        pts = np.ascontiguousarray(pts, np.float32)
        out = np.zeros_like(pts)
        self.lib.oracle_transform(pts, pts.shape[0], np.ascontiguousarray(m16, np.float32).reshape(16), out)
        return out

    def trial_value(self, *args):
        return self.lib.oracle_trial_value(*[float(a) for a in args])

    def update_interval(self, io6, a_t, f_t, g_t):
        io = np.ascontiguousarray(io6, np.float64).copy()
        r = self.lib.oracle_update_interval(io, a_t, f_t, g_t)
        return bool(r), io


class Reference:
    """The unmodified reference kernel (oracle/_ref), or None if not built."""

    def __init__(self, variant="serial"):
        path = REF_SO[variant]
        self.lib = L = C.CDLL(str(path))
        L.ref_align.argtypes = [_f32p, C.c_int, _f32p, _f32p, C.c_int, _f32p, C.POINTER(C.c_int)]
        L.ref_align.restype = C.c_int
        L.ref_align_batch.argtypes = [C.c_int, C.c_void_p, _i32p, _f32p, C.c_void_p, _i32p, _f32p,
                                      _i32p, C.c_int]
        L.ref_align_batch.restype = C.c_int
        L.ref_grid.argtypes = [_f32p, C.c_int, _f32p, _i32p, C.c_void_p, C.c_longlong]
        L.ref_grid.restype = C.c_longlong
        L.ref_derivatives.argtypes = [_f32p, C.c_int, _f32p, _f32p, C.c_int, _f64p, C.c_double,
                                      C.c_double, C.c_int, _f64p, _f64p]
        L.ref_derivatives.restype = C.c_double
        L.ref_radius_search.argtypes = [_f32p, C.c_int, _f32p, _f64p, C.c_int]
        L.ref_radius_search.restype = C.c_int
        L.ref_update_pair.argtypes = [_f64p, _f64p, _f64p, _f64p, C.c_double, C.c_double, C.c_int, _f64p, _f64p]
        L.ref_update_pair.restype = C.c_double
        L.ref_angle_terms.argtypes = [_f64p, _f64p]
        L.ref_build_tm.argtypes = [_f64p, _f32p]
        L.ref_euler.argtypes = [_f32p, _f64p]
        L.ref_solve.argtypes = [_f64p, _f64p, _f64p]
        L.ref_invert.argtypes = [_f64p]
        L.ref_transform.argtypes = [_f32p, C.c_int, _f32p, _f32p]
        L.ref_trial_value.argtypes = [C.c_double] * 9
        L.ref_trial_value.restype = C.c_double
        L.ref_update_interval.argtypes = [_f64p, C.c_double, C.c_double, C.c_double]
        L.ref_update_interval.restype = C.c_int

    @staticmethod
    def available(variant="serial"):
        return REF_SO[variant].exists()

    def align(self, scan, guess, cloud):
        scan = np.ascontiguousarray(scan, np.float32)
        cloud = np.ascontiguousarray(cloud, np.float32)
        out = np.zeros(16, np.float32)
        conv = C.c_int()
        rc = self.lib.ref_align(scan, scan.shape[0], np.ascontiguousarray(guess, np.float32).reshape(16),
                                cloud, cloud.shape[0], out, C.byref(conv))
        if rc:
            raise RuntimeError(f"ref_align failed: {rc}")
        return out, conv.value

    def align_batch(self, scans, guesses, clouds, nthreads=1):
        scans = [np.ascontiguousarray(s, np.float32) for s in scans]
        clouds = [np.ascontiguousarray(c, np.float32) for c in clouds]
        B = len(scans)
        ns = np.array([s.shape[0] for s in scans], np.int32)
        ms = np.array([c.shape[0] for c in clouds], np.int32)
        g = np.ascontiguousarray(np.asarray(guesses, np.float32).reshape(B, 16))
        out = np.zeros((B, 16), np.float32)
        conv = np.zeros(B, np.int32)
        rc = self.lib.ref_align_batch(B, _ptr_array(scans), ns, g, _ptr_array(clouds), ms, out, conv,
                                      nthreads)
        if rc:
            raise RuntimeError(f"ref_align_batch failed: {rc}")
        return out, conv

    def grid(self, cloud, cells=True):
        cloud = np.ascontiguousarray(cloud, np.float32)
        bbox = np.zeros(6, np.float32)
        dims = np.zeros(3, np.int32)
        G = self.lib.ref_grid(cloud, cloud.shape[0], bbox, dims, None, 0)
        arr = None
        if cells:
            arr = np.zeros((G, 13), np.float64)
            self.lib.ref_grid(cloud, cloud.shape[0], bbox, dims, arr.ctypes.data, G)
        return bbox, dims, arr

    def derivatives(self, cloud, scan, trans, p6, d1, d2, hessian=True):
        g = np.zeros(6)
        H = np.zeros(36)
        s = self.lib.ref_derivatives(np.ascontiguousarray(cloud, np.float32), cloud.shape[0],
                                     np.ascontiguousarray(scan, np.float32),
                                     np.ascontiguousarray(trans, np.float32), scan.shape[0],
                                     np.ascontiguousarray(p6, np.float64), d1, d2, int(hessian), g, H)
        return s, g, H.reshape(6, 6)

    def angle_terms(self, p6):
        """computeAngleDerivatives (kernel.cpp:707-825): j_ang a..h then h_ang a2..f3, 3 each (69 doubles)."""
        out = np.zeros(69)
        self.lib.ref_angle_terms(np.ascontiguousarray(p6, np.float64), out)
        return out

    def update_pair(self, p6, x, xt, icov, d1, d2, hessian=True, g=None, H=None):
        """The reference's computeAngleDerivatives + computePointDerivatives + updateDerivatives for one pair."""
        g = np.zeros(6) if g is None else np.array(g, np.float64)
        H = np.zeros(36) if H is None else np.array(H, np.float64).reshape(36)
        f = lambda a: np.ascontiguousarray(a, np.float64)  # noqa: E731
        s = self.lib.ref_update_pair(f(p6), f(x), f(xt), f(np.reshape(icov, 9)), d1, d2, int(hessian), g, H)
        return s, g, H.reshape(6, 6)

    def radius_search(self, cloud, pt):
        """The reference's voxelRadiusSearch (kernel.cpp:246-286) on the grid of cloud."""
        cloud = np.ascontiguousarray(cloud, np.float32)
        means = np.zeros((64, 3))
        k = self.lib.ref_radius_search(cloud, cloud.shape[0], np.ascontiguousarray(pt, np.float32).reshape(4),
                                       means, 64)
        return means[:min(k, 64)]

    def build_tm(self, p6, base=None):
        m = np.eye(4, dtype=np.float32).reshape(16).copy() if base is None else \
            np.ascontiguousarray(base, np.float32).reshape(16).copy()
        self.lib.ref_build_tm(np.ascontiguousarray(p6, np.float64), m)
        return m

    def euler(self, m16):
        out = np.zeros(3)
        self.lib.ref_euler(np.ascontiguousarray(m16, np.float32).reshape(16), out)
        return out

    def solve(self, A, b):
        x = np.zeros(6)
        self.lib.ref_solve(np.ascontiguousarray(A, np.float64).reshape(36),
                           np.ascontiguousarray(b, np.float64), x)
        return x

    def invert(self, m9):
        m = np.ascontiguousarray(m9, np.float64).reshape(9).copy()
        self.lib.ref_invert(m)
        return m

    def transform(self, pts, m16):
        pts = np.ascontiguousarray(pts, np.float32)
        out = np.zeros_like(pts)
        self.lib.ref_transform(pts, pts.shape[0], np.ascontiguousarray(m16, np.float32).reshape(16), out)
        return out

    def trial_value(self, *args):
        return self.lib.ref_trial_value(*[float(a) for a in args])

    def update_interval(self, io6, a_t, f_t, g_t):
        io = np.ascontiguousarray(io6, np.float64).copy()
        r = self.lib.ref_update_interval(io, a_t, f_t, g_t)
        return bool(r), io


if __name__ == "__main__":  # pragma: no cover
    build(quiet=False)
    sys.exit(0)
