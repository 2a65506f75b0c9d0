"""ctypes binding of libndt_b200.so (include/ndt_b200.h) with numpy buffers.

The host-side mirror of the reference's align call: `Context.align(scan, guess)`
is partial_points_callback (src/CPU/ndt_mapping/kernel.cpp:1405) against the
map set by `Context.set_map`, returning (final_transformation[16], converged,
fitness).  There is no CPU fallback: loading fails loudly when the CUDA library
has not been built, and every call raises NdtError when the library reports an
error (no device, bad argument, ...).
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "_build" / "libndt_b200.so"
CSRC = PKG / "csrc"

NDT_OK = 0
ERRORS = {-1: "NDT_E_ARG", -2: "NDT_E_CUDA", -3: "NDT_E_NOMAP", -4: "NDT_E_GRID", -5: "NDT_E_WATCHDOG",
          -6: "NDT_E_CAPACITY"}

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class NdtError(RuntimeError):
    pass


class Params(C.Structure):
    """ndt_params (include/ndt_b200.h)."""

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


class Counters(C.Structure):
    """ndt_counters (include/ndt_b200.h)."""

    _fields_ = [("evaluations", C.c_int64), ("points", C.c_int64), ("probes", C.c_int64),
                ("occupied_probes", C.c_int64), ("pairs", C.c_int64), ("tiles", C.c_int64), ("launches", C.c_int64),
                ("rounds", C.c_int64), ("deriv_launches", C.c_int64), ("deriv_ms", C.c_double),
                ("grid_ms", C.c_double)]


def build(quiet=True):
    """Compile libndt_b200.so for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-C", str(CSRC), "-j4"], check=True, stdout=subprocess.DEVNULL if quiet else None)
    return LIB_PATH


_LIB = None


def lib():
    """The loaded CUDA library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise NdtError(f"{LIB_PATH} is missing: build the CUDA library first (make -C {CSRC})")
        L = C.CDLL(str(LIB_PATH))
        P = C.POINTER(Params)
        ctxp = C.c_void_p
        L.ndt_params_reference.argtypes = [P]
        L.ndt_params_corrected.argtypes = [P]
        L.ndt_create.argtypes = [P, C.c_int, C.POINTER(ctxp)]
        L.ndt_destroy.argtypes = [ctxp]
        L.ndt_last_error.argtypes = [ctxp]
        L.ndt_last_error.restype = C.c_char_p
        L.ndt_set_map.argtypes = [ctxp, C.c_void_p, C.c_int]
        L.ndt_set_map_device.argtypes = [ctxp, C.c_void_p, C.c_int]
        L.ndt_map_append.argtypes = [ctxp, C.c_void_p, C.c_int]
        L.ndt_map_append_device.argtypes = [ctxp, C.c_void_p, C.c_int]
        L.ndt_align.argtypes = [ctxp, _f32p, C.c_int, _f32p, _f32p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.ndt_align_with_map.argtypes = [ctxp, _f32p, C.c_int, _f32p, _f32p, C.c_int, _f32p, C.POINTER(C.c_int),
                                         C.POINTER(C.c_double)]
        L.ndt_align_batch.argtypes = [ctxp, C.c_int, C.c_void_p, _i32p, _f32p, _f32p, _i32p, _f64p, C.c_void_p]
        L.ndt_align_batch_device.argtypes = [ctxp, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ndt_align_batch_packed.argtypes = [ctxp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p]
        L.ndt_align_batch_packed_with_map.argtypes = [ctxp, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ndt_set_profiling.argtypes = [ctxp, C.c_int]
        L.ndt_set_batch_graphs.argtypes = [ctxp, C.c_int]
        L.ndt_score_batch_device.argtypes = [ctxp, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                             C.c_void_p]
        L.ndt_kernel_variants.argtypes = []
        L.ndt_kernel_variant_shape.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ndt_set_kernel_variant.argtypes = [ctxp, C.c_int]
        L.ndt_set_side_queue_capacity.argtypes = [ctxp, C.c_int]
        L.ndt_get_kernel_variant.argtypes = [ctxp]
        L.ndt_set_chunk_tiles.argtypes = [ctxp, C.c_int]
        L.ndt_get_chunk_tiles.argtypes = [ctxp]
        L.ndt_autotune_batch_device.argtypes = [ctxp, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                                C.POINTER(C.c_int), _f32p]
        L.ndt_synchronize.argtypes = [ctxp]
        L.ndt_stream.argtypes = [ctxp]
        L.ndt_stream.restype = C.c_void_p
        L.ndt_get_counters.argtypes = [ctxp, C.POINTER(Counters)]
        L.ndt_grid_info.argtypes = [ctxp, _f32p, _i32p, C.POINTER(C.c_int)]
        L.ndt_grid_cells.argtypes = [ctxp, C.c_int, _i32p, _i32p, _f64p, _f64p]
        L.ndt_window_info.argtypes = [ctxp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.ndt_derivatives.argtypes = [ctxp, _f32p, _f32p, C.c_int, _f64p, C.POINTER(C.c_double), _f64p, _f64p]
        for name in ("ndt_create", "ndt_set_map", "ndt_set_map_device", "ndt_map_append", "ndt_map_append_device",
                     "ndt_align", "ndt_align_with_map",
                     "ndt_align_batch", "ndt_align_batch_device", "ndt_synchronize", "ndt_get_counters",
                     "ndt_grid_info", "ndt_grid_cells", "ndt_derivatives", "ndt_align_batch_packed",
                     "ndt_align_batch_packed_with_map",
                     "ndt_set_profiling", "ndt_kernel_variants", "ndt_kernel_variant_shape",
                     "ndt_set_kernel_variant", "ndt_window_info", "ndt_set_batch_graphs",
                     "ndt_set_side_queue_capacity", "ndt_get_kernel_variant", "ndt_autotune_batch_device",
                     "ndt_score_batch_device", "ndt_set_chunk_tiles", "ndt_get_chunk_tiles"):
            getattr(L, name).restype = C.c_int
        _LIB = L
    return _LIB


def kernel_variants():
    """[(tile, blocks_per_sm), ...] of the FP32 derivative-pass launch shapes."""
    L = lib()
    out = []
    for v in range(L.ndt_kernel_variants()):
        t, b = C.c_int(), C.c_int()
        L.ndt_kernel_variant_shape(v, C.byref(t), C.byref(b))
        out.append((t.value, b.value))
    return out


def reference_params(resolution=1.0, precision=0, dense_probe=0):
    p = Params()
    lib().ndt_params_reference(C.byref(p))
    p.resolution = resolution
    p.precision = precision
    p.dense_probe = dense_probe
    return p


def corrected_params(resolution=1.0, precision=0, dense_probe=0):
    p = Params()
    lib().ndt_params_corrected(C.byref(p))
    p.resolution = resolution
    p.precision = precision
    p.dense_probe = dense_probe
    return p


def _f32(a, cols=4):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a.reshape(-1, cols) if cols else a


class Context:
    """One ndt_ctx: a device, a stream, a map grid and batch buffers."""

    def __init__(self, params: Params | None = None, device: int = 0):
        self.L = lib()
        self.params = params if params is not None else reference_params()
        h = C.c_void_p()
        rc = self.L.ndt_create(C.byref(self.params), device, C.byref(h))
        if rc != NDT_OK:
            raise NdtError(f"ndt_create failed: {ERRORS.get(rc, rc)}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.ndt_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc < 0:
            msg = self.L.ndt_last_error(self.h)
            raise NdtError(f"{what}: {ERRORS.get(rc, rc)}: {msg.decode() if msg else ''}")
        return rc

    @property
    def stream(self):
        return self.L.ndt_stream(self.h)

    def set_map(self, cloud):
        cloud = _f32(cloud)
        self._check(self.L.ndt_set_map(self.h, cloud.ctypes.data, cloud.shape[0]), "ndt_set_map")

    def set_map_device(self, ptr: int, m: int):
        self._check(self.L.ndt_set_map_device(self.h, C.c_void_p(ptr), m), "ndt_set_map_device")

    def map_append(self, points):
        """Grows the map by `points` (host array); the grid then equals set_map of the grown map."""
        points = _f32(points)
        self._check(self.L.ndt_map_append(self.h, points.ctypes.data if len(points) else None, points.shape[0]),
                    "ndt_map_append")

    def map_append_device(self, ptr: int, k: int):
        """Same, with the points on the device (raw pointer)."""
        self._check(self.L.ndt_map_append_device(self.h, C.c_void_p(ptr), k), "ndt_map_append_device")

    def align(self, scan, guess):
        scan = _f32(scan)
        out = np.zeros(16, np.float32)
        conv, fit = C.c_int(), C.c_double()
        self._check(self.L.ndt_align(self.h, scan, scan.shape[0], _f32(guess, 0).reshape(16), out, C.byref(conv),
                                     C.byref(fit)), "ndt_align")
        return out, conv.value, fit.value

    def align_with_map(self, scan, guess, cloud):
        scan, cloud = _f32(scan), _f32(cloud)
        out = np.zeros(16, np.float32)
        conv, fit = C.c_int(), C.c_double()
        self._check(self.L.ndt_align_with_map(self.h, scan, scan.shape[0], _f32(guess, 0).reshape(16), cloud,
                                              cloud.shape[0], out, C.byref(conv), C.byref(fit)),
                    "ndt_align_with_map")
        return out, conv.value, fit.value

    def align_batch(self, scans, guesses):
        scans = [_f32(s) for s in scans]
        B = len(scans)
        ptrs = (C.c_void_p * B)(*[s.ctypes.data for s in scans])
        ns = np.array([s.shape[0] for s in scans], np.int32)
        g = np.ascontiguousarray(np.asarray(guesses, np.float32).reshape(B, 16))
        out = np.zeros((B, 16), np.float32)
        conv = np.zeros(B, np.int32)
        fit = np.zeros(B, np.float64)
        status = np.zeros(B, np.int32)
        self._check(self.L.ndt_align_batch(self.h, B, ptrs, ns, g, out, conv, fit, status.ctypes.data),
                    "ndt_align_batch")
        return out, conv, fit, status

    def align_batch_device(self, B, d_points, d_offsets, total, d_guesses, d_out, d_conv, d_fit, d_status=0):
        """Device pointers (ints, e.g. torch tensor .data_ptr()); enqueued on self.stream."""
        self._check(self.L.ndt_align_batch_device(self.h, B, C.c_void_p(d_points), C.c_void_p(d_offsets), total,
                                                  C.c_void_p(d_guesses), C.c_void_p(d_out), C.c_void_p(d_conv),
                                                  C.c_void_p(d_fit), C.c_void_p(d_status)), "ndt_align_batch_device")

    def align_batch_packed(self, points, offsets, guesses, out, conv, fit, status=None):
        """One packed host batch; all arguments are host numpy arrays (pinned or not)."""
        B = len(offsets) - 1
        self._check(self.L.ndt_align_batch_packed(self.h, B, points.ctypes.data, offsets.ctypes.data,
                                                  guesses.ctypes.data, out.ctypes.data, conv.ctypes.data,
                                                  fit.ctypes.data, status.ctypes.data if status is not None else None),
                    "ndt_align_batch_packed")

    def align_batch_packed_ptr(self, B, points, offsets, guesses, out, conv, fit, status=0):
        """Same, with raw host pointers (ints), e.g. pinned torch tensors."""
        self._check(self.L.ndt_align_batch_packed(self.h, B, C.c_void_p(points), C.c_void_p(offsets),
                                                  C.c_void_p(guesses), C.c_void_p(out), C.c_void_p(conv),
                                                  C.c_void_p(fit), C.c_void_p(status) if status else None),
                    "ndt_align_batch_packed")

    def align_batch_packed_with_map_ptr(self, map_ptr, m, B, points, offsets, guesses, out, conv, fit, status=0):
        """The batch with its map (raw host pointers, e.g. pinned torch tensors); the map's grid stays set."""
        self._check(self.L.ndt_align_batch_packed_with_map(self.h, C.c_void_p(map_ptr), m, B, C.c_void_p(points),
                                                           C.c_void_p(offsets), C.c_void_p(guesses),
                                                           C.c_void_p(out), C.c_void_p(conv), C.c_void_p(fit),
                                                           C.c_void_p(status) if status else None),
                    "ndt_align_batch_packed_with_map")

    def set_map_ptr(self, ptr: int, m: int):
        """Host map by raw pointer (e.g. a pinned torch tensor)."""
        self._check(self.L.ndt_set_map(self.h, C.c_void_p(ptr), m), "ndt_set_map")

    def score_batch_device(self, B, d_points, d_offsets, total, d_poses, d_score):
        """NDT score of B scans at B poses (device pointers), into d_score (B doubles)."""
        self._check(self.L.ndt_score_batch_device(self.h, B, C.c_void_p(d_points), C.c_void_p(d_offsets), total,
                                                  C.c_void_p(d_poses), C.c_void_p(d_score)),
                    "ndt_score_batch_device")

    def set_batch_graphs(self, on=True):
        self._check(self.L.ndt_set_batch_graphs(self.h, int(on)), "ndt_set_batch_graphs")

    def set_profiling(self, on=True):
        self._check(self.L.ndt_set_profiling(self.h, int(on)), "ndt_set_profiling")

    def set_kernel_variant(self, v):
        self._check(self.L.ndt_set_kernel_variant(self.h, int(v)), "ndt_set_kernel_variant")

    def set_side_queue_capacity(self, pairs=0):
        """FP64 side-queue capacity in pairs per derivative pass (0 = default 2^20)."""
        self._check(self.L.ndt_set_side_queue_capacity(self.h, int(pairs)), "set_side_queue_capacity")

    def kernel_variant(self):
        return self._check(self.L.ndt_get_kernel_variant(self.h), "ndt_get_kernel_variant")

    def set_chunk_tiles(self, tiles):
        """Tiles per large chunk of the FP32 derivative pass (1..64; default 8)."""
        self._check(self.L.ndt_set_chunk_tiles(self.h, int(tiles)), "ndt_set_chunk_tiles")

    def chunk_tiles(self):
        return self._check(self.L.ndt_get_chunk_tiles(self.h), "ndt_get_chunk_tiles")

    def autotune_device(self, B, d_points, d_offsets, total, d_guesses, repeats=2):
        """ndt_autotune_batch_device: times the batch with every launch shape, selects the fastest, then
        the chunk size (chunk_tiles()); returns (best, ms per variant)."""
        best = C.c_int()
        ms = np.zeros(self.L.ndt_kernel_variants(), np.float32)
        self._check(self.L.ndt_autotune_batch_device(self.h, B, C.c_void_p(d_points), C.c_void_p(d_offsets), total,
                                                     C.c_void_p(d_guesses), repeats, C.byref(best), ms),
                    "ndt_autotune_batch_device")
        return best.value, ms

    def synchronize(self):
        self._check(self.L.ndt_synchronize(self.h), "ndt_synchronize")

    def counters(self):
        k = Counters()
        self._check(self.L.ndt_get_counters(self.h, C.byref(k)), "ndt_get_counters")
        return {f: getattr(k, f) for f, _ in Counters._fields_}

    def grid_info(self):
        bbox = np.zeros(6, np.float32)
        dims = np.zeros(3, np.int32)
        occ = C.c_int()
        self._check(self.L.ndt_grid_info(self.h, bbox, dims, C.byref(occ)), "ndt_grid_info")
        return bbox, dims, occ.value

    def window_info(self):
        """(windows, entries) of the probe-window table; (0, 0) when the dense index is probed."""
        w, e = C.c_longlong(), C.c_longlong()
        self._check(self.L.ndt_window_info(self.h, C.byref(w), C.byref(e)), "ndt_window_info")
        return w.value, e.value

    def grid_cells(self):
        _, _, K = self.grid_info()
        cell = np.zeros(max(K, 1), np.int32)
        count = np.zeros(max(K, 1), np.int32)
        mean = np.zeros((max(K, 1), 3), np.float64)
        icov = np.zeros((max(K, 1), 9), np.float64)
        self._check(self.L.ndt_grid_cells(self.h, max(K, 1), cell, count, mean, icov), "ndt_grid_cells")
        return cell[:K], count[:K], mean[:K], icov[:K]

    def derivatives(self, scan, trans, p6):
        scan, trans = _f32(scan), _f32(trans)
        score = C.c_double()
        g = np.zeros(6)
        H = np.zeros(36)
        self._check(self.L.ndt_derivatives(self.h, scan, trans, scan.shape[0], np.ascontiguousarray(p6, np.float64),
                                           C.byref(score), g, H), "ndt_derivatives")
        return score.value, g, H.reshape(6, 6)


class DatFile:
    """An ndt_input.dat opened on the fast path (include/ndt_b200.h ndt_dat_*):
    memory-mapped and indexed once; `case(i)` gives copies of a test case's
    arrays, `relation(i)` how its map relates to the previous case's
    (MAP_NEW / MAP_SAME / MAP_GROWN), `align(ctx, first, count)` runs the
    cases through the library in chunks that share a map."""

    MAP_NEW, MAP_SAME, MAP_GROWN = 0, 1, 2

    def __init__(self, path):
        self.L = lib()
        L = self.L
        if not getattr(L, "_dat_ready", False):
            p = C.c_void_p
            L.ndt_dat_open.argtypes = [C.c_char_p, C.POINTER(p)]
            L.ndt_dat_close.argtypes = [p]
            L.ndt_dat_close.restype = None
            L.ndt_dat_last_error.argtypes = [p]
            L.ndt_dat_last_error.restype = C.c_char_p
            L.ndt_dat_count.argtypes = [p]
            fp = C.POINTER(C.POINTER(C.c_float))
            L.ndt_dat_case.argtypes = [p, C.c_int, fp, fp, C.POINTER(C.c_int), fp, C.POINTER(C.c_int)]
            L.ndt_dat_map_relation.argtypes = [p, C.c_int]
            L.ndt_dat_align.argtypes = [p, p, C.c_int, C.c_int, p, p, p, p]
            for n in ("ndt_dat_open", "ndt_dat_count", "ndt_dat_case", "ndt_dat_map_relation", "ndt_dat_align"):
                getattr(L, n).restype = C.c_int
            L._dat_ready = True
        h = C.c_void_p()
        rc = L.ndt_dat_open(str(path).encode(), C.byref(h))
        self.h = h
        if rc != 0:
            msg = L.ndt_dat_last_error(h).decode() if h else ""
            self.close()
            raise NdtError(f"ndt_dat_open: {ERRORS.get(rc, rc)}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.L.ndt_dat_close(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return self.L.ndt_dat_count(self.h)

    def case(self, i):
        g, sc, mp = (C.POINTER(C.c_float)(), C.POINTER(C.c_float)(), C.POINTER(C.c_float)())
        n, m = C.c_int(), C.c_int()
        if self.L.ndt_dat_case(self.h, i, C.byref(g), C.byref(sc), C.byref(n), C.byref(mp), C.byref(m)) != 0:
            raise IndexError(i)
        arr = lambda ptr, k: np.ctypeslib.as_array(ptr, (k,)).copy() if k else np.zeros(0, np.float32)
        return arr(g, 16), arr(sc, 4 * n.value).reshape(-1, 4), arr(mp, 4 * m.value).reshape(-1, 4)

    def relation(self, i):
        return self.L.ndt_dat_map_relation(self.h, i)

    def align(self, ctx, first=0, count=None):
        count = len(self) - first if count is None else count
        out = np.zeros((max(count, 1), 16), np.float32)
        conv = np.zeros(max(count, 1), np.int32)
        fit = np.zeros(max(count, 1), np.float64)
        status = np.zeros(max(count, 1), np.int32)
        rc = self.L.ndt_dat_align(ctx.h, self.h, first, count, out.ctypes.data, conv.ctypes.data, fit.ctypes.data,
                                  status.ctypes.data)
        if rc != 0:
            raise NdtError(f"ndt_dat_align: {ERRORS.get(rc, rc)}: {self.L.ndt_dat_last_error(self.h).decode()}")
        return out[:count], conv[:count], fit[:count], status[:count]
