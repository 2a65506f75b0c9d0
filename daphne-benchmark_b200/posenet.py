"""Learned initial pose: Python side of the point-feature network
(csrc/posenet.cu, include/ndt_b200.h `ndt_mlp_*`).

`PoseNet` owns the network's device weights and its stream; the forward and
training calls take device pointers (torch CUDA tensors here).  The pose
helpers convert between 4x4 transforms and the pose vector of the corrected
NDT parametrisation T = Trans(x, y, z) Rx(roll) Ry(pitch) Rz(yaw), in which
the network's correction is expressed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ndt as _ndt

H1, H2, H3, OUT = 64, 128, 64, 6
DELTA_SCALE = np.array([1.0, 1.0, 0.1, 0.02, 0.02, 0.1], np.float32)  # m, m, m, rad, rad, rad
MAX_LEVELS = 8  # NDT_LEARNED_MAX_LEVELS
# FP32 weight blob layout (ndt_mlp_num_weights values): W1[64][3], b1, W2[128][64], b2, W3[64][128], b3, W4[6][64], b4
_OFF = np.cumsum([0, H1 * 3, H1, H2 * H1, H2, H3 * H2, H3, OUT * H3, OUT])


def init_weights(seed=0):
    """He-style initialisation: normal weights with variance 2 / fan-in (the output layer scaled by 0.1 of
    1 / fan-in, so the first proposals stay near the guess), zero biases."""
    rng = np.random.default_rng(seed)
    w = np.zeros(int(_OFF[-1]), np.float32)
    w[_OFF[0]:_OFF[1]] = rng.normal(0, np.sqrt(2.0 / 3), H1 * 3)
    w[_OFF[2]:_OFF[3]] = rng.normal(0, np.sqrt(2.0 / H1), H2 * H1)
    w[_OFF[4]:_OFF[5]] = rng.normal(0, np.sqrt(2.0 / H2), H3 * H2)
    w[_OFF[6]:_OFF[7]] = rng.normal(0, np.sqrt(1.0 / H3) * 0.1, OUT * H3)
    return w


class LearnedParams(C.Structure):
    """ndt_learned_params (include/ndt_b200.h): the learned-init pipeline's set-up."""
    _fields_ = [("max_points", C.c_int32), ("passes", C.c_int32), ("grid_xy", C.c_int32), ("grid_yaw", C.c_int32),
                ("step_xy", C.c_float), ("step_yaw_deg", C.c_float), ("judge_level", C.c_int32),
                ("judge_points", C.c_int32), ("level_points", C.c_int32 * MAX_LEVELS)]


def learned_params(**kw):
    """The library's defaults (ndt_learned_params_default), overridden by keyword."""
    p = LearnedParams()
    _lib().ndt_learned_params_default(C.byref(p))
    for k, v in kw.items():
        if k == "level_points":
            for i, n in enumerate(v):
                p.level_points[i] = int(n)
        else:
            setattr(p, k, v)
    return p


def _lib():
    L = _ndt.lib()
    if not getattr(L, "_pn_ready", False):
        p = C.c_void_p
        L.ndt_mlp_num_weights.restype = C.c_int
        L.ndt_mlp_create.argtypes = [C.c_int, C.POINTER(p)]
        L.ndt_mlp_destroy.argtypes = [p]
        L.ndt_mlp_destroy.restype = None
        L.ndt_mlp_last_error.argtypes = [p]
        L.ndt_mlp_last_error.restype = C.c_char_p
        L.ndt_mlp_set_input_frame.argtypes = [p, C.POINTER(C.c_float), C.c_float, C.POINTER(C.c_float)]
        L.ndt_mlp_set_weights.argtypes = [p, C.POINTER(C.c_float), C.c_int]
        L.ndt_mlp_get_weights.argtypes = [p, C.POINTER(C.c_float), C.c_int]
        L.ndt_mlp_forward_device.argtypes = [p, C.c_int, p, p, p, C.c_int, p]
        L.ndt_mlp_train_step_device.argtypes = [p, C.c_int, p, p, p, p, C.c_int, C.c_float, C.c_int,
                                                C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.ndt_mlp_maxpool_device.argtypes = [p, p, C.c_int]
        L.ndt_mlp_synchronize.argtypes = [p, C.POINTER(C.c_int)]
        L.ndt_mlp_set_wait_limit.argtypes = [p, C.c_int]
        L.ndt_mlp_stream.argtypes = [p]
        L.ndt_mlp_stream.restype = p
        L.ndt_mlp_set_stream.argtypes = [p, p]
        L.ndt_mlp_propose_device.argtypes = [p, C.c_int, p, p, p, C.c_int, C.c_int, p, p]
        L.ndt_mlp_judge_device.argtypes = [p, C.c_int, p, p, p, p, p, p]
        L.ndt_learned_params_default.argtypes = [C.POINTER(LearnedParams)]
        L.ndt_learned_params_default.restype = None
        L.ndt_align_batch_learned_device.argtypes = [p, C.POINTER(C.c_void_p), C.c_int, C.POINTER(LearnedParams),
                                                     C.c_int, p, p, C.c_int, p, p, p, p, p, p, p]
        L.ndt_align_batch_learned_device.restype = C.c_int
        L.ndt_align_batch_learned.argtypes = [p, C.POINTER(C.c_void_p), C.c_int, C.POINTER(LearnedParams),
                                              C.c_int, p, p, p, p, p, p, p, p, p]
        L.ndt_align_batch_learned.restype = C.c_int
        for n in ("ndt_mlp_create", "ndt_mlp_set_input_frame", "ndt_mlp_set_weights", "ndt_mlp_get_weights",
                  "ndt_mlp_forward_device", "ndt_mlp_train_step_device", "ndt_mlp_maxpool_device",
                  "ndt_mlp_synchronize", "ndt_mlp_set_wait_limit", "ndt_mlp_set_stream", "ndt_mlp_propose_device", "ndt_mlp_judge_device"):
            getattr(L, n).restype = C.c_int
        L._pn_ready = True
    return L


def num_weights():
    return _lib().ndt_mlp_num_weights()


def _f32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class PoseNet:
    """Device weights, Adam state and stream of one network."""

    def __init__(self, device=0, center=(0.0, 0.0, 0.0), scale=1.0, delta_scale=DELTA_SCALE):
        self.L = _lib()
        h = C.c_void_p()
        rc = self.L.ndt_mlp_create(device, C.byref(h))
        if rc != 0:
            raise _ndt.NdtError(f"ndt_mlp_create failed ({rc})")
        self.h = h
        self.n_w = self.L.ndt_mlp_num_weights()
        self.delta_scale = np.asarray(delta_scale, np.float32)
        self.set_input_frame(center, scale, self.delta_scale)

    def _check(self, rc, what):
        if rc != 0:
            raise _ndt.NdtError(f"{what}: {self.L.ndt_mlp_last_error(self.h).decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.L.ndt_mlp_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def set_input_frame(self, center, scale, delta_scale):
        c = np.ascontiguousarray(center, np.float32)
        d = np.ascontiguousarray(delta_scale, np.float32)
        self.center, self.scale = c, float(scale)
        self._check(self.L.ndt_mlp_set_input_frame(self.h, _f32p(c), float(scale), _f32p(d)), "set_input_frame")

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == self.n_w
        self._check(self.L.ndt_mlp_set_weights(self.h, _f32p(w), self.n_w), "set_weights")

    def get_weights(self):
        w = np.zeros(self.n_w, np.float32)
        self._check(self.L.ndt_mlp_get_weights(self.h, _f32p(w), self.n_w), "get_weights")
        return w

    def forward(self, B, d_points, d_offsets, d_guesses, d_y, max_points=1024):
        self._check(self.L.ndt_mlp_forward_device(self.h, B, C.c_void_p(d_points), C.c_void_p(d_offsets),
                                                  C.c_void_p(d_guesses), max_points, C.c_void_p(d_y)), "forward")

    def train_step(self, B, d_points, d_offsets, d_guesses, d_target, lr=1e-3, update=True, max_points=1024,
                   want_grad=False):
        loss = np.zeros(1, np.float32)
        grad = np.zeros(self.n_w, np.float32) if want_grad else None
        self._check(self.L.ndt_mlp_train_step_device(self.h, B, C.c_void_p(d_points), C.c_void_p(d_offsets),
                                                     C.c_void_p(d_guesses), C.c_void_p(d_target), max_points,
                                                     float(lr), int(update), _f32p(loss),
                                                     _f32p(grad) if grad is not None else None), "train_step")
        return float(loss[0]), grad

    def maxpool(self, d_out, B):
        self._check(self.L.ndt_mlp_maxpool_device(self.h, C.c_void_p(d_out), B), "maxpool")

    def set_wait_limit(self, polls=-1):
        """Polls of the tensor-core barrier before a wait gives up (-1 = default; 0 exercises the error path)."""
        self._check(self.L.ndt_mlp_set_wait_limit(self.h, int(polls)), "set_wait_limit")

    def synchronize_status(self):
        """Waits for the network's stream; True when a tensor-core wait gave up since the last check."""
        e = C.c_int()
        self._check(self.L.ndt_mlp_synchronize(self.h, C.byref(e)), "synchronize")
        return bool(e.value)

    def synchronize(self):
        e = C.c_int()
        self._check(self.L.ndt_mlp_synchronize(self.h, C.byref(e)), "synchronize")
        if e.value:
            raise _ndt.NdtError("tensor-core wait gave up (mbarrier wait limit)")

    def set_stream(self, stream):
        """Run on a caller's stream (an int handle, e.g. Context.stream), or its own (None)."""
        self._check(self.L.ndt_mlp_set_stream(self.h, C.c_void_p(stream) if stream else None), "set_stream")

    def propose_device(self, B, d_points, d_offsets, d_guesses, d_y, d_prop, passes=3, max_points=1024):
        self._check(self.L.ndt_mlp_propose_device(self.h, B, C.c_void_p(d_points), C.c_void_p(d_offsets),
                                                  C.c_void_p(d_guesses), max_points, passes, C.c_void_p(d_y),
                                                  C.c_void_p(d_prop)), "propose")

    def align_learned_device(self, levels, lp, B, d_points, d_offsets, total, d_guesses, d_out, d_conv, d_fit,
                             d_status=0, d_choice=0, d_start=0):
        """ndt_align_batch_learned_device: proposals from lp's starts, the NDT judge, refinement through
        `levels` (ndt.Context objects, coarse to fine).  Device pointers as ints; enqueued, ready after
        levels[-1].synchronize()."""
        arr = (C.c_void_p * len(levels))(*[c.h.value if isinstance(c.h, C.c_void_p) else c.h for c in levels])
        rc = self.L.ndt_align_batch_learned_device(self.h, arr, len(levels), C.byref(lp), B, C.c_void_p(d_points),
                                                   C.c_void_p(d_offsets), int(total), C.c_void_p(d_guesses),
                                                   C.c_void_p(d_out), C.c_void_p(d_conv), C.c_void_p(d_fit),
                                                   C.c_void_p(d_status or None), C.c_void_p(d_choice or None),
                                                   C.c_void_p(d_start or None))
        if rc != 0:
            raise _ndt.NdtError(f"ndt_align_batch_learned_device ({_ndt.ERRORS.get(rc, rc)}): "
                                f"{self.L.ndt_mlp_last_error(self.h).decode()}")

    def align_learned(self, levels, lp, B, points, offsets, guesses, out, conv, fit, status=0, choice=0, start=0):
        """ndt_align_batch_learned: the same with host buffers (addresses as ints, e.g. of pinned tensors);
        returns when the results are on the host."""
        arr = (C.c_void_p * len(levels))(*[c.h.value if isinstance(c.h, C.c_void_p) else c.h for c in levels])
        rc = self.L.ndt_align_batch_learned(self.h, arr, len(levels), C.byref(lp), B, C.c_void_p(points),
                                            C.c_void_p(offsets), C.c_void_p(guesses), C.c_void_p(out),
                                            C.c_void_p(conv), C.c_void_p(fit), C.c_void_p(status or None),
                                            C.c_void_p(choice or None), C.c_void_p(start or None))
        if rc != 0:
            raise _ndt.NdtError(f"ndt_align_batch_learned ({_ndt.ERRORS.get(rc, rc)}): "
                                f"{self.L.ndt_mlp_last_error(self.h).decode()}")

    def judge_device(self, B, d_prop, d_guesses, d_s_prop, d_s_guess, d_start, d_used=0):
        self._check(self.L.ndt_mlp_judge_device(self.h, B, C.c_void_p(d_prop), C.c_void_p(d_guesses),
                                                C.c_void_p(d_s_prop), C.c_void_p(d_s_guess), C.c_void_p(d_start),
                                                C.c_void_p(d_used) if d_used else None), "judge")

    @property
    def stream(self):
        return self.L.ndt_mlp_stream(self.h)


# ---------------------------------------------------------------------------
# Pose vectors of the corrected parametrisation T = Trans Rx(a) Ry(b) Rz(c).
def pose_from_matrix(T):
    T = np.asarray(T, np.float64).reshape(4, 4)
    R = T[:3, :3]
    b = np.arcsin(np.clip(R[0, 2], -1.0, 1.0))
    a = np.arctan2(-R[1, 2], R[2, 2])
    c = np.arctan2(-R[0, 1], R[0, 0])
    return np.array([T[0, 3], T[1, 3], T[2, 3], a, b, c])


def matrix_from_pose(p):
    x, y, z, a, b, c = [float(v) for v in p]
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    Rx = np.array([[1, 0, 0], [0, ca, -sa], [0, sa, ca]])
    Ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    Rz = np.array([[cc, -sc, 0], [sc, cc, 0], [0, 0, 1]])
    T = np.eye(4)
    T[:3, :3] = Rx @ Ry @ Rz
    T[:3, 3] = [x, y, z]
    return T


def wrap_angle(a):
    return (np.asarray(a) + np.pi) % (2 * np.pi) - np.pi


def correction_target(guess16, converged16, delta_scale=DELTA_SCALE):
    """Normalised pose correction from a guess to a converged pose."""
    d = pose_from_matrix(converged16) - pose_from_matrix(guess16)
    d[3:] = wrap_angle(d[3:])
    return (d / delta_scale).astype(np.float32)


def apply_correction(guess16, y, delta_scale=DELTA_SCALE):
    """The proposed 4x4 (float32, row major) from a guess and a network output."""
    p = pose_from_matrix(guess16) + np.asarray(y, np.float64) * delta_scale
    return matrix_from_pose(p).astype(np.float32).reshape(16)


def poses_from_matrices(T):
    """Vectorised pose_from_matrix: (B, 16) or (B, 4, 4) -> (B, 6)."""
    T = np.asarray(T, np.float64).reshape(-1, 4, 4)
    b = np.arcsin(np.clip(T[:, 0, 2], -1.0, 1.0))
    a = np.arctan2(-T[:, 1, 2], T[:, 2, 2])
    c = np.arctan2(-T[:, 0, 1], T[:, 0, 0])
    return np.stack([T[:, 0, 3], T[:, 1, 3], T[:, 2, 3], a, b, c], 1)


def matrices_from_poses(p):
    """Vectorised matrix_from_pose: (B, 6) -> (B, 16) float32."""
    p = np.asarray(p, np.float64)
    a, b, c = p[:, 3], p[:, 4], p[:, 5]
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    T = np.zeros((len(p), 4, 4))
    # Rx(a) Ry(b) Rz(c)
    T[:, 0, 0] = cb * cc
    T[:, 0, 1] = -cb * sc
    T[:, 0, 2] = sb
    T[:, 1, 0] = ca * sc + sa * sb * cc
    T[:, 1, 1] = ca * cc - sa * sb * sc
    T[:, 1, 2] = -sa * cb
    T[:, 2, 0] = sa * sc - ca * sb * cc
    T[:, 2, 1] = sa * cc + ca * sb * sc
    T[:, 2, 2] = ca * cb
    T[:, :3, 3] = p[:, :3]
    T[:, 3, 3] = 1.0
    return T.astype(np.float32).reshape(-1, 16)


def correction_targets(guesses16, converged16, delta_scale=DELTA_SCALE):
    d = poses_from_matrices(converged16) - poses_from_matrices(guesses16)
    d[:, 3:] = wrap_angle(d[:, 3:])
    return (d / delta_scale).astype(np.float32)


def apply_corrections(guesses16, y, delta_scale=DELTA_SCALE):
    return matrices_from_poses(poses_from_matrices(guesses16) + np.asarray(y, np.float64) * delta_scale)
