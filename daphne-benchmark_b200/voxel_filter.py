"""Scan pre-filter: Python side of the batched voxel-grid downsampling
(csrc/voxel_filter.cu, include/ndt_b200.h `ndt_filter_*`,
`ndt_voxel_filter_device`).

`VoxelFilter.filter_device` takes device pointers (e.g. torch CUDA tensors'
data_ptr()); `VoxelFilter.filter` takes a packed host batch and returns host
arrays, using torch for the device buffers.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ndt as _ndt


def _lib():
    L = _ndt.lib()
    if not getattr(L, "_vf_ready", False):
        p = C.c_void_p
        L.ndt_filter_create.argtypes = [C.c_int, C.POINTER(p)]
        L.ndt_filter_create.restype = C.c_int
        L.ndt_filter_destroy.argtypes = [p]
        L.ndt_filter_destroy.restype = None
        L.ndt_filter_last_error.argtypes = [p]
        L.ndt_filter_last_error.restype = C.c_char_p
        L.ndt_filter_stream.argtypes = [p]
        L.ndt_filter_stream.restype = p
        L.ndt_voxel_filter_device.argtypes = [p, C.c_int, p, p, C.c_int, C.c_float, p, p, C.POINTER(C.c_int)]
        L.ndt_voxel_filter_device.restype = C.c_int
        L._vf_ready = True
    return L


class VoxelFilter:
    """A filter handle: its device scratch and stream on one GPU."""

    def __init__(self, device=0):
        self.L = _lib()
        h = C.c_void_p()
        rc = self.L.ndt_filter_create(device, C.byref(h))
        if rc != 0:
            raise _ndt.NdtError(f"ndt_filter_create failed ({_ndt.ERRORS.get(rc, rc)})")
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.L.ndt_filter_destroy(self.h)
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

    @property
    def stream(self):
        return self.L.ndt_filter_stream(self.h)

    def filter_device(self, B, d_points, d_offsets, total_points, leaf, d_out, d_out_offsets):
        """Filters B packed device scans into d_out / d_out_offsets; returns the output point count."""
        n = C.c_int()
        rc = self.L.ndt_voxel_filter_device(self.h, B, C.c_void_p(d_points), C.c_void_p(d_offsets), total_points,
                                            float(leaf), C.c_void_p(d_out), C.c_void_p(d_out_offsets), C.byref(n))
        if rc != 0:
            raise _ndt.NdtError(f"ndt_voxel_filter_device: {_ndt.ERRORS.get(rc, rc)}: "
                                f"{self.L.ndt_filter_last_error(self.h).decode()}")
        return n.value

    def filter(self, points, offsets, leaf):
        """Host batch (points: total x 4 float32, offsets: B + 1) -> (out points, out offsets)."""
        import torch

        points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        offsets = np.ascontiguousarray(offsets, np.int32)
        B, total = len(offsets) - 1, len(points)
        dev = torch.device("cuda", self.device)
        d_pts = torch.from_numpy(points).to(dev) if total else torch.zeros((1, 4), device=dev)
        d_off = torch.from_numpy(offsets).to(dev)
        d_out = torch.empty((max(total, 1), 4), dtype=torch.float32, device=dev)
        d_oo = torch.empty(B + 1, dtype=torch.int32, device=dev)
        torch.cuda.current_stream(dev).synchronize()
        k = self.filter_device(B, d_pts.data_ptr(), d_off.data_ptr(), total, leaf, d_out.data_ptr(),
                               d_oo.data_ptr())
        return d_out[:k].cpu().numpy(), d_oo.cpu().numpy()
