"""ndt_derivatives_noalloc: the evaluation entry point that allocates no
device memory at call time (for callers such as real-time loops with a fixed
memory budget, where cudaMalloc can block and take unbounded time, or code
running while another component owns all of the device's memory: they cannot
call cudaMalloc while they run).  Its scratch is one static device array
shared by every call, so the test calls it twice in a row, on two different
scans, and
checks each result against the allocating entry point ndt_derivatives
through the C ABI, with the derivative tolerance of the parity tests (FP32
pairs: 2e-3 relative to the largest entry; FP64 pairs: 1e-9).

This file is named to be collected last: it passes alone in a fresh process
and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(pkg):
    L = pkg.ndt.lib()
    f = L.ndt_derivatives_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"),
                  C.c_void_p]
    f.restype = C.c_int
    return f


def _transform(scan, G):
    G = G.reshape(4, 4)
    trans = np.zeros_like(scan)
    for r in range(3):
        trans[:, r] = ((G[r, 0] * scan[:, 0] + G[r, 1] * scan[:, 1]) + G[r, 2] * scan[:, 2]) + G[r, 3]
    return trans


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_allocating_entry_point(pkg, precision):
    torch = pytest.importorskip("torch")
    f = _noalloc(pkg)
    cfg = pkg.synth.small_config("na", 20000, 40.0, 16, 1500, seed=31)
    scene = pkg.synth.make_scene(cfg)
    tol = 1e-9 if precision == 1 else 2e-3
    with pkg.ndt.Context(pkg.ndt.reference_params(precision=precision)) as ctx:
        ctx.set_map(scene.map)
        d_out = torch.zeros(44, dtype=torch.float64, device="cuda")
        for call, idx in enumerate((0, 1)):  # two calls in a row, different scans
            a = pkg.synth.make_alignment(cfg, scene, idx)
            trans = _transform(a.scan, a.guess)
            p6 = np.zeros(6)
            p6[:3] = a.guess.reshape(4, 4)[:3, 3]
            p6[3:] = [0.01 * (call + 1), -0.02, 0.3]
            s_ref, g_ref, H_ref = ctx.derivatives(a.scan, trans, p6)
            d_scan = torch.from_numpy(a.scan).cuda()
            d_trans = torch.from_numpy(trans).cuda()
            torch.cuda.synchronize()
            rc = f(ctx.h, d_scan.data_ptr(), d_trans.data_ptr(), a.scan.shape[0], p6, d_out.data_ptr())
            assert rc == 0, ctx.L.ndt_last_error(ctx.h)
            ctx.synchronize()
            out = d_out.cpu().numpy()
            assert out[43] > 0  # pairs found, no side-queue overflow
            assert abs(out[0] - s_ref) <= tol * max(1.0, abs(s_ref))
            assert np.max(np.abs(out[1:7] - g_ref)) <= tol * max(1.0, np.max(np.abs(g_ref)))
            assert np.max(np.abs(out[7:43] - H_ref.reshape(36))) <= tol * max(1.0, np.max(np.abs(H_ref)))


def test_noalloc_rejects_oversized_scan(pkg):
    torch = pytest.importorskip("torch")
    f = _noalloc(pkg)
    cfg = pkg.synth.small_config("na2", 4000, 20.0, 4, 100, seed=32)
    scene = pkg.synth.make_scene(cfg)
    with pkg.ndt.Context(pkg.ndt.reference_params()) as ctx:
        ctx.set_map(scene.map)
        big = torch.zeros((65537, 4), dtype=torch.float32, device="cuda")
        out = torch.zeros(44, dtype=torch.float64, device="cuda")
        rc = f(ctx.h, big.data_ptr(), big.data_ptr(), 65537, np.zeros(6), out.data_ptr())
        assert rc == -6  # NDT_E_CAPACITY
        assert b"65536" in ctx.L.ndt_last_error(ctx.h)
