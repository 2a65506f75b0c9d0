"""The library's failure paths, made to fire without faulting or hanging the
GPU (the reference has none of these: it calls exit(-3) on I/O errors,
src/CPU/ndt_mapping/kernel.cpp:157-159, 211-214, and has no budgets).

* evaluation watchdog: a corrected-mode budget of 2 derivative evaluations
  per alignment; the round loop is bounded, so the alignments stop with
  NDT_ST_WATCHDOG (batch) or NDT_E_WATCHDOG (single call);
* FP64 side-queue overflow: a map that fits one voxel (dense grid size 1, so
  the reference's covariance is scaled by G - 1 = 0 and its inverse is NaN:
  every pair with it goes to the FP64 side queue), with a queue capacity
  below the pair count: NDT_ST_OVERFLOW; the no-allocation evaluation, whose
  queue holds 2048 pairs, reports the pair count -1;
* tensor-core wait: the point-network kernel's bounded mbarrier wait set to
  give up before its first poll; the kernel still waits (with the normal
  limit) for its MMAs before it frees its tensor memory, and the flag comes
  back through ndt_mlp_synchronize; the next call with the normal limit is
  correct again.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NDT_ST_WATCHDOG, NDT_ST_OVERFLOW = 1, 2


def _one_voxel_map_and_scans(seed=5, m=500, n=3000, B=2):
    rng = np.random.default_rng(seed)
    cloud = np.ones((m, 4), np.float32)
    cloud[:, :3] = rng.uniform(0.0, 0.5, (m, 3))
    scans = []
    for _ in range(B):
        s = np.ones((n, 4), np.float32)
        s[:, :3] = rng.uniform(0.0, 0.5, (n, 3))
        scans.append(s)
    return cloud, scans


def test_watchdog_stops_alignments(pkg):
    cfg = pkg.synth.small_config("wd", 20000, 40.0, 16, 1500, seed=41, dt=1.0, dyaw_deg=5.0)
    scene = pkg.synth.make_scene(cfg)
    aligns = [pkg.synth.make_alignment(cfg, scene, i) for i in range(6)]
    scans, guesses = [a.scan for a in aligns], [a.guess for a in aligns]
    prm = pkg.ndt.corrected_params()
    with pkg.ndt.Context(prm) as ctx:
        ctx.set_map(scene.map)
        _, _, _, st_free = ctx.align_batch(scans, guesses)
        ctx.set_profiling(True)
        ctx.align_batch(scans, guesses)
        evals = ctx.counters()["evaluations"]
    assert (st_free == 0).all()
    assert evals > 2 * len(aligns)  # the alignments need more than the budget below
    prm.watchdog_evals = 2
    with pkg.ndt.Context(prm) as ctx:
        ctx.set_map(scene.map)
        out, conv, _, st = ctx.align_batch(scans, guesses)
        assert (st & NDT_ST_WATCHDOG).all() and not (conv != 0).any()
        assert np.isfinite(out).all()
        with pytest.raises(pkg.ndt.NdtError, match="NDT_E_WATCHDOG"):
            ctx.align(scans[0], guesses[0])
        # the context stays usable
        prm_ok = pkg.ndt.corrected_params()
    with pkg.ndt.Context(prm_ok) as ctx:
        ctx.set_map(scene.map)
        _, _, _, st2 = ctx.align_batch(scans, guesses)
        assert (st2 == 0).all()


def test_side_queue_overflow(pkg, oracle, binding_mod):
    cloud, scans = _one_voxel_map_and_scans()
    guesses = [np.eye(4, dtype=np.float32).reshape(16)] * len(scans)
    prm = binding_mod.reference_params()
    ref = [oracle.align(prm, s, g, cloud) for s, g in zip(scans, guesses)]
    with pkg.ndt.Context(pkg.ndt.reference_params()) as ctx:
        ctx.set_map(cloud)
        out, conv, _, st = ctx.align_batch(scans, guesses)
        assert (st == 0).all()  # the default queue (2^20 pairs) holds them
        for i, (r, rc, _, _) in enumerate(ref):  # every pair on the FP64 side path, as the reference evaluates it
            assert np.array_equal(np.isnan(out[i]), np.isnan(r))
            fin = np.isfinite(r)
            assert np.max(np.abs(out[i][fin] - r[fin]), initial=0.0) <= 1e-6
            assert conv[i] == rc
        ctx.set_side_queue_capacity(1000)  # below the 3000 pairs of one scan
        _, _, _, st = ctx.align_batch(scans, guesses)
        assert (st & NDT_ST_OVERFLOW).all()
        with pytest.raises(pkg.ndt.NdtError, match="NDT_E_CAPACITY"):
            ctx.align(scans[0], guesses[0])
        ctx.set_side_queue_capacity(0)
        _, _, _, st = ctx.align_batch(scans, guesses)
        assert (st == 0).all()
        with pytest.raises(pkg.ndt.NdtError, match="NDT_E_ARG"):
            ctx.set_side_queue_capacity(-1)


def test_noalloc_side_queue_limit(pkg):
    torch = pytest.importorskip("torch")
    L = pkg.ndt.lib()
    f = L.ndt_derivatives_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                  np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"), C.c_void_p]
    f.restype = C.c_int
    cloud, scans = _one_voxel_map_and_scans(B=1)
    scan = scans[0]
    with pkg.ndt.Context(pkg.ndt.reference_params()) as ctx:
        ctx.set_map(cloud)
        s_ref, g_ref, _ = ctx.derivatives(scan, scan, np.zeros(6))  # 3000 side pairs: within 2^20
        assert s_ref == 0.0 and (g_ref == 0).all()  # the reference rejects every NaN pair (kernel.cpp:460-463)
        d_scan = torch.from_numpy(scan).cuda()
        d_out = torch.zeros(44, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = f(ctx.h, d_scan.data_ptr(), d_scan.data_ptr(), scan.shape[0], np.zeros(6), d_out.data_ptr())
        assert rc == 0, ctx.L.ndt_last_error(ctx.h)
        ctx.synchronize()
        assert d_out[43].item() == -1.0  # more than 2048 side pairs
        small = np.ascontiguousarray(scan[:500])
        d_small = torch.from_numpy(small).cuda()
        torch.cuda.synchronize()
        rc = f(ctx.h, d_small.data_ptr(), d_small.data_ptr(), small.shape[0], np.zeros(6), d_out.data_ptr())
        assert rc == 0
        ctx.synchronize()
        assert d_out[43].item() == 500.0 and d_out[0].item() == 0.0


def test_noalloc_rejects_misaligned_pointers(pkg):
    torch = pytest.importorskip("torch")
    L = pkg.ndt.lib()
    f = L.ndt_derivatives_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                  np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"), C.c_void_p]
    f.restype = C.c_int
    cloud, scans = _one_voxel_map_and_scans(B=1, n=100)
    with pkg.ndt.Context(pkg.ndt.reference_params()) as ctx:
        ctx.set_map(cloud)
        buf = torch.zeros((101, 4), dtype=torch.float32, device="cuda")
        out = torch.zeros(45, dtype=torch.float64, device="cuda")
        base, ob = buf.data_ptr(), out.data_ptr()
        for args in ((base + 4, base, ob), (base, base + 8, ob), (base, base, ob + 4)):
            rc = f(ctx.h, args[0], args[1], 100, np.zeros(6), args[2])
            assert rc == -1  # NDT_E_ARG, refused before any work
            assert b"aligned" in ctx.L.ndt_last_error(ctx.h)
        ctx.synchronize()


def test_tensor_core_wait_gives_up(pkg):
    torch = pytest.importorskip("torch")
    cfg = pkg.synth.small_config("tcw", 20000, 40.0, 16, 1500, seed=43)
    scene = pkg.synth.make_scene(cfg)
    aligns = [pkg.synth.make_alignment(cfg, scene, i) for i in range(4)]
    pts = torch.from_numpy(np.concatenate([a.scan for a in aligns])).cuda()
    offs = np.zeros(len(aligns) + 1, np.int32)
    offs[1:] = np.cumsum([len(a.scan) for a in aligns])
    d_offs = torch.from_numpy(offs).cuda()
    g = torch.from_numpy(np.stack([a.guess for a in aligns]).astype(np.float32)).cuda()
    y_ok = torch.zeros((len(aligns), 6), dtype=torch.float32, device="cuda")
    y2 = torch.zeros_like(y_ok)
    net = pkg.posenet.PoseNet(center=scene.map[:, :3].mean(0), scale=4.0)
    net.set_weights(np.random.default_rng(0).normal(0.0, 0.2, net.n_w).astype(np.float32))
    torch.cuda.synchronize()
    net.forward(len(aligns), pts.data_ptr(), d_offs.data_ptr(), g.data_ptr(), y_ok.data_ptr(), 512)
    assert not net.synchronize_status()
    net.set_wait_limit(0)  # give up before the first poll
    net.forward(len(aligns), pts.data_ptr(), d_offs.data_ptr(), g.data_ptr(), y2.data_ptr(), 512)
    assert net.synchronize_status()  # the give-up is reported ...
    assert not net.synchronize_status()  # ... once
    net.set_wait_limit(-1)
    net.forward(len(aligns), pts.data_ptr(), d_offs.data_ptr(), g.data_ptr(), y2.data_ptr(), 512)
    assert not net.synchronize_status()
    assert torch.equal(y_ok, y2) and bool(torch.any(y_ok != 0))  # the kernel and the context are fine afterwards
    net.close()
