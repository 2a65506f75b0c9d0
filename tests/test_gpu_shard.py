"""The sharded path with the real align call: two `gloo` ranks (spawned
processes), each with its own context on cuda:0, split one batch by scan size
(shard.balance), align their shares with Context.align_batch and all-gather
the results (shard.align_sharded).  Every rank must hold the whole batch, bit
for bit equal to one process aligning it in one batch (an alignment's result
does not depend on the batch it is in).  The ranks' kernels never wait on one
another: the only exchange is the host-side gather."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _load_pkg():
    import importlib.util
    import pathlib
    import sys

    name = "daphne_benchmark_b200"
    if name in sys.modules:
        return sys.modules[name]
    root = pathlib.Path(__file__).resolve().parents[1] / "daphne-benchmark_b200"
    spec = importlib.util.spec_from_file_location(name, root / "__init__.py", submodule_search_locations=[str(root)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def _case(pkg):
    cfg = pkg.synth.small_config("shard", 30000, 50.0, 20, 3000, seed=81)
    scene = pkg.synth.make_scene(cfg)
    aligns = [pkg.synth.make_alignment(cfg, scene, i, n_points=500 + 400 * (i % 7)) for i in range(13)]
    return scene, [a.scan for a in aligns], np.stack([a.guess for a in aligns])


def _worker(rank, world, port, q):
    import torch.distributed as dist

    pkg = _load_pkg()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=120))
    scene, scans, guesses = _case(pkg)
    with pkg.ndt.Context(pkg.ndt.reference_params(), device=0) as ctx:
        ctx.set_map(scene.map)
        out, conv, fit, status = pkg.shard.align_sharded(ctx.align_batch, scans, guesses, rank, world)
    q.put((rank, out, conv, fit, status))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_align_two_ranks_equals_one_batch(pkg):
    scene, scans, guesses = _case(pkg)
    with pkg.ndt.Context(pkg.ndt.reference_params(), device=0) as ctx:
        ctx.set_map(scene.map)
        ref = ctx.align_batch(scans, guesses)
    ctxmp = mp.get_context("spawn")
    q = ctxmp.Queue()
    port = _free_port()
    procs = [ctxmp.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, out, conv, fit, status in res:
        assert np.array_equal(out.view(np.uint32), ref[0].view(np.uint32)), rank
        assert np.array_equal(conv, ref[1]) and np.array_equal(fit.view(np.uint64), ref[2].view(np.uint64))
        assert np.array_equal(status, ref[3])
