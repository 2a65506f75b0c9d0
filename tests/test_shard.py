"""Multi-GPU sharding host logic, with world_size 2 gloo ranks on the CPU
(the GPU align call is replaced by a deterministic stand-in)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def test_balance_covers_every_alignment_once(pkg):
    ns = np.array([1000, 16000, 3000, 8000, 2000, 12000, 500, 7000])
    for world in (1, 2, 3, 8):
        parts = pkg.shard.balance(ns, world)
        allidx = np.sort(np.concatenate(parts))
        assert allidx.tolist() == list(range(len(ns)))
        loads = [ns[p].sum() for p in parts]
        assert max(loads) - min(loads) <= ns.max()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import importlib.util
    import pathlib
    import sys
    import torch.distributed as dist

    root = pathlib.Path(__file__).resolve().parents[1] / "daphne-benchmark_b200"
    spec = importlib.util.spec_from_file_location("shard", root / "shard.py")
    shard = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(shard)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    rng = np.random.default_rng(0)
    scans = [np.zeros((int(n), 4), np.float32) + i for i, n in enumerate(rng.integers(10, 100, 9))]
    guesses = np.arange(9 * 16, dtype=np.float32).reshape(9, 16)

    def fake_align(sc, g):
        # stands in for Context.align_batch: output encodes which alignment it was
        B = len(sc)
        out = np.asarray(g, np.float32).reshape(B, 16) * 2
        conv = np.ones(B, np.int32)
        fit = np.array([s[0, 0] for s in sc], np.float64)
        return out, conv, fit, np.zeros(B, np.int32) + rank

    out, conv, fit, status = shard.align_sharded(fake_align, scans, guesses, rank, world)
    q.put((rank, out, conv, fit, status))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_gather_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    guesses = np.arange(9 * 16, dtype=np.float32).reshape(9, 16)
    for rank, out, conv, fit, status in res:
        assert np.array_equal(out, guesses * 2)
        assert conv.tolist() == [1] * 9
        assert fit.tolist() == [float(i) for i in range(9)]
        assert set(status.tolist()) == {0, 1}  # both ranks aligned part of the batch
