"""Sharding of independent systems across ranks: the plan, and a
world-size-2 run over gloo on CPU (each rank solves its share with the CPU
oracle; rank 0 gathers and compares with the one-process result)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from ssf_b200 import decks, shard


def test_partition_is_deterministic_and_complete():
    w = np.random.default_rng(0).uniform(1, 100, 513)
    for world in (1, 2, 3, 8):
        p1 = shard.partition(w, world)
        p2 = shard.partition(w, world)
        assert p1 == p2
        flat = sorted(i for part in p1 for i in part)
        assert flat == list(range(513))
        assert shard.imbalance(w, p1) < 1.05


def test_partition_plate_batch_balances():
    plates = decks.plate_batch(64, seed=0)
    w = [shard.plate_weight(p) for p in plates]
    parts = shard.partition(w, 4)
    assert shard.imbalance(w, parts) < 1.1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, queue):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        plates = decks.plate_batch(6, seed=5, lo=3, hi=9)
        for p in plates:
            p.loads *= 1e6
        parts = shard.partition([shard.plate_weight(p) for p in plates], world)
        mine = {}
        for k in parts[rank]:
            adr, ci, a = O.assemble(plates[k], sym=True)
            x, st, ani, _ = O.scr_cg_prec(adr, ci, a, O.load_vector(plates[k]), ni=20000, res=1e-20)
            mine[k] = (st, ani, x)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            queue.put(sorted((k, v[0], v[1], float(np.linalg.norm(v[2]))) for k, v in merged.items()))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharded_batch(oracle):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every plate solved exactly once, same as one process
    plates = decks.plate_batch(6, seed=5, lo=3, hi=9)
    assert [r[0] for r in res] == list(range(len(plates)))
    for (k, st, ani, nrm), p in zip(res, plates):
        p.loads *= 1e6
        adr, ci, a = oracle.assemble(p, sym=True)
        x, st1, ani1, _ = oracle.scr_cg_prec(adr, ci, a, oracle.load_vector(p), ni=20000, res=1e-20)
        assert st == st1 == 0 and ani == ani1 and nrm == pytest.approx(float(np.linalg.norm(x)), rel=0, abs=0)
