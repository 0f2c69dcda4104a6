"""Replica bookkeeping of the multi-GPU bench path, as world-size-2 gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from salsaa_b200.replicas import proof_seed


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from salsaa_b200 import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, _ = replicas.rank_info()
        seeds = [replicas.proof_seed(r, step, slot, 4) for step in range(-3, 5) for slot in range(4)]
        replicas.barrier()
        mx = replicas.max_over_ranks(10.0 + 5 * rank)
        out.put((r, w, seeds, mx))
    finally:
        dist.destroy_process_group()


def test_two_ranks_disjoint_seeds_and_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert all(r[3] == 15.0 for r in res)  # max over ranks seen by every rank
    s0, s1 = set(res[0][2]), set(res[1][2])
    assert len(s0) == len(res[0][2]) and not (s0 & s1)


def test_seed_ranges():
    assert proof_seed(0, 0, 0, 8) != proof_seed(1, 0, 0, 8)
    assert proof_seed(0, 1, 0, 8) == proof_seed(0, 0, 7, 8) + 1
    with pytest.raises(ValueError):
        proof_seed(0, 0, 8, 8)
