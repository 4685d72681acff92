"""Multi-rank path on CPU (gloo, world size 2): each rank transforms its own
slice of the fields and the gathered result equals the single-process one.
The per-rank transform here is the NumPy oracle (no GPU on this machine); on
GPUs the same sharding runs the CUDA transform (bench.py under torchrun)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from shtns_b200.sharding import field_shard


def test_field_shard_covers_all_fields():
    for n in (1, 7, 64, 65):
        for w in (1, 2, 3, 8):
            got = []
            for r in range(w):
                sl = field_shard(n, r, w)
                got.extend(range(n)[sl])
            assert got == list(range(n))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q, out):
    import torch
    import torch.distributed as dist
    from oracle.sht_np import NpSHT
    from shtns_b200.sharding import field_shard, gather_fields
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = NpSHT(31, 31, 1, 0, 48, 64)
        sl = field_shard(q.shape[0], rank, world)
        v = sh.synth(q[sl])
        full = gather_fields(torch.from_numpy(v), q.shape[0])
        if rank == 0:
            out.put(full.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_synthesis_matches_single_process():
    from oracle.sht_np import NpSHT
    from tests.common import rand_spec
    q = rand_spec(31, 31, 1, 5, nfields=5)
    ref = NpSHT(31, 31, 1, 0, 48, 64).synth(q)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = out.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(got, ref)
