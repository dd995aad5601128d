"""Host side of the multi-GPU bench on CPU: two gloo ranks (127.0.0.1).
Each rank gets its own shard (seed), the timed seconds reduce to the maximum
over ranks, and the synthetic inputs of the two shards differ."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import bench
    from racon_b200 import synthetic
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seconds = 0.5 + rank  # rank 1 is the slow one
        m = bench.max_over_ranks(seconds, world)
        seed = bench.shard_seed(1, rank)
        r, o, t, info = synthetic.contig(os.path.join(out_dir, "r%d" % rank), 0, seed=seed, scale=0.05)
        with open(t, "rb") as fh:
            draft = fh.read()
        q.put((rank, m, seed, hash(draft)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path), q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [1.5, 1.5]       # max over ranks on every rank
    assert res[0][2] != res[1][2]                  # distinct shard seeds
    assert res[0][3] != res[1][3]                  # distinct inputs


def test_single_rank_max_is_identity():
    import bench
    assert bench.max_over_ranks(2.5, 1) == 2.5
