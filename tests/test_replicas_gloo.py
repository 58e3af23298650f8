"""The multi-rank path of the benchmark on CPU: two gloo ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import td16_b200 as td
    from td16_b200 import replicas
    perms, _ = td.synth_perms(replicas.rank_seed(2, rank), 64, 16, 16, 50, 1, 4)
    t = replicas.max_over_ranks(1.5 + rank, dist)
    s = replicas.sum_over_ranks([10 * (rank + 1), rank], dist)
    q.put((rank, t, s, perms.tobytes()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction_and_disjoint_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [2.5, 2.5]          # job time = max over ranks
    assert [o[2] for o in out] == [[30.0, 1.0]] * 2   # counts summed
    a = np.frombuffer(out[0][3], np.int8).reshape(64, 16)
    b = np.frombuffer(out[1][3], np.int8).reshape(64, 16)
    assert not (a == b).all(axis=1).any()              # ranks search different instances
