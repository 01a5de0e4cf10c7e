"""Multi-rank plumbing of the benchmark on CPU (gloo, world size 2): each rank
gets its own instances of the sweep (rank 0 the standard one, none shared),
single-instance workloads are replicated, and the timing / cell-count
reductions are max / sum over ranks."""
import hashlib
import multiprocessing as mp
import os
import socket
from datetime import timedelta


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from microsim_b200 import ranks
        _, cases = ranks.shard_workload("c4", rank, world, n=8)
        sig = [hashlib.sha1((c.input_text() + c.filling_text()).encode()).hexdigest() for c in cases]
        every = [None] * world
        dist.all_gather_object(every, sig)
        _, single = ranks.shard_workload("c2", rank, world)
        one = [None] * world
        dist.all_gather_object(one, single[0].input_text())
        mx = ranks.allreduce(rank + 1.5, world, "max")
        sm = ranks.allreduce(rank + 1.0, world, "sum")
        q.put((rank, every, one, mx, sm))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_instances_and_reduce():
    from microsim_b200 import configs
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, every, one, mx, sm in out:
        assert mx == 2.5 and sm == 3.0
        assert one[0] == one[1]                       # single instance: replicas
        assert not set(every[0]) & set(every[1])      # sweep: no instance on two ranks
        std = [hashlib.sha1((c.input_text() + c.filling_text()).encode()).hexdigest() for c in configs.c4(n=8)]
        assert every[0] == std                         # rank 0 runs the standard sweep
