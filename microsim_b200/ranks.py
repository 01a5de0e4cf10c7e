"""Multi-GPU plumbing of the benchmark: one process per GPU, no data-path
collective.

Independent instances shard: under torchrun every rank runs its own batch of
the sweep, drawn from its own seed (rank 0 gets the standard sweep), so the
ranks never exchange fields; the per-GPU work is fixed as N grows ("weak").
A single-instance workload does not shard here: every rank runs a replica.
The only collectives are the scalar reductions of the timing (max over ranks)
and of the cell counts (sum), in FP64, on whatever backend the process group
uses (NCCL on the GPUs, gloo on the CPU tests).
"""
from __future__ import annotations

from . import configs


def shard_workload(name: str, rank: int = 0, world: int = 1, n: int = 256):
    """(workload label, cases of this rank)."""
    if name == "c4":
        label = f"batched_sweep_{n}_instances_128-512" + (f"_per_rank_x{world}" if world > 1 else "")
        return label, configs.c4(n=n, rng_seed=4 + rank)
    if name == "c2":
        return "dendrite_1024x1024_delta0.02_supersat0.55 (growing gap)", [configs.c2(literal=False, steps=50000)]
    if name == "c1":
        return "isotropic_200x200_seed10 (growing gap)", [configs.c1(literal=False, steps=10000)]
    raise ValueError("unknown workload " + name)


def allreduce(v: float, world: int, op: str = "max") -> float:
    """Scalar max / sum over ranks (identity for one rank)."""
    if world == 1:
        return float(v)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())
