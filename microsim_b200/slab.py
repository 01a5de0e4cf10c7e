"""One grid split across ranks along x (the reference's slow index): each rank
steps a slab of rows with the plain C ABI context, the slabs exchanging halo
rows every `depth` steps.

Layout: rank r owns the global rows [own_lo, own_hi) and holds the local rows
[lo, hi) = [own_lo - H, own_hi + H), H = 3 * depth halo rows on each side
(none on a side where the global boundary copy is a Neumann mirror: there the
slab's own first/last row is the grid's).  A periodic x boundary takes depth 1:
the reference's periodic copy (period M - 1) is no continuation of the grid.  A step needs phi at +-2 rows and mu
at +-1 row of every updated row (Delta-phi on one ring around it); so after an
exchange the owned rows stay exact for `depth` steps while the halo rows decay
from the outside in.  The halo rows are ordinary rows of the local grid: no
kernel change, the boundary map acts only where the slab ends.  Global rows
outside [0, M) (periodic x) come from the partner of the reference's periodic
copy, period M - 1 (microsim_b200/csrc/gp_common.cuh gp_map).

The exchange is written against a small transport: `numpy` (host arrays of a
process group over torch.distributed: gloo on the CPU, for the oracle), or
torch tensors (exchange_tensors: NCCL between GPUs, ordered on the stepping
context's stream with no host synchronisation; the same code on host tensors
over gloo), or local device copies when the slabs of one process share a GPU.
"""
from __future__ import annotations

from dataclasses import dataclass

NEUMANN, PERIODIC = 1, 3


def gmap(v: int, M: int, bc: int) -> int:
    """The reference's ghost index map (gp_map)."""
    if v < 0:
        return -v if bc == NEUMANN else M - 1 + v
    if v >= M:
        return 2 * M - 2 - v if bc == NEUMANN else 1 + v - M
    return v


@dataclass
class Slab:
    rank: int
    own_lo: int
    own_hi: int
    lo: int
    hi: int

    @property
    def rows(self) -> int:
        return self.hi - self.lo


def plan(mx: int, world: int, bc_x: int, depth: int = 1):
    """Slabs of every rank and the halo copies [(src rank, src local row, dst
    rank, dst local row)] one exchange makes."""
    if bc_x == PERIODIC and depth > 1:
        # the reference's periodic copy (period M - 1) is no continuation of the
        # grid: row -1 takes row M - 2 while row M - 2's own neighbour is M - 1,
        # so wrapped halo rows must be refreshed from their partner every step
        raise ValueError("a periodic x boundary needs an exchange every step (depth 1)")
    H = 3 * depth
    slabs = []
    for r in range(world):
        o0, o1 = r * mx // world, (r + 1) * mx // world
        if o1 - o0 < H:
            raise ValueError(f"rank {r} owns {o1 - o0} rows, fewer than the halo depth {H}")
        lo = o0 - H if (o0 > 0 or bc_x == PERIODIC) else o0
        hi = o1 + H if (o1 < mx or bc_x == PERIODIC) else o1
        slabs.append(Slab(r, o0, o1, lo, hi))
    owner = {}
    for s in slabs:
        for g in range(s.own_lo, s.own_hi):
            owner[g] = s
    copies = []
    for s in slabs:
        for g in list(range(s.lo, s.own_lo)) + list(range(s.own_hi, s.hi)):
            src_g = gmap(g, mx, bc_x) if (g < 0 or g >= mx) else g
            o = owner[src_g]
            copies.append((o.rank, src_g - o.lo, s.rank, g - s.lo))
    return slabs, copies


def blocks(copies, rank: int):
    """This rank's sends and receives grouped by partner: {partner: [(src row,
    dst row), ...]} in a fixed order both sides agree on."""
    sends, recvs = {}, {}
    for (sr, srow, dr, drow) in copies:
        if sr == rank and dr != rank:
            sends.setdefault(dr, []).append((srow, drow))
        if dr == rank and sr != rank:
            recvs.setdefault(sr, []).append((srow, drow))
    local = [(srow, drow) for (sr, srow, dr, drow) in copies if sr == rank and dr == rank]
    return sends, recvs, local


def local_model(model, slab: Slab):
    """The slab's model: its rows, and the Neumann map at an edge that is a halo
    (any map would do: those rows are overwritten by the next exchange)."""
    m = model.copy()
    m.mesh_x = slab.rows
    bp, bm = list(m.bc_phi), list(m.bc_mu)
    if slab.lo != slab.own_lo or slab.hi != slab.own_hi:
        bp[0] = bp[1] = NEUMANN
        bm[0] = bm[1] = NEUMANN
    for i in range(4):
        m.bc_phi[i] = bp[i]
        m.bc_mu[i] = bm[i]
    return m


# ------------------------------------------------------------------ exchanges

def exchange_numpy(fields, copies, rank: int, world: int):
    """Halo rows of host arrays fields = [array [planes, rows, ny], ...] (all
    planes of the local state, rows along axis 1) over torch.distributed (gloo)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    sends, recvs, local = blocks(copies, rank)
    for (srow, drow) in local:
        for f in fields:
            f[:, drow] = f[:, srow]
    planes = [f.shape[0] for f in fields]
    ops, bufs = [], []
    for partner in sorted(set(sends) | set(recvs)):
        if partner in sends:  # [rows][all planes][ny]
            data = np.stack([np.concatenate([f[:, srow] for f in fields]) for (srow, _) in sends[partner]])
            ops.append(dist.P2POp(dist.isend, torch.from_numpy(np.ascontiguousarray(data)), partner))
        if partner in recvs:
            t = torch.empty((len(recvs[partner]), sum(planes), fields[0].shape[2]),
                            dtype=torch.from_numpy(np.ascontiguousarray(fields[0][:1, :1, :1])).dtype)
            ops.append(dist.P2POp(dist.irecv, t, partner))
            bufs.append((partner, t))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for partner, t in bufs:
        a = t.numpy()
        for i, (_, drow) in enumerate(recvs[partner]):
            o = 0
            for f, n in zip(fields, planes):
                f[:, drow] = a[i, o:o + n]
                o += n


def exchange_tensors(phi, mu, copies, rank: int, stream=None):
    """Halo rows of one rank's state given as tensors phi [P, rows, ny], mu [Q,
    rows, ny] (device or host) over torch.distributed: local copies, then one
    batch of sends and receives per partner (rows packed [phi planes, mu planes]
    in the order blocks() fixes on both sides), then the received rows
    unpacked.  With `stream` (a CUDA stream: the stepping context's own), every
    operation is ordered on it and the host never waits: the NCCL work is
    joined to the stream (Work.wait() makes the stream, not the host, wait), so
    the next step launched on that stream sees the new rows.  On host tensors
    (gloo) the same code runs synchronously."""
    import contextlib
    import torch
    import torch.distributed as dist
    sends, recvs, local = blocks(copies, rank)
    P, Q, ny = phi.shape[0], mu.shape[0], phi.shape[2]
    ctx = torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()
    with ctx:
        for (srow, drow) in local:
            phi[:, drow].copy_(phi[:, srow])
            mu[:, drow].copy_(mu[:, srow])
        ops, bufs = [], []
        for partner in sorted(set(sends) | set(recvs)):
            if partner in sends:
                rows = [r for (r, _) in sends[partner]]
                ops.append(dist.P2POp(dist.isend, torch.cat([phi[:, rows].reshape(-1), mu[:, rows].reshape(-1)]),
                                      partner))
            if partner in recvs:
                t = torch.empty((P + Q) * len(recvs[partner]) * ny, dtype=phi.dtype, device=phi.device)
                ops.append(dist.P2POp(dist.irecv, t, partner))
                bufs.append((partner, t))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for partner, t in bufs:
            rows = [d for (_, d) in recvs[partner]]
            n = len(rows)
            phi[:, rows] = t[: P * n * ny].reshape(P, n, ny)
            mu[:, rows] = t[P * n * ny:].reshape(Q, n, ny)


def exchange_local(ctxs, copies):
    """Halo rows between contexts of one process (the slabs share the GPU):
    device-to-device copies of whole rows, ordered on the GPU (every context's
    stream is joined into one copy stream and waits on it afterwards; the host
    does not wait)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    streams = [torch.cuda.ExternalStream(c.stream, device=dev) for c in ctxs]
    cs = torch.cuda.current_stream(dev)
    for s in streams:
        ev = torch.cuda.Event()
        ev.record(s)
        cs.wait_event(ev)
    views = [c.device_state() for c in ctxs]
    with torch.cuda.stream(cs):
        for (sr, srow, dr, drow) in copies:
            for k in range(2):  # phi planes, mu planes
                views[dr][k][:, drow].copy_(views[sr][k][:, srow])
    done = torch.cuda.Event()
    done.record(cs)
    for s, c in zip(streams, ctxs):
        s.wait_event(done)
        c.state_changed()


def exchange_nccl(ctx, copies, rank: int, index: int | None = None):
    """Halo rows of this rank's state with the other ranks (torch.distributed
    over NCCL; one process per GPU, the context or batch created after
    microsim_b200.set_device(local rank)), stream-ordered on the context's (or
    the batch's) own stream: no host synchronisation.  `ctx` is a Context, or a
    Batch with `index` the instance holding this rank's slab."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    phi, mu = ctx.device_state() if index is None else ctx.device_state(index)
    exchange_tensors(phi, mu, copies, rank, stream=torch.cuda.ExternalStream(ctx.stream, device=dev))
    ctx.state_changed()


def exchange_batch_local(batch, copies):
    """Halo rows between the instances of one batch (instance r holds slab r; one
    GPU): device copies ordered on the batch's own stream (no host wait), then
    the batch's purity words reset (also on its stream)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    views = [batch.device_state(i) for i in range(len(batch.models))]
    with torch.cuda.stream(torch.cuda.ExternalStream(batch.stream, device=dev)):
        for (sr, srow, dr, drow) in copies:
            for k in range(2):  # phi planes, mu planes
                views[dr][k][:, drow].copy_(views[sr][k][:, srow])
    batch.state_changed()
