"""One grid split into x-slabs on two gloo ranks (CPU, the oracle as the
stepper): owned rows after every exchange equal the single-grid run bit for
bit, for Neumann and periodic x boundaries and halo depths 1 and 2, through the
host-array exchange and through exchange_tensors (the code the GPUs run on
their contexts' streams over NCCL, here on host tensors over gloo)."""
import copy
import multiprocessing as mp
import os
import socket
from datetime import timedelta

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _local_state(gphi, gmu, slab, mx, bc_x):
    """Ghost-padded local arrays of a slab cut from ghost-padded global ones."""
    from microsim_b200 import slab as S
    rows = [S.gmap(g, mx, bc_x) if (g < 0 or g >= mx) else g for g in range(slab.lo, slab.hi)]
    inner_p = gphi[:, 3:-3][:, rows]
    inner_u = gmu[:, 3:-3][:, rows]
    P, U = inner_p.shape[0], inner_u.shape[0]
    lp = np.zeros((P, slab.rows + 6, gphi.shape[2]))
    lu = np.zeros((U, slab.rows + 6, gmu.shape[2]))
    lp[:, 3:-3] = inner_p
    lu[:, 3:-3] = inner_u
    return lp, lu


def _worker(rank, world, port, case, depth, steps, q, transport="numpy"):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import sys
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        from conftest import load_golden, oracle_model
        from oracle import gp_oracle as O
        from microsim_b200 import slab as S
        g = load_golden(case)
        m = oracle_model(g)
        mx, bc_x = m.mesh_x, m.bc_phi[0]
        slabs, copies = S.plan(mx, world, bc_x, depth)
        s = slabs[rank]
        lm = copy.copy(m)
        lm.mesh_x = s.rows
        if s.lo != s.own_lo or s.hi != s.own_hi:
            lm.bc_phi = (1, 1) + tuple(m.bc_phi[2:])
            lm.bc_mu = (1, 1) + tuple(m.bc_mu[2:])
        lp, lu = _local_state(g["phi_0"], g["mu_0"], s, mx, bc_x)
        O.apply_bc(lm, lp, lu)
        done = 0
        while done < steps:
            O.step(lm, lp, lu, depth)
            done += depth
            if transport == "numpy":
                S.exchange_numpy([lp[:, 3:-3], lu[:, 3:-3]], copies, rank, world)
            else:
                import torch
                S.exchange_tensors(torch.from_numpy(lp[:, 3:-3]), torch.from_numpy(lu[:, 3:-3]), copies, rank)
            O.apply_bc(lm, lp, lu)
        own = slice(3 + s.own_lo - s.lo, 3 + s.own_hi - s.lo)
        q.put((rank, s.own_lo, s.own_hi, lp[:, own, 3:-3].copy(), lu[:, own, 3:-3].copy()))
    except Exception as e:  # report instead of leaving the parent waiting
        q.put((rank, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,depth,transport", [("iso_obst_bin", 1, "numpy"), ("iso_obst_bin", 2, "numpy"),
                                                   ("aniso_obst_bin_per", 1, "numpy"),
                                                   ("iso_obst_bin", 2, "tensors"),
                                                   ("aniso_obst_bin_per", 1, "tensors")])
def test_slabs_on_two_gloo_ranks_equal_the_single_grid(case, depth, transport):
    from conftest import load_golden, oracle_model
    from oracle import gp_oracle as O
    steps = 12
    g = load_golden(case)
    m = oracle_model(g)
    phi, mu = g["phi_0"].copy(), g["mu_0"].copy()
    O.step(m, phi, mu, steps)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, case, depth, steps, q, transport)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=180) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    assert all(len(o) == 5 for o in out), [o for o in out if len(o) != 5]
    assert all(p.exitcode == 0 for p in ps)
    covered = 0
    for rank, lo, hi, lp, lu in out:
        assert np.array_equal(lp, phi[:, 3 + lo:3 + hi, 3:-3]), (rank, np.abs(lp - phi[:, 3 + lo:3 + hi, 3:-3]).max())
        assert np.array_equal(lu, mu[:, 3 + lo:3 + hi, 3:-3])
        covered += hi - lo
    assert covered == m.mesh_x


def test_plan_covers_every_row_once():
    from microsim_b200 import slab as S
    with pytest.raises(ValueError):
        S.plan(64, 2, 3, 2)  # the periodic copy is refreshed every step
    for mx, world, bc, depth in [(100, 4, 1, 2), (37, 3, 3, 1), (64, 8, 3, 1), (90, 5, 1, 3)]:
        slabs, copies = S.plan(mx, world, bc, depth)
        owned = sorted(g for s in slabs for g in range(s.own_lo, s.own_hi))
        assert owned == list(range(mx))
        for (sr, srow, dr, drow) in copies:
            src = slabs[sr]
            assert src.own_lo <= src.lo + srow < src.own_hi  # halos come from owned rows only
