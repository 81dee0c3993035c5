"""Partitioned evaluation: slab partition, ghost planes and the halo exchange.

CPU (gloo, 2 and 3 ranks as processes): every rank fills its owned planes, exchanges the
ghost planes with ``HaloExchange`` (the same code that runs over NCCL between GPUs), checks
them against the global vector, evaluates its part with the oracle on the part's grid
descriptor, and the owned results are compared with the oracle on the global grid -- for a
periodic Euler operator, a periodic advection-diffusion operator and a Dirichlet SIP operator
(whose penalty needs the global boundary through ``global_n``/``global_offset``).

GPU (one device): the ranks of a partition are evaluated one after the other on the device
through ``bosss_b200_apply_device`` on the interior and rim cell ranges of each part (ghost
planes cut from the global vector, as the exchange delivers them); the assembled result
equals the single-grid device evaluation to 1e-14 relative (bit for bit in practice for the
residual and JVP), for residual, JVP and VJP.
"""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bosss_b200 import _capi as C
from bosss_b200 import distributed as Dd
from bosss_b200 import operator as O
from bosss_b200 import problems as P
from oracle import oracle as orc

CASES = {
    "euler": lambda: P.euler3d(n=6, k=1, seed=61),
    "advdiff": lambda: P.advection_diffusion3d(n=6, k=2, seed=62),
    "sip_dirichlet": lambda: P.nonlinear_diffusion3d(n=6, k=2, seed=63, source=1.0),
}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _dofs_per_cell(pr):
    return pr.n_dofs // pr.grid.NoOfCells


def _rank_main(rank, world, port, case, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        pr = CASES[case]()
        opd, _ = pr.descs()
        part = Dd.SlabPartition(pr.grid, world, rank, _dofs_per_cell(pr))
        V = np.random.default_rng(5).uniform(-1, 1, pr.n_dofs)
        U_part = torch.zeros(part.n_dofs, dtype=torch.float64)
        V_part = torch.zeros(part.n_dofs, dtype=torch.float64)
        part.own(U_part)[:] = torch.from_numpy(pr.U[part.global_slice()])
        part.own(V_part)[:] = torch.from_numpy(V[part.global_slice()])
        Dd.HaloExchange(part).exchange(U_part, V_part)
        ok_halo = bool(np.array_equal(U_part.numpy(), part.from_global(pr.U))
                       and np.array_equal(V_part.numpy(), part.from_global(V)))
        gd = part.grid_desc()
        a, b = part.own_cells()
        npc = part.dofs_per_cell
        R = orc.evaluate(opd, gd, U_part.numpy())[a * npc:b * npc]
        JV = orc.jvp(opd, gd, U_part.numpy(), V_part.numpy())[a * npc:b * npc]
        got = [None] * world
        dist.all_gather_object(got, (part.first, ok_halo, R, JV))
        if rank == 0:
            got.sort(key=lambda t: t[0])
            q.put((all(t[1] for t in got), np.concatenate([t[2] for t in got]),
                   np.concatenate([t[3] for t in got])))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", sorted(CASES))
def test_halo_exchange_and_part_evaluation_on_cpu(world, case):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        ok_halo, R, JV = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert ok_halo
    pr = CASES[case]()
    opd, gd = pr.descs()
    V = np.random.default_rng(5).uniform(-1, 1, pr.n_dofs)
    Rg = orc.evaluate(opd, gd, pr.U)
    JVg = orc.jvp(opd, gd, pr.U, V)
    assert np.max(np.abs(R - Rg)) <= 1e-13 * np.max(np.abs(Rg))
    assert np.max(np.abs(JV - JVg)) <= 1e-13 * np.max(np.abs(JVg))


def test_partition_ranges_cover_the_owned_cells():
    for per in (True, False):
        g = O.Cartesian3DGrid(np.linspace(0, 1, 10), np.linspace(0, 1, 4), np.linspace(0, 1, 3), per, True, True)
        for world in (1, 2, 3, 9):
            counts = []
            for r in range(world):
                p = Dd.SlabPartition(g, world, r, 4)
                cells = set()
                for a, b in [p.interior_cells()] + p.rim_cells():
                    assert not cells & set(range(a, b))
                    cells |= set(range(a, b))
                assert cells == set(range(*p.own_cells()))
                counts.append(p.count)
                d = p.grid_desc()
                assert d.n[0] == p.n_planes and d.lo[0] == g.lo[0] and d.hi[0] == g.hi[0]
            assert sum(counts) == 9
    with pytest.raises(ValueError):
        Dd.SlabPartition(g, 10, 0, 4)


def test_part_grid_desc_rejected_where_inconsistent():
    # a part may be periodic only in a direction it spans completely
    pr = P.advection_diffusion3d(n=6, k=1, seed=1)
    opd, gd = pr.descs()
    gd.global_n[0], gd.global_n[1], gd.global_n[2] = 12, 6, 6
    gd.global_periodic[0] = gd.global_periodic[1] = gd.global_periodic[2] = 1
    h = ctypes.c_void_p()
    rc = C.lib().bosss_b200_create(ctypes.byref(opd), ctypes.byref(gd), None, ctypes.byref(h))
    assert rc == C.ERR_BAD_ARG


def test_apply_device_rejects_bad_ranges():
    L = C.lib()
    assert L.bosss_b200_apply_device(None, 0, 1.0, 0.0, None, None, None, 0.0, 0, 1, None) == C.ERR_BAD_ARG


# ------------------------------------------------------------------------------- GPU


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3, 4])
@pytest.mark.parametrize("case", sorted(CASES))
def test_partitioned_device_evaluation_matches_global(world, case):
    import torch
    pr = CASES[case]()
    opd, gd = pr.descs()
    nvar = len(pr.dom)
    k = pr.dom[0].degree
    dev = torch.device("cuda", 0)
    W = np.random.default_rng(9).uniform(-1, 1, pr.n_dofs)
    Ug = torch.from_numpy(pr.U).to(dev)
    Wg = torch.from_numpy(W).to(dev)
    ev = pr.evaluator()
    try:
        Rg = torch.zeros_like(Ug)
        ev.Evaluate(1.0, 0.0, Rg, Ug)
        JVg = ev.jvp(Ug, Wg)
        JTg = ev.vjp(Ug, Wg)
        torch.cuda.synchronize()
    finally:
        ev.Dispose()
    outs = {m: np.zeros(pr.n_dofs) for m in ("res", "jvp", "vjp")}
    for r in range(world):
        part = Dd.SlabPartition(pr.grid, world, r, _dofs_per_cell(pr))
        pe = Dd.PartEvaluator(pr.op, pr.grid, [k] * nvar, [k] * nvar, part)
        try:
            U = part.from_global(Ug)
            V = part.from_global(Wg)
            for name, mode in (("res", C.MODE_RESIDUAL), ("jvp", C.MODE_JVP), ("vjp", C.MODE_VJP)):
                out = torch.full_like(U, float("nan"))
                for cells in [part.interior_cells()] + part.rim_cells():
                    pe.apply(mode, U, V, out, cells)
                torch.cuda.synchronize()
                outs[name][part.global_slice()] = part.own(out).cpu().numpy()
        finally:
            pe.Dispose()
    for name, ref in (("res", Rg), ("jvp", JVg), ("vjp", JTg)):
        # the same arithmetic per cell; only the tile a cell shares with its neighbours differs,
        # which can move the last bit of the VJP
        ref = ref.cpu().numpy()
        assert np.max(np.abs(outs[name] - ref)) <= 1e-14 * np.max(np.abs(ref)), name
    Ro = orc.evaluate(opd, gd, pr.U)
    assert np.max(np.abs(outs["res"] - Ro)) <= 1e-12 * np.max(np.abs(Ro))
