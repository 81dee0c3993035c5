"""Batched persistent evaluation of independent instances (mixed sizes and degrees):
results equal the single-instance evaluator per instance and the oracle, for residual,
JVP and VJP; CUDA-graph replay reproduces the direct launch; the autotuner persists and
reloads its table."""
import os

import numpy as np
import pytest

from bosss_b200 import _capi as C
from bosss_b200 import operator as O
from bosss_b200 import problems as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def small_batch():
    return P.batched_advection_diffusion(n_instances=10, seed=77, sizes=(3, 4, 5), degrees=(1, 2, 3, 4))


@pytest.mark.parametrize("kernel", [C.KERNEL_AUTO, C.KERNEL_GENERIC, C.KERNEL_SLAB],
                         ids=["auto", "generic_tiles", "slab_tiles"])
def test_batch_matches_single_and_oracle(kernel):
    probs = small_batch()
    U = np.concatenate([p.U for p in probs])
    r = np.random.default_rng(1)
    V = r.uniform(-1, 1, U.size)
    with O.BatchEvaluator(probs, kernel=kernel) as b:
        off = b.dom_offsets
        R = b.evaluate(C.MODE_RESIDUAL, U)
        JV = b.evaluate(C.MODE_JVP, U, V)
        G = b.evaluate(C.MODE_VJP, U, V)
    for i, p in enumerate(probs):
        sl = slice(off[i], off[i + 1])
        ref = orc.evaluate(*p.descs(), p.U)
        assert rel(R[sl], ref) <= 1e-12
        assert rel(JV[sl], orc.jvp(*p.descs(), p.U, V[sl])) <= 1e-12
        with p.evaluator() as ev:
            assert rel(G[sl], ev.vjp(p.U, V[sl])) <= 1e-13
            single = np.zeros(p.n_dofs)
            ev.Evaluate(1.0, 0.0, single, p.U)
            assert rel(R[sl], single) <= 1e-13


def test_batch_graph_replay_and_autotune(tmp_path):
    import torch
    probs = small_batch()
    U = torch.from_numpy(np.concatenate([p.U for p in probs])).cuda()
    W = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, U.numel())).cuda()
    R = torch.zeros_like(U)
    G = torch.zeros_like(U)
    table = str(tmp_path / "tiles.txt")
    with O.BatchEvaluator(probs) as b:
        Rd = b.evaluate(C.MODE_RESIDUAL, U)
        Gd = b.evaluate(C.MODE_VJP, U, W)
        b.autotune(U, W, R, G, table)
        assert os.path.exists(table)
        b.capture(U, W, R, G)
        R.zero_()
        G.zero_()
        b.replay()
        torch.cuda.synchronize()
        assert torch.equal(R, Rd) and torch.equal(G, Gd)
        tiles = {kq: b.tiles(*kq) for kq in [(1, 2), (2, 3), (3, 4), (4, 5)]}
    # a second batch reads the persisted table instead of re-timing
    with O.BatchEvaluator(probs) as b2:
        b2.autotune(U, W, R, G, table)
        assert {kq: b2.tiles(*kq) for kq in tiles} == tiles


@pytest.mark.parametrize("schedule", ["classes", "lpt", "fifo"])
def test_batch_schedules_match_single_instances(tmp_path, schedule):
    """Each schedule (persisted in the autotuner's table) gives the single-instance results."""
    import torch
    probs = small_batch()
    U = torch.from_numpy(np.concatenate([p.U for p in probs])).cuda()
    W = torch.from_numpy(np.random.default_rng(4).uniform(-1, 1, U.numel())).cuda()
    R = torch.zeros_like(U)
    G = torch.zeros_like(U)
    table = tmp_path / "tiles.txt"
    table.write_text("schedule %s\n" % schedule)
    with O.BatchEvaluator(probs) as b:
        b.autotune(U, W, R, G, str(table))
        assert b.tiles(1, 2)[1] == schedule
        Rb = b.evaluate(C.MODE_RESIDUAL, U)
        JV = b.evaluate(C.MODE_JVP, U, W)
        Gb = b.evaluate(C.MODE_VJP, U, W)
        torch.cuda.synchronize()
        off = b.dom_offsets
    for i, p in enumerate(probs):
        sl = slice(int(off[i]), int(off[i + 1]))
        Ui, Wi = U[sl], W[sl]
        with p.evaluator() as ev:
            Rs = torch.zeros_like(Ui)
            ev.Evaluate(1.0, 0.0, Rs, Ui)
            JVs = ev.jvp(Ui, Wi)
            Gs = ev.vjp(Ui, Wi)
            torch.cuda.synchronize()
        assert rel(Rb[sl].cpu().numpy(), Rs.cpu().numpy()) <= 1e-13
        assert rel(JV[sl].cpu().numpy(), JVs.cpu().numpy()) <= 1e-13
        assert rel(Gb[sl].cpu().numpy(), Gs.cpu().numpy()) <= 1e-13


def test_full_c5_mix_one_instance_per_class_matches_oracle():
    """The full seed-5000 mix (256 instances, 16..48^3, k = 1..4, 188M DOFs): residual and
    VJP of the whole batch in one launch per mode; the first instance of every
    (grid size, degree) class against the oracle's residual and exact VJP."""
    import torch
    probs = P.batched_advection_diffusion(n_instances=256, seed=5000)
    n = sum(p.n_dofs for p in probs)
    U = torch.from_numpy(np.concatenate([p.U for p in probs])).cuda()
    W = torch.from_numpy(np.random.default_rng(7).uniform(-1, 1, n)).cuda()
    with O.BatchEvaluator(probs) as b:
        off = b.dom_offsets
        R = b.evaluate(C.MODE_RESIDUAL, U)
        G = b.evaluate(C.MODE_VJP, U, W)
        torch.cuda.synchronize()
    seen = {}
    for i, p in enumerate(probs):
        key = (p.grid.n[0], p.dom[0].degree)
        if key not in seen:
            seen[key] = i
    assert len(seen) == 16, sorted(seen)
    for key, i in sorted(seen.items()):
        p = probs[i]
        sl = slice(int(off[i]), int(off[i + 1]))
        opd, gd = p.descs()
        Wi = W[sl].cpu().numpy()
        assert rel(R[sl].cpu().numpy(), orc.evaluate(opd, gd, p.U)) <= 1e-12, key
        assert rel(G[sl].cpu().numpy(), orc.vjp(opd, gd, p.U, Wi)) <= 1e-12, key
