"""Per-instance implicit-step solves over a batch (``bosss_b200_batch_solve``): FP32 GMRES
inside FP64 iterative refinement, matrix-free on the instance's JVP (forward systems) or VJP
(adjoint systems), block-Jacobi on probed diagonal blocks or no preconditioner.

Checked against the oracle for every instance: the true residual of (I/dt + A_i) x_i = b_i
(and of the transposed system) <= 1e-10 relative, and the dense solve of the oracle's
assembled matrix for the smallest instance.
"""
import numpy as np
import pytest

from bosss_b200 import operator as O
from bosss_b200 import problems as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _batch():
    # SIPLaplace discretises +nu Laplace(u) (ipLaplace.cs:183-186), so nu < 0 makes the
    # advection-diffusion operator dissipative (du/dt = -Op(u) stable) and I/dt + J positive
    return P.batched_advection_diffusion(n_instances=6, seed=78, sizes=(3, 4, 5), degrees=(1, 2, 3), nu=-0.01)


def _dt(probs):
    # one cell per time step at the instance's transport speed
    return np.array([(1.0 / p.grid.n[0]) / np.linalg.norm(p.config["velocity"]) for p in probs])


@pytest.mark.parametrize("precond", [1, 0, 2], ids=["block_jacobi", "none", "multigrid"])
def test_batch_solve_forward_and_adjoint(precond):
    import torch
    probs = _batch()
    n = sum(p.n_dofs for p in probs)
    b = np.random.default_rng(3).uniform(-1, 1, n)
    dt = _dt(probs)
    with O.BatchEvaluator(probs) as B:
        off = B.dom_offsets
        bt = torch.from_numpy(b).cuda()
        x, reps = B.solve(dt, bt, precond=precond)
        xa, repa = B.solve(dt, bt, transpose=True, precond=precond)
        x, xa = x.cpu().numpy(), xa.cpu().numpy()
    assert all(r["converged"] for r in reps + repa), (reps, repa)
    assert max(r["outer_iters"] for r in reps) >= 2      # FP32 inner solves need refinement
    for i, p in enumerate(probs):
        sl = slice(off[i], off[i + 1])
        opd, gd = p.descs()
        zero = np.zeros(p.n_dofs)
        Ax = orc.jvp(opd, gd, zero, x[sl])
        assert rel(x[sl] / dt[i] + Ax, b[sl]) <= 1e-10, i
        ATx = orc.vjp(opd, gd, zero, xa[sl])
        assert rel(xa[sl] / dt[i] + ATx, b[sl]) <= 1e-10, i
    # the smallest instance against a dense solve of the oracle's matrix
    i = int(np.argmin([p.n_dofs for p in probs]))
    p = probs[i]
    A = orc.jacobian_dense(*p.descs(), np.zeros(p.n_dofs)) + np.eye(p.n_dofs) / dt[i]
    sl = slice(off[i], off[i + 1])
    assert rel(x[sl], np.linalg.solve(A, b[sl])) <= 1e-9
    assert rel(xa[sl], np.linalg.solve(A.T, b[sl])) <= 1e-9


def test_batch_solve_rejects_bad_arguments():
    import torch
    from bosss_b200 import _capi as C
    probs = _batch()[:2]
    n = sum(p.n_dofs for p in probs)
    with O.BatchEvaluator(probs) as B:
        bt = torch.ones(n, dtype=torch.float64, device="cuda")
        for dt, kw in ((-1.0, {}), (0.1, {"precond": 3})):
            with pytest.raises(C.BosssError) as ei:
                B.solve(dt, bt, **kw)
            assert ei.value.code == C.ERR_BAD_ARG
