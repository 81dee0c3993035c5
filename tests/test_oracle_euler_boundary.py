"""The oracle's HLLC boundary flux (OptimizedHLLCFlux.BorderEdgeFlux with the outer state
from the boundary-state table) on the CPU: free-stream preservation on a bounded grid
(uniform state, the same state outside: zero residual, a known answer), a state-dependent
check that the boundary terms are active (another outer state changes only the boundary
cells), and the exact VJP equal to the transposed cell-block Jacobian."""
import numpy as np

from bosss_b200 import problems as P
from oracle import oracle as orc


def _constant(pr, state, h):
    Np = pr.dom[0].Np
    J = pr.grid.NoOfCells
    U = np.zeros((J, len(state), Np))
    U[:, :, 0] = np.asarray(state) * np.sqrt(h ** pr.grid.dim)
    return U.ravel()


def test_free_stream_with_boundaries():
    pr = P.euler2d(n=4, k=2, seed=91, periodic=(False, False))
    opd, gd = pr.descs()
    state = np.array([1.2, 0.3, -0.2, 2.7])
    U = _constant(pr, state, 0.25)
    n = orc.n_boundary_nodes(opd, gd)
    R = orc.evaluate(opd, gd, U, bnd=np.tile(state, (n, 1)))
    assert np.abs(R).max() <= 1e-13
    # a different outer state: only cells with a boundary face change
    R2 = orc.evaluate(opd, gd, U, bnd=np.tile(state * np.array([1.1, 1.0, 1.0, 1.05]), (n, 1)))
    per_cell = np.abs(R2.reshape(16, -1)).max(axis=1)
    ij = np.stack(np.unravel_index(np.arange(16), (4, 4)), axis=1)
    on_bnd = (ij == 0).any(axis=1) | (ij == 3).any(axis=1)
    assert np.all(per_cell[on_bnd] > 1e-6) and np.all(per_cell[~on_bnd] <= 1e-13)


def test_vjp_is_transposed_jacobian_with_boundaries():
    pr = P.euler3d(n=3, k=1, seed=92, periodic=(False, True, False))
    opd, gd = pr.descs()
    n = orc.n_boundary_nodes(opd, gd)
    bnd = np.tile([1.05, 0.1, 0.05, -0.1, 2.6], (n, 1)) * (1 + 0.05 * np.random.default_rng(1).uniform(-1, 1, (n, 1)))
    W = np.random.default_rng(2).uniform(-1, 1, pr.n_dofs)
    A = orc.jacobian_dense(opd, gd, pr.U, bnd=bnd)
    G = orc.vjp(opd, gd, pr.U, W, bnd=bnd)
    assert np.linalg.norm(G - A.T @ W) <= 1e-12 * np.linalg.norm(G)
