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


def boundary_kinds_by_face(gd, nq, kind_of):
    """Kinds in the boundary-node order (cell, direction d, side s, face node) from
    kind_of(d, s); nq Gauss nodes per direction."""
    D = gd.dim
    n = [gd.n[d] for d in range(D)]
    nqf = nq ** (D - 1)
    out = []
    for j in range(int(np.prod(n))):
        ijk = np.unravel_index(j, n)
        for d in range(D):
            for s in range(2):
                if not gd.periodic[d] and ijk[d] == (0 if s == 0 else n[d] - 1):
                    out += [kind_of(d, s)] * nqf
    return np.array(out, dtype=np.int32)


def test_free_stream_with_inflow_outlet_and_walls():
    """Uniform flow along x in a 2D channel: inflow state at x = 0 (table), supersonic-outlet
    state at x = 1, slip walls at y = 0, 1 (the flow is tangential there): zero residual."""
    pr = P.euler2d(n=4, k=2, seed=93, periodic=(False, False))
    opd, gd = pr.descs()
    state = np.array([1.1, 0.4, 0.0, 2.9])
    U = _constant(pr, state, 0.25)
    nq = orc.sizes(opd, gd)[2]
    kinds = boundary_kinds_by_face(gd, nq, lambda d, s: (0 if s == 0 else 1) if d == 0 else 2)
    nb = orc.n_boundary_nodes(opd, gd)
    assert len(kinds) == nb
    with orc.boundary_kinds(kinds):
        R = orc.evaluate(opd, gd, U, bnd=np.tile(state, (nb, 1)))
    assert np.abs(R).max() <= 1e-13
    # a wall-normal velocity is reflected, not kept: the residual is no longer zero
    state2 = np.array([1.1, 0.4, 0.3, 2.9])
    with orc.boundary_kinds(kinds):
        R2 = orc.evaluate(opd, gd, _constant(pr, state2, 0.25), bnd=np.tile(state2, (nb, 1)))
    assert np.abs(R2).max() > 1e-6


def test_vjp_with_boundary_kinds_is_transposed_jacobian():
    pr = P.euler3d(n=3, k=1, seed=94, periodic=(False, True, False))
    opd, gd = pr.descs()
    nb = orc.n_boundary_nodes(opd, gd)
    kinds = np.random.default_rng(3).integers(0, 3, nb).astype(np.int32)
    bnd = np.tile([1.05, 0.1, 0.05, -0.1, 2.6], (nb, 1))
    W = np.random.default_rng(4).uniform(-1, 1, pr.n_dofs)
    V = np.random.default_rng(5).uniform(-1, 1, pr.n_dofs)
    with orc.boundary_kinds(kinds):
        A = orc.jacobian_dense(opd, gd, pr.U, bnd=bnd)
        G = orc.vjp(opd, gd, pr.U, W, bnd=bnd)
        JV = orc.jvp(opd, gd, pr.U, V, bnd=bnd)
        # central differences of the residual in direction V (state-dependent outer states)
        eps = 1e-6
        fd = (orc.evaluate(opd, gd, pr.U + eps * V, bnd=bnd) - orc.evaluate(opd, gd, pr.U - eps * V, bnd=bnd)) / (2 * eps)
    assert np.linalg.norm(G - A.T @ W) <= 1e-12 * np.linalg.norm(G)
    assert np.linalg.norm(JV - A @ V) <= 1e-12 * np.linalg.norm(JV)
    assert np.linalg.norm(fd - JV) <= 1e-7 * np.linalg.norm(JV)
