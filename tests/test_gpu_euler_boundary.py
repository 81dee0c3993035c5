"""HLLC fluxes on grids with boundary faces (OptimizedHLLCFlux.BorderEdgeFlux,
OptimizedHLLCFlux.cs:61-131): the outer state comes from the boundary-state table, then the
inner-edge HLLC flux is evaluated with the outward normal.

GPU against the oracle with the same table (relative L2 <= 1e-12): residual, JVP, VJP (and
the VJP against the transposed oracle Jacobian) on 2D and 3D grids bounded in some or all
directions; free-stream preservation (uniform state, table = that state: zero residual);
missing table and slab-kernel requests rejected.
"""
import numpy as np
import pytest

from bosss_b200 import _capi as C
from bosss_b200 import problems as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


CASES = [
    ("euler2d_5_k2_bounded", lambda: P.euler2d(n=5, k=2, seed=81, periodic=(False, False))),
    ("euler2d_6_k1_x_bounded", lambda: P.euler2d(n=6, k=1, seed=82, periodic=(False, True))),
    ("euler3d_3_k2_bounded", lambda: P.euler3d(n=3, k=2, seed=83, periodic=(False, False, False))),
    ("euler3d_4_k1_z_bounded", lambda: P.euler3d(n=4, k=1, seed=84, periodic=(True, True, False))),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_bounded_euler_matches_oracle(name, make):
    pr = make()
    opd, gd = pr.descs()
    r = np.random.default_rng(9)
    V = r.uniform(-1, 1, pr.n_dofs)
    W = r.uniform(-1, 1, pr.n_dofs)
    with pr.evaluator() as ev:
        assert ev.kernel_info(C.MODE_RESIDUAL)[0] == 1          # generic kernel
        xyz = ev.boundary_nodes()
        bnd = P.euler_boundary_states(xyz)
        ev.SetBoundaryState(bnd)
        R = np.zeros(pr.n_dofs)
        ev.Evaluate(1.0, 0.0, R, pr.U)
        JV = ev.jvp(pr.U, V)
        G = ev.vjp(pr.U, W)
    assert orc.n_boundary_nodes(opd, gd) == len(xyz)
    assert rel(R, orc.evaluate(opd, gd, pr.U, bnd=bnd)) <= TOL
    assert rel(JV, orc.jvp(opd, gd, pr.U, V, bnd=bnd)) <= TOL
    assert rel(G, orc.vjp(opd, gd, pr.U, W, bnd=bnd)) <= TOL
    A = orc.jacobian_dense(opd, gd, pr.U, bnd=bnd)
    assert rel(G, A.T @ W) <= 1e-11
    assert rel(JV, A @ V) <= 1e-11


def test_bounded_euler_free_stream():
    pr = P.euler3d(n=3, k=2, seed=85, periodic=(False, True, False))
    Np = pr.dom[0].Np
    J = pr.grid.NoOfCells
    state = np.array([1.1, 0.2, -0.1, 0.15, 2.9])
    U = np.zeros((J, 5, Np))
    # constant field: mode 0 only, value * sqrt(cell volume) (orthonormal basis, 1/sqrt(detJ) scaling)
    h = 1.0 / 3
    U[:, :, 0] = state * np.sqrt(h ** 3)
    U = U.ravel()
    with pr.evaluator() as ev:
        n = len(ev.boundary_nodes())
        ev.SetBoundaryState(np.tile(state, (n, 1)))
        R = np.zeros(pr.n_dofs)
        ev.Evaluate(1.0, 0.0, R, U)
    assert np.abs(R).max() <= 1e-13


def test_bounded_euler_needs_table_and_generic_kernel():
    pr = P.euler2d(n=4, k=1, seed=86, periodic=(False, True))
    with pr.evaluator() as ev:
        with pytest.raises(C.BosssError) as ei:
            ev.Evaluate(1.0, 0.0, np.zeros(pr.n_dofs), pr.U)
        assert ei.value.code == C.ERR_BAD_ARG
    pr3 = P.euler3d(n=3, k=1, seed=87, periodic=(False, True, True))
    for kern in (C.KERNEL_SLAB, C.KERNEL_FACES):
        with pytest.raises(C.BosssError) as ei:
            pr3.evaluator(kernel=kern)
        assert ei.value.code == C.ERR_BAD_ARG


@pytest.mark.parametrize("name,make", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_boundary_kinds_match_oracle(name, make):
    """Outlet (inner state) and slip-wall (normal momentum reflected) nodes mixed with
    prescribed ones: residual, JVP and VJP against the oracle."""
    import test_oracle_euler_boundary as TB
    pr = make()
    opd, gd = pr.descs()
    r = np.random.default_rng(11)
    V = r.uniform(-1, 1, pr.n_dofs)
    W = r.uniform(-1, 1, pr.n_dofs)
    nq = orc.sizes(opd, gd)[2]
    kinds = TB.boundary_kinds_by_face(gd, nq, lambda d, s: (d + s) % 3)
    with pr.evaluator() as ev:
        bnd = P.euler_boundary_states(ev.boundary_nodes())
        ev.SetBoundaryState(bnd)
        ev.SetBoundaryKinds(kinds)
        R = np.zeros(pr.n_dofs)
        ev.Evaluate(1.0, 0.0, R, pr.U)
        JV = ev.jvp(pr.U, V)
        G = ev.vjp(pr.U, W)
    with orc.boundary_kinds(kinds):
        assert rel(R, orc.evaluate(opd, gd, pr.U, bnd=bnd)) <= TOL
        assert rel(JV, orc.jvp(opd, gd, pr.U, V, bnd=bnd)) <= TOL
        assert rel(G, orc.vjp(opd, gd, pr.U, W, bnd=bnd)) <= TOL


def test_walls_and_outlets_need_no_table():
    pr = P.euler2d(n=4, k=1, seed=88, periodic=(False, False))
    opd, gd = pr.descs()
    with pr.evaluator() as ev:
        n = len(ev.boundary_nodes())
        ev.SetBoundaryKinds(np.full(n, 2, dtype=np.int32))
        R = np.zeros(pr.n_dofs)
        ev.Evaluate(1.0, 0.0, R, pr.U)
        with pytest.raises(C.BosssError):
            ev.SetBoundaryKinds(np.full(n, 3, dtype=np.int32))
    with orc.boundary_kinds(np.full(n, 2, dtype=np.int32)):
        assert rel(R, orc.evaluate(opd, gd, pr.U)) <= TOL
