"""Pins of the CPU oracle against the reference's own data and known answers.

* operator output: the oracle reproduces the reference's stored ``Evaluate`` results of
  the CNS SIPG consistency test (``CNS/Tests/DiffusiveFlux/SIPGConsistencyRefSolution_p{1,2,3}.txt``,
  fixtures ``tests/golden/sipg_consistency_p*.json``) DOF by DOF within the reference's
  own threshold 1e-11 (``SIPGConsistency.cs:87-160``); perturbed physics misses them;
* basis tables: the oracle's orthonormal polynomials equal the reference's
  ``Square.cs`` / ``Cube_polynomials.cs`` tables (fixtures extracted by
  ``tests/golden/make_golden.py``), coefficient by coefficient and in the same order;
* Gauss rules: equal to the reference's ``LineQuadRules_bin.txt`` resource;
* DerivativeTest-style known answers (``DerivativeTestMain.cs:880-1160``):
  orthonormality (mass matrix = I), consistency of the upwind transport operator
  and of the SIP Laplacian (constant and nonlinear viscosity) on polynomial
  fields, free-stream preservation of the HLLC Euler operator;
* exact JVP against central finite differences (eps = 1e-6), the assembled
  Jacobian against the JVP, and the adjoint product (VJP) against the transposed
  assembled Jacobian.
"""
import json
import os

import numpy as np
import pytest
from numpy.polynomial import legendre as npleg

from bosss_b200 import operator as O
from bosss_b200 import problems as P
from oracle import oracle as orc

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("p", [1, 2, 3])
def test_oracle_reproduces_reference_sipg_consistency_output(p):
    import cns_sipg_case as S
    opd, gd, U, bnd = S.case(p)
    R = orc.evaluate(opd, gd, U, bnd=bnd)
    ref = S.reference_values(p)
    assert R.shape == ref.shape == (9 * 4 * (p + 1) * (p + 2) // 2,)
    # the reference's check: |refSol[i] - output[i]| < 1e-11 for every DOF
    assert np.abs(R - ref).max() < 1e-11
    # the density rows are zero (OptimizedSIPGDensityFlux has no terms)
    Np = (p + 1) * (p + 2) // 2
    assert np.all(R.reshape(9, 4, Np)[:, 0, :] == 0.0)


@pytest.mark.parametrize("i,value", [(6, 0.3), (7, 1.001), (4, 0.01)])
def test_reference_sipg_output_pins_the_physics(i, value):
    """Perturbing the Sutherland ratio, the penalty scaling or the bulk viscosity ratio
    moves the oracle off the reference's stored values: the pin is not vacuous."""
    import cns_sipg_case as S
    p = 2
    params = [S.GAMMA, S.MACH, 1.0, 1.0, 0.0, 1.0, S.SUTHERLAND, 1.0]
    params[i] = value
    opd, gd, U, bnd = S.case(p)
    opd2 = S.op_desc(p, params)
    R = orc.evaluate(opd2, gd, U, bnd=bnd)
    assert np.abs(R - S.reference_values(p)).max() > 1e-6


def test_oracle_sipg_vjp_is_transposed_jacobian():
    import cns_sipg_case as S
    opd, gd, U, bnd = S.case(2)
    W = np.random.default_rng(4).uniform(-1, 1, U.size)
    nd = U.size
    # Jacobian columns by exact JVPs (small case)
    A = np.stack([orc.jvp(opd, gd, U, np.eye(nd)[i], bnd=bnd) for i in range(nd)], axis=1)
    g = orc.vjp(opd, gd, U, W, bnd=bnd)
    assert np.linalg.norm(g - A.T @ W) <= 1e-12 * np.linalg.norm(A.T @ W)


def _load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


@pytest.mark.parametrize("dim,fname", [(2, "ref_basis_2d.json"), (3, "ref_basis_3d.json")])
def test_basis_matches_reference_tables(dim, fname):
    ref = _load(fname)["polys"]
    mine = orc.basis_monomials(dim, 5)
    assert len(mine) == len(ref)
    for i, (p, r) in enumerate(zip(mine, ref)):
        assert r["index"] == i
        rt = {tuple(e): c for c, e in r["terms"]}
        mt = {tuple(int(x) for x in e): c for c, e in p}
        assert set(rt) == set(mt), (i, rt, mt)
        for e in rt:
            # the reference stores 15-17 significant digits
            assert abs(rt[e] - mt[e]) <= 2e-14 * max(1.0, abs(rt[e])), (i, e, rt[e], mt[e])


def test_gauss_rules_match_reference():
    for r in _load("ref_gauss_rules.json")["rules"]:
        n = len(r["nodes"])
        assert r["order"] == 2 * n - 1
        x, w = orc.gauss_rule(n)
        assert np.max(np.abs(x - np.array(r["nodes"]))) < 1e-14
        assert np.max(np.abs(w - np.array(r["weights"]))) < 1e-14


@pytest.mark.parametrize("dim,k", [(2, 3), (3, 4)])
def test_orthonormal_mass_matrix(dim, k):
    nq = k + 1
    x, w = orc.gauss_rule(nq)
    grids = np.meshgrid(*([x] * dim), indexing="ij")
    pts = np.stack([g.ravel() for g in grids], axis=1)
    W = np.ones(len(pts))
    for d, g in enumerate(np.meshgrid(*([w] * dim), indexing="ij")):
        W *= g.ravel()
    phi, _ = orc.basis_eval(dim, k, pts)
    M = (phi * W) @ phi.T
    assert np.max(np.abs(M - np.eye(len(M)))) < 1e-13


def _project_function(grid, k, f, nq=8):
    """L2 projection (high-order quadrature) of f(x) onto the orthonormal basis."""
    dim = grid.dim
    phi, W, xi = P.volume_basis(dim, k, nq)
    ijk = grid.cell_ijk()
    h = [(grid.hi[d] - grid.lo[d]) / grid.n[d] for d in range(dim)]
    detJ = np.prod([0.5 * hd for hd in h])
    X = [grid.lo[d] + (ijk[:, d:d + 1] + 0.5 + 0.5 * xi[None, :, d]) * h[d] for d in range(dim)]
    vals = f(*X)
    return ((vals * W[None, :]) @ phi * (detJ / np.sqrt(detJ))).ravel()


def test_transport_consistency_2d():
    """Upwind transport of a global polynomial u in P_k: R_n = int (a . grad u) phi_n."""
    k = 2
    g = O.Cartesian2DGrid(np.linspace(0, 1, 5), np.linspace(0, 2, 4), False, False)
    a = (1.0, -0.5)
    op = O.DifferentialOperator(["u"], [], ["R"], O.QuadOrderFunc.FixedOrder(2 * k + 1))
    op.EquationComponents["R"].Add(O.ScalarTransportFlux(a, "u"))
    op.Commit()
    u = lambda x, y: 1 + 2 * x - y + 0.5 * x * x + x * y - 0.3 * y * y
    adu = lambda x, y: a[0] * (2 + x + y) + a[1] * (-1 + x - 0.6 * y)
    U = _project_function(g, k, u)
    opd, gd = op.descriptor([k], [k], 2), g.desc()
    R = orc.evaluate(opd, gd, U)
    Rex = _project_function(g, k, adu)
    assert np.max(np.abs(R - Rex)) < 1e-12 * max(1, np.max(np.abs(Rex)))


@pytest.mark.parametrize("nu2", [0.0, 1.0])
def test_sip_consistency_3d(nu2):
    """SIP with g_D = u on the boundary, u = c0 + c1.x + c2.x^2:
    R_n = int div(nu(u) grad u) phi_n (DerivativeTest Laplace check)."""
    k = 2
    g = O.Cartesian3DGrid(np.linspace(0, 1, 4), np.linspace(0, 1, 3), np.linspace(-1, 1, 4), False, False, False)
    c0, c1, c2 = 0.3, np.array([1.0, -0.5, 0.25]), np.array([0.7, -0.4, 0.2])
    op = O.DifferentialOperator(["u"], [], ["R"], O.QuadOrderFunc.NonLinear(3))
    op.EquationComponents["R"].Add(O.SIPLaplace(4.0, "u", nu0=1.0, nu2=nu2, dirichlet=True, g0=c0, g1=c1, g2=c2))
    op.Commit()
    u = lambda x, y, z: c0 + c1[0] * x + c1[1] * y + c1[2] * z + c2[0] * x * x + c2[1] * y * y + c2[2] * z * z

    def div_flux(x, y, z):
        uu = u(x, y, z)
        gr = [c1[0] + 2 * c2[0] * x, c1[1] + 2 * c2[1] * y, c1[2] + 2 * c2[2] * z]
        lap = 2 * (c2[0] + c2[1] + c2[2])
        nu = 1.0 + nu2 * uu * uu
        dnu = 2 * nu2 * uu
        return nu * lap + dnu * (gr[0] ** 2 + gr[1] ** 2 + gr[2] ** 2)

    U = _project_function(g, k, u)
    R = orc.evaluate(*(op.descriptor([k], [k], 3), g.desc()), U)
    if nu2 == 0.0:
        Rex = _project_function(g, k, div_flux)
        # penalty terms of size ~pen*u cancel; the reference checks this at 1e-8
        assert np.max(np.abs(R - Rex)) < 1e-9 * max(1, np.max(np.abs(Rex)))
    else:
        # nu(u) grad u is degree 5 > k: the DG residual equals the projection of the
        # divergence only up to the projection of the interior jumps (none: u is smooth);
        # compare with the projection of div(nu grad u), which is exact here
        Rex = _project_function(g, k, div_flux)
        assert np.max(np.abs(R - Rex)) < 1e-9 * max(1, np.max(np.abs(Rex)))


def test_euler_free_stream():
    pr = P.euler3d(n=3, k=2, seed=7)
    J = pr.grid.NoOfCells
    Np = pr.dom[0].Np
    U = np.zeros((J, 5 * Np))
    detJ = (1.0 / 3 / 2) ** 3
    const = np.array([1.2, 0.3, -0.2, 0.1, 2.9])
    for f in range(5):
        U[:, f * Np] = const[f] * np.sqrt(8 * detJ)   # phi_0 = 1/sqrt(vol)
    R = orc.evaluate(*pr.descs(), U.ravel())
    assert np.max(np.abs(R)) < 1e-12


CASES = [
    ("transport2d", lambda: P.transport2d(n=4, k=2, seed=11)),
    ("euler3d", lambda: P.euler3d(n=3, k=1, seed=12)),
    ("sip3d", lambda: P.nonlinear_diffusion3d(n=3, k=2, seed=13)),
    ("advdiff3d", lambda: P.advection_diffusion3d(n=3, k=2, seed=14)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_oracle_jvp_matches_central_fd(name, make):
    pr = make()
    opd, gd = pr.descs()
    r = np.random.default_rng(5)
    V = r.uniform(-1, 1, pr.n_dofs)
    jv = orc.jvp(opd, gd, pr.U, V)
    eps = 1e-6
    fd = (orc.evaluate(opd, gd, pr.U + eps * V) - orc.evaluate(opd, gd, pr.U - eps * V)) / (2 * eps)
    rel = np.linalg.norm(jv - fd) / np.linalg.norm(jv)
    assert rel < 1e-7, rel


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_oracle_jacobian_matches_jvp(name, make):
    pr = make()
    opd, gd = pr.descs()
    A = orc.jacobian_dense(opd, gd, pr.U)
    V = np.random.default_rng(6).uniform(-1, 1, pr.n_dofs)
    jv = orc.jvp(opd, gd, pr.U, V)
    assert np.linalg.norm(A @ V - jv) <= 1e-13 * np.linalg.norm(jv)


@pytest.mark.parametrize("name,make", [
    ("transport2d_bnd", lambda: P.transport2d(n=4, k=2, seed=7, periodic=False)),
    ("euler3d", lambda: P.euler3d(n=3, k=1, seed=5)),
    ("sip3d", lambda: P.nonlinear_diffusion3d(n=3, k=2, seed=6)),
    ("advdiff3d", lambda: P.advection_diffusion3d(n=3, k=2, seed=8)),
])
def test_oracle_vjp_matches_transposed_jacobian(name, make):
    pr = make()
    opd, gd = pr.descs()
    nd, nc, _ = orc.sizes(opd, gd)
    W = np.random.default_rng(1).uniform(-1, 1, nc)
    ref = orc.jacobian_dense(opd, gd, pr.U).T @ W
    assert np.linalg.norm(orc.vjp(opd, gd, pr.U, W) - ref) <= 1e-13 * np.linalg.norm(ref)
