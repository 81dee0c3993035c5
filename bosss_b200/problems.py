"""Seeded synthetic problems of the benchmark configurations.

No public dataset is involved: every input is drawn from
``numpy.random.Generator(PCG64(seed))`` with the distributions of the workload
definitions below, and every builder returns the operator, the fields and the
FP64 coefficient vector in the reference's cell-major layout.

* :func:`transport2d`  -- 2D scalar linear advection, upwind, periodic [0,1]^2,
  64x64 cells, k=2 (Np=6), Gauss order 2k+1, coefficients iid U[-1,1].
* :func:`euler3d`      -- 3D compressible Euler with HLLC, periodic [0,1]^3, 32^3
  hexes, k=3 (Np=20 per variable), order 7 (= 2k+1), gamma=1.4, Ma=1/sqrt(gamma); primitive
  state rho=1+0.1U, u_d=0.3U, p=1+0.1U sampled at the volume nodes and
  L2-projected onto the basis.
* :func:`nonlinear_diffusion3d` -- -div((1+u^2) grad u) with SIP (penalty base 4,
  degree factor (k+1)^2, cell length scale as in the reference), Dirichlet g=0,
  [0,1]^3, 48^3 hexes, k=2..4, order 4k (NonLinear(3)); u sampled iid U[-1,1] at the
  (k+1)^3 Gauss nodes of every cell and L2-projected (iid coefficients of the
  orthonormal basis would give physical values ~ (2/h)^1.5, i.e. nu(u) ~ 1e6).
* :func:`advection_diffusion3d` -- upwind transport (a ~ U[-1,1]^3) + SIP with
  nu=0.01, periodic, order 2k (Linear()).
"""
import numpy as np
from numpy.polynomial import legendre as npleg

from . import operator as O


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


class Problem:
    def __init__(self, name, op, grid, dom, cod, U, config):
        self.name, self.op, self.grid, self.dom, self.cod, self.U, self.config = name, op, grid, dom, cod, U, config

    def descs(self):
        """(OpDesc, GridDesc) of the C-ABI -- also what the oracle consumes."""
        return (self.op.descriptor([f.degree for f in self.dom], [f.degree for f in self.cod], self.grid.dim),
                self.grid.desc())

    def evaluator(self, **kw):
        return self.op.GetEvaluatorEx(self.dom, None, self.cod, **kw)

    @property
    def n_dofs(self):
        return len(self.U)


def _linspace_nodes(n, lo=0.0, hi=1.0):
    return np.linspace(lo, hi, n + 1)


def transport2d(n=64, k=2, seed=1000, velocity=(1.0, 0.5), periodic=True):
    g = O.Cartesian2DGrid(_linspace_nodes(n), _linspace_nodes(n), periodic, periodic)
    op = O.DifferentialOperator(["u"], [], ["R"], O.QuadOrderFunc.FixedOrder(2 * k + 1))
    op.EquationComponents["R"].Add(O.ScalarTransportFlux(velocity, "u"))
    op.Commit()
    u = O.DGField(g, k, "u")
    r = O.DGField(g, k, "R")
    U = rng(seed).uniform(-1.0, 1.0, g.NoOfCells * u.Np)
    return Problem("transport2d", op, g, [u], [r], U,
                   {"workload": "transport2d_upwind_%dx%d_k%d" % (n, n, k), "cells": g.NoOfCells, "k": k,
                    "seed": seed})


def _legendre_table(k, x):
    """L_a(x) = sqrt((2a+1)/2) P_a(x), shape (len(x), k+1)."""
    T = np.empty((len(x), k + 1))
    for a in range(k + 1):
        c = np.zeros(a + 1)
        c[a] = 1.0
        T[:, a] = np.sqrt((2 * a + 1) / 2.0) * npleg.legval(x, c)
    return T


def basis_modes(dim, k):
    """Exponent tuples in the reference polynomial order."""
    m = []
    for deg in range(k + 1):
        if dim == 2:
            m += [(a, deg - a) for a in range(deg + 1)]
        else:
            m += [(a, b, deg - a - b) for a in range(deg + 1) for b in range(deg - a + 1)]
    return m


def volume_basis(dim, k, nq):
    """Reference basis at the tensor Gauss nodes (reference node order), weights:
    returns (phi[Q, Np], W[Q], xi[Q, dim])."""
    x, w = npleg.leggauss(nq)
    L = _legendre_table(k, x)
    modes = basis_modes(dim, k)
    if dim == 2:
        qy, qx = np.meshgrid(np.arange(nq), np.arange(nq), indexing="ij")
        qi = [qx.ravel(), qy.ravel()]
    else:
        qz, qy, qx = np.meshgrid(np.arange(nq), np.arange(nq), np.arange(nq), indexing="ij")
        qi = [qx.ravel(), qy.ravel(), qz.ravel()]
    phi = np.ones((len(qi[0]), len(modes)))
    for n, e in enumerate(modes):
        for d in range(dim):
            phi[:, n] *= L[qi[d], e[d]]
    W = np.ones(len(qi[0]))
    for d in range(dim):
        W *= w[qi[d]]
    xi = np.stack([x[qi[d]] for d in range(dim)], axis=1)
    return phi, W, xi


def project_nodal(dim, k, nq, h, nodal):
    """L2 projection of nodal values nodal[J, Q] onto the orthonormal basis
    (coefficients of phi_n = phi_ref_n / sqrt(detJ))."""
    phi, W, _ = volume_basis(dim, k, nq)
    detJ = np.prod([0.5 * hd for hd in h])
    scaling = 1.0 / np.sqrt(detJ)
    return (nodal * W[None, :]) @ phi * (detJ * scaling)


def euler3d(n=32, k=3, seed=2000, gamma=1.4, quad_order=None, nx=None, periodic=(True, True, True)):
    """``nx``: cells along x (default n) on [0, nx/n] -- the same cell size, an elongated
    periodic box (the global grid of an x-slab partition with n planes per part).
    ``periodic``: per direction; boundary faces need the boundary-state table
    (:func:`euler_boundary_states`)."""
    quad_order = 2 * k + 1 if quad_order is None else quad_order
    nx = n if nx is None else nx
    g = O.Cartesian3DGrid(np.linspace(0.0, nx / n, nx + 1), _linspace_nodes(n), _linspace_nodes(n), *periodic)
    names = ["rho", "m0", "m1", "m2", "rhoE"]
    op = O.DifferentialOperator(names, [], ["R_" + s for s in names], O.QuadOrderFunc.FixedOrder(quad_order))
    mat = O.Material(gamma)
    op.EquationComponents["R_rho"].Add(O.OptimizedHLLCDensityFlux(mat, 3))
    for d in range(3):
        op.EquationComponents["R_m%d" % d].Add(O.OptimizedHLLCMomentumFlux(mat, d, 3))
    op.EquationComponents["R_rhoE"].Add(O.OptimizedHLLCEnergyFlux(mat, 3))
    op.Commit()
    dom = [O.DGField(g, k, s) for s in names]
    cod = [O.DGField(g, k, "R_" + s) for s in names]
    nq = (quad_order + 2) // 2
    J = g.NoOfCells
    Q = nq ** 3
    r = rng(seed)
    rho = 1.0 + 0.1 * r.uniform(-1, 1, (J, Q))
    vel = 0.3 * r.uniform(-1, 1, (3, J, Q))
    p = 1.0 + 0.1 * r.uniform(-1, 1, (J, Q))
    gMs = gamma * mat.Mach ** 2
    E = p / (gamma - 1.0) + 0.5 * gMs * rho * (vel ** 2).sum(axis=0)
    h = [1.0 / n] * 3
    Np = dom[0].Np
    U = np.empty((J, 5 * Np))
    fields = [rho, rho * vel[0], rho * vel[1], rho * vel[2], E]
    for f, val in enumerate(fields):
        U[:, f * Np:(f + 1) * Np] = project_nodal(3, k, nq, h, val)
    return Problem("euler3d", op, g, dom, cod, U.ravel(),
                   {"workload": ("euler3d_hllc_%d^3_k%d" % (n, k)) if nx == n else
                    ("euler3d_hllc_%dx%d^2_k%d" % (nx, n, k)), "cells": J, "k": k, "seed": seed,
                    "gamma": gamma, "quad_order": quad_order})


def euler2d(n=16, k=2, seed=2500, gamma=1.4, quad_order=None, periodic=(True, True)):
    """2D Euler / HLLC on [0,1]^2 with the seeded state of :func:`euler3d` (two velocity
    components)."""
    quad_order = 2 * k + 1 if quad_order is None else quad_order
    g = O.Cartesian2DGrid(_linspace_nodes(n), _linspace_nodes(n), *periodic)
    names = ["rho", "m0", "m1", "rhoE"]
    op = O.DifferentialOperator(names, [], ["R_" + s for s in names], O.QuadOrderFunc.FixedOrder(quad_order))
    mat = O.Material(gamma)
    op.EquationComponents["R_rho"].Add(O.OptimizedHLLCDensityFlux(mat, 2))
    for d in range(2):
        op.EquationComponents["R_m%d" % d].Add(O.OptimizedHLLCMomentumFlux(mat, d, 2))
    op.EquationComponents["R_rhoE"].Add(O.OptimizedHLLCEnergyFlux(mat, 2))
    op.Commit()
    dom = [O.DGField(g, k, s) for s in names]
    cod = [O.DGField(g, k, "R_" + s) for s in names]
    nq = (quad_order + 2) // 2
    J = g.NoOfCells
    Q = nq ** 2
    r = rng(seed)
    rho = 1.0 + 0.1 * r.uniform(-1, 1, (J, Q))
    vel = 0.3 * r.uniform(-1, 1, (2, J, Q))
    p = 1.0 + 0.1 * r.uniform(-1, 1, (J, Q))
    gMs = gamma * mat.Mach ** 2
    E = p / (gamma - 1.0) + 0.5 * gMs * rho * (vel ** 2).sum(axis=0)
    Np = dom[0].Np
    U = np.empty((J, 4 * Np))
    for f, val in enumerate([rho, rho * vel[0], rho * vel[1], E]):
        U[:, f * Np:(f + 1) * Np] = project_nodal(2, k, nq, [1.0 / n] * 2, val)
    return Problem("euler2d", op, g, dom, cod, U.ravel(),
                   {"workload": "euler2d_hllc_%d^2_k%d" % (n, k), "cells": J, "k": k, "seed": seed,
                    "gamma": gamma, "quad_order": quad_order})


def euler_boundary_states(xyz, gamma=1.4, mach=None):
    """Conservative outer states at boundary face nodes (rows of ``xyz``): a smooth prescribed
    inflow field, rho = 1 + 0.1 sin(2 pi x), u_d = 0.3 cos(2 pi (x_d + d / 4)),
    p = 1 + 0.1 cos(2 pi sum x) -- what a far-field / supersonic-inlet map returns."""
    xyz = np.atleast_2d(xyz)
    D = xyz.shape[1]
    mach = 1.0 / np.sqrt(gamma) if mach is None else mach
    rho = 1.0 + 0.1 * np.sin(2 * np.pi * xyz[:, 0])
    vel = np.stack([0.3 * np.cos(2 * np.pi * (xyz[:, d] + d / 4.0)) for d in range(D)])
    p = 1.0 + 0.1 * np.cos(2 * np.pi * xyz.sum(axis=1))
    E = p / (gamma - 1.0) + 0.5 * gamma * mach ** 2 * rho * (vel ** 2).sum(axis=0)
    return np.stack([rho] + [rho * vel[d] for d in range(D)] + [E], axis=1)


def nonlinear_diffusion3d(n=48, k=2, seed=3000, penalty_base=4.0, source=0.0):
    g = O.Cartesian3DGrid(_linspace_nodes(n), _linspace_nodes(n), _linspace_nodes(n), False, False, False)
    op = O.DifferentialOperator(["u"], [], ["R"], O.QuadOrderFunc.NonLinear(3))
    op.EquationComponents["R"].Add(O.SIPLaplace(penalty_base, "u", nu0=1.0, nu2=1.0, dirichlet=True))
    if source:
        op.EquationComponents["R"].Add(O.ConstantSource(source, "u"))
    op.Commit()
    u = O.DGField(g, k, "u")
    r_ = O.DGField(g, k, "R")
    nq = k + 1
    nodal = rng(seed).uniform(-1.0, 1.0, (g.NoOfCells, nq ** 3))
    U = project_nodal(3, k, nq, [1.0 / n] * 3, nodal).ravel()
    return Problem("nonlinear_diffusion3d", op, g, [u], [r_], U,
                   {"workload": "sip_nonlinear_%d^3_k%d" % (n, k), "cells": g.NoOfCells, "k": k, "seed": seed})


def advection_diffusion3d(n=16, k=2, seed=5000, nu=0.01, penalty_base=4.0, velocity=None, periodic=True):
    """Upwind transport with a ~ U[-1,1]^3 plus SIPLaplace(nu). SIPLaplace discretises
    +nu Laplace(u) (its volume form is -nu grad u . grad v, ipLaplace.cs:183-186), so the
    operator is div(a u) + nu Laplace(u): nu < 0 gives the dissipative advection-diffusion
    operator of du/dt = -Op(u)."""
    r = rng(seed)
    a = r.uniform(-1, 1, 3) if velocity is None else np.asarray(velocity, dtype=float)
    g = O.Cartesian3DGrid(_linspace_nodes(n), _linspace_nodes(n), _linspace_nodes(n), periodic, periodic, periodic)
    op = O.DifferentialOperator(["u"], [], ["R"], O.QuadOrderFunc.Linear())
    op.EquationComponents["R"].Add(O.ScalarTransportFlux(a, "u"))
    op.EquationComponents["R"].Add(O.SIPLaplace(penalty_base, "u", nu0=nu, nu2=0.0, dirichlet=True))
    op.Commit()
    u = O.DGField(g, k, "u")
    r_ = O.DGField(g, k, "R")
    U = r.uniform(-1.0, 1.0, g.NoOfCells * u.Np)
    return Problem("advection_diffusion3d", op, g, [u], [r_], U,
                   {"workload": "advdiff_%d^3_k%d" % (n, k), "cells": g.NoOfCells, "k": k, "seed": seed,
                    "velocity": list(map(float, a)), "nu": nu})


def batched_advection_diffusion(n_instances=256, seed=5000, sizes=(16, 24, 32, 48), degrees=(1, 2, 3, 4), nu=0.01):
    """The batched mixed workload: independent advection-diffusion instances with grid
    sizes drawn from ``sizes``^3 and DG degrees from ``degrees`` (seeded), each with its
    own velocity a ~ U[-1,1]^3 and FP64 coefficients U[-1,1]; periodic, Linear() order."""
    r = rng(seed)
    ns = r.choice(sizes, n_instances)
    ks = r.choice(degrees, n_instances)
    return [advection_diffusion3d(n=int(n), k=int(k), seed=seed * 1000 + i, nu=nu)
            for i, (n, k) in enumerate(zip(ns, ks))]


def xdg_poisson3d(n=128, k=2, seed=4000, muA=1.0, muB=10.0, radius=0.4, penalty_base=4.0):
    """XDG two-phase Poisson with jump, bulk part: -div(mu grad u) = 1 on [-1,1]^3, n^3 hexes,
    phi = |x - c| - radius with c ~ 0.05 U[-1,1]^3 (seeded), mu = muA inside, muB outside,
    Dirichlet 0, uncut cells with the Gauss rule of order 5. Returns (opA, opB, grid, center,
    UA, UB) with species frames UA, UB (coefficients iid U[-1,1])."""
    r = rng(seed)
    c = 0.05 * r.uniform(-1, 1, 3)
    nodes = np.linspace(-1.0, 1.0, n + 1)
    g = O.Cartesian3DGrid(nodes, nodes, nodes, False, False, False)
    ops = []
    for mu in (muA, muB):
        op = O.DifferentialOperator(["u"], [], ["R"], O.QuadOrderFunc.FixedOrder(5))
        op.EquationComponents["R"].Add(O.SIPLaplace(penalty_base, "u", nu0=mu, nu2=0.0, dirichlet=True))
        op.EquationComponents["R"].Add(O.ConstantSource(1.0, "u"))
        op.Commit()
        ops.append(op)
    Np = O.np_of(3, k)
    UA = r.uniform(-1, 1, g.NoOfCells * Np)
    UB = r.uniform(-1, 1, g.NoOfCells * Np)
    return ops[0], ops[1], g, c, UA, UB


def hex_block_pattern(n, np_cell, seed=3000, periodic=False):
    """Block-sparse pattern of a DG operator on an n^3 hex grid (generator cell order): each
    block row (cell) holds its own block and one per face neighbour (7 blocks inside, fewer at
    non-periodic boundaries), blocks np_cell x np_cell with seeded values U[-1, 1] -- the
    shape of the C3 Jacobian (48^3, k = 2: 110,592 block rows x 7 blocks of 10 x 10).
    Returns (row_ptr, col_idx, values[nnz, np_cell, np_cell])."""
    J = n ** 3
    idx = np.arange(J)
    i, j, k = idx // (n * n), (idx // n) % n, idx % n
    cols = [idx]
    valid = [np.ones(J, dtype=bool)]
    for d, (a, st) in enumerate(((i, n * n), (j, n), (k, 1))):
        for s in (-1, 1):
            a2 = a + s
            ok = (a2 >= 0) & (a2 < n)
            if periodic:
                a2 = a2 % n
                ok = np.ones(J, dtype=bool)
            cols.append(idx + (a2 - a) * st)
            valid.append(ok)
    C = np.stack(cols, axis=1)
    V = np.stack(valid, axis=1)
    order = np.argsort(np.where(V, C, J + 1), axis=1, kind="stable")
    C = np.take_along_axis(C, order, axis=1)
    V = np.take_along_axis(V, order, axis=1)
    counts = V.sum(axis=1)
    row_ptr = np.zeros(J + 1, dtype=np.int64)
    row_ptr[1:] = np.cumsum(counts)
    col_idx = C[V].astype(np.int32)
    vals = rng(seed).uniform(-1.0, 1.0, (len(col_idx), np_cell, np_cell))
    return row_ptr, col_idx, vals
