"""The reference's CNS SIPG consistency case, restated for the oracle (test helper).

``src/L4-application/CNS/Tests/DiffusiveFlux/SIPGConsistency.cs:165-225`` sets up a 3x3
Cartesian grid on [0, 2 pi]^2 (not periodic, every boundary edge tagged
"supersonicinlet"), an ideal gas with gamma = 2, Mach = 1/sqrt(gamma) (so MachScaling =
1), Reynolds = Prandtl = 1, Sutherland's viscosity law (S/T0 = 110.4/273.15,
``SutherlandLaw.cs``), the OptimizedSIPG viscous fluxes with penalty scaling 1, DG degree p
for all four conservative variables, and the primitive initial / boundary values

    rho = 0.1 sin x + 0.1 cos y + 1,   u = sin x + cos y + 1,
    v   = cos x + sin y + 1,            p = cos x + sin x + 4.

``RunSolverOneStep`` (``:49-52``) evaluates the diffusive operator once,
``Evaluate(1.0, 0.0, ...)``, and ``SIPGconsistencyTest`` compares every DOF with the stored
``SIPGConsistencyRefSolution_p{p}.txt`` to 1e-11 (``:87-160``).

Restated here:

* the conservative initial fields are L2 projections of rho, rho u, rho v and
  E = p/(gamma-1) + MachScaling rho |u|^2 / 2 (``CNSFieldSet.ProjectInitialValues``,
  ``CNSFieldSet.cs:196-239``; ``StateVector.FromPrimitiveQuantities``, ``StateVector.cs:111-123``)
  with the quadrature order 2p + 2 of ``DGField.ProjectField`` (``DGField.cs:263-278``),
  i.e. p + 2 Gauss nodes per direction;
* the operator has the quadrature order ``QuadOrderFunc.NonLinearWithoutParameters(2)``
  (``CNS/EquationSystem/Operator.cs:143-152``): 3p;
* the supersonic-inlet boundary state is the conservative state of the primitive boundary
  values at each boundary face node (``SupersonicInlet.GetBoundaryState``), passed to the
  oracle as its boundary-state table;
* the DOF order of the stored vectors is the local cell order of ``Grid2D.Cartesian2DGrid``
  (x index outer, y inner, ``Grid2D.cs:566-586``), which is the generator order here.
"""
import json
import math
import os

import numpy as np

from bosss_b200 import _capi as C
from oracle import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
GAMMA = 2.0
MACH = 1.0 / math.sqrt(GAMMA)
SUTHERLAND = 110.4 / 273.15
N_CELLS = 3

# component ids of the OptimizedSIPG{Density,Momentum,Energy}Flux (C-ABI and oracle)
COMP_CNS_SIPG_DENSITY = C.COMP_CNS_SIPG_DENSITY_FLUX
COMP_CNS_SIPG_MOMENTUM = C.COMP_CNS_SIPG_MOMENTUM_FLUX
COMP_CNS_SIPG_ENERGY = C.COMP_CNS_SIPG_ENERGY_FLUX


def primitive(x, y):
    rho = 0.1 * np.sin(x) + 0.1 * np.cos(y) + 1.0
    u = np.sin(x) + np.cos(y) + 1.0
    v = np.cos(x) + np.sin(y) + 1.0
    p = np.cos(x) + np.sin(x) + 4.0
    return rho, u, v, p


def conservative(x, y):
    rho, u, v, p = primitive(x, y)
    ms = GAMMA * MACH * MACH
    E = p / (GAMMA - 1.0) + 0.5 * ms * rho * (u * u + v * v)
    return np.stack([rho, rho * u, rho * v, E], axis=-1)


def grid_desc(n=N_CELLS):
    g = C.GridDesc()
    g.dim = 2
    for d in range(3):
        g.n[d] = n if d < 2 else 1
        g.lo[d] = 0.0
        g.hi[d] = 2.0 * math.pi if d < 2 else 1.0
        g.periodic[d] = 0
    g.cell_order = C.CELLS_GENERATOR
    return g


def op_desc(p, params=None):
    """The diffusive operator of the CNS solver: OptimizedSIPG fluxes on (rho, m0, m1, rhoE)."""
    d = C.OpDesc()
    d.n_domain = d.n_codomain = 4
    for i in range(4):
        d.domain_degree[i] = d.codomain_degree[i] = p
    d.quad_kind, d.quad_param = C.QUAD_NONLINEAR, 2
    base = params or [GAMMA, MACH, 1.0, 1.0, 0.0, 1.0, SUTHERLAND, 1.0]
    types = [(COMP_CNS_SIPG_DENSITY, 0), (COMP_CNS_SIPG_MOMENTUM, 0), (COMP_CNS_SIPG_MOMENTUM, 1),
             (COMP_CNS_SIPG_ENERGY, 0)]
    for c, (t, comp) in enumerate(types):
        cp = d.components[c]
        cp.type, cp.codomain, cp.n_args = t, c, 4
        for a in range(4):
            cp.args[a] = a
        for i, v in enumerate(base):
            cp.params[i] = v
        cp.params[8] = float(comp)
    d.n_components = 4
    return d


def cell_centers(gd):
    n = [gd.n[0], gd.n[1]]
    h = [(gd.hi[d] - gd.lo[d]) / n[d] for d in range(2)]
    ix, iy = np.unravel_index(np.arange(n[0] * n[1]), n)   # generator order: x outer
    return np.stack([gd.lo[0] + (ix + 0.5) * h[0], gd.lo[1] + (iy + 0.5) * h[1]], axis=1), h


def project(gd, p, fun):
    """L2 projection of fun(x, y) -> (..., nvar) onto the orthonormal basis of degree p with
    (p + 2)^2 Gauss nodes; returns the cell-major coefficient vector [cell][var][mode]."""
    nq = p + 2
    x1, w1 = orc.gauss_rule(nq)
    # Square.cs:110-127 ordering: node (x_j, y_i) at i*nq + j
    X, Y = np.meshgrid(x1, x1)              # X[i, j] = x_j, Y[i, j] = y_i
    pts = np.stack([X.ravel(), Y.ravel()], axis=1)
    wts = np.outer(w1, w1).ravel()
    phi, _ = orc.basis_eval(2, p, pts)      # [mode, node]
    cen, h = cell_centers(gd)
    detJ = 0.25 * h[0] * h[1]
    scaling = 1.0 / math.sqrt(detJ)
    J = len(cen)
    out = []
    for j in range(J):
        xs = cen[j, 0] + 0.5 * h[0] * pts[:, 0]
        ys = cen[j, 1] + 0.5 * h[1] * pts[:, 1]
        f = fun(xs, ys)                     # [node, var]
        coef = (phi * (wts * detJ * scaling)) @ f   # [mode, var]
        out.append(coef.T.ravel())
    return np.concatenate(out)


def boundary_nodes(gd, p):
    """Physical coordinates of the boundary face nodes in the boundary-state table's order
    (cell by cell, then face direction d, then side s, then the face's Gauss node)."""
    nq = max(1, (3 * p + 2) // 2)           # smallest n with 2n - 1 >= 3p
    t, _ = orc.gauss_rule(nq)
    n = [gd.n[0], gd.n[1]]
    cen, h = cell_centers(gd)
    ix, iy = np.unravel_index(np.arange(n[0] * n[1]), n)
    idx = [ix, iy]
    pts = []
    for j in range(len(cen)):
        for d in range(2):
            for s in range(2):
                if (s == 0 and idx[d][j] == 0) or (s == 1 and idx[d][j] == n[d] - 1):
                    o = 1 - d
                    for q in range(nq):
                        xy = [0.0, 0.0]
                        xy[d] = cen[j, d] + (0.5 if s else -0.5) * h[d]
                        xy[o] = cen[j, o] + 0.5 * h[o] * t[q]
                        pts.append(xy)
    return np.array(pts)


def case(p):
    """(op_desc, grid_desc, U, boundary table) of the consistency case for degree p."""
    gd = grid_desc()
    opd = op_desc(p)
    U = project(gd, p, conservative)
    xb = boundary_nodes(gd, p)
    bnd = conservative(xb[:, 0], xb[:, 1])
    return opd, gd, U, bnd


def reference_values(p):
    with open(os.path.join(HERE, "golden", "sipg_consistency_p%d.json" % p)) as f:
        return np.array(json.load(f)["values"])


def problem(p):
    """The case registered through the operator mirror the way the CNS solver builds its
    diffusive operator (OperatorFactory / Operator.ToSpatialOperator, CNS/EquationSystem/
    Operator.cs:143-174): (op, grid, domain fields, codomain fields)."""
    from bosss_b200 import operator as O
    x = np.linspace(0.0, 2.0 * math.pi, N_CELLS + 1)
    g = O.Cartesian2DGrid(x, x, False, False)
    names = ["rho", "m0", "m1", "rhoE"]
    op = O.DifferentialOperator(names, [], names, O.QuadOrderFunc.NonLinear(2))
    mat = O.CNSMaterial(gamma=GAMMA, Mach=MACH, Reynolds=1.0, Prandtl=1.0, ViscosityRatio=0.0, sutherland=True,
                        sutherland_ratio=SUTHERLAND, SIPGPenaltyScaling=1.0)
    op.EquationComponents["rho"].Add(O.OptimizedSIPGDensityFlux(mat, 2))
    for d in range(2):
        op.EquationComponents["m%d" % d].Add(O.OptimizedSIPGMomentumFlux(mat, d, 2))
    op.EquationComponents["rhoE"].Add(O.OptimizedSIPGEnergyFlux(mat, 2))
    op.Commit()
    dom = [O.DGField(g, p, n) for n in names]
    cod = [O.DGField(g, p, n) for n in names]
    return op, g, dom, cod
