"""Explicit Runge-Kutta time stepping (RungeKutta.Perform, TimeStepping/RungeKutta.cs:242-313).

CPU: tableau checks of the named schemes (order conditions), the oracle's RK restatement
against the exact Taylor polynomial of exp(-dt A) for a linear operator (classical RK4 and the
explicit Euler step are known answers there), and the C-ABI entry points' argument errors.
GPU: device steps against the oracle's RK steps (FP64, 1e-12 relative), graph replay equal
to plain launches bit for bit, and the temporal order of RK4 on smooth periodic transport.
"""
import ctypes

import numpy as np
import pytest

from bosss_b200 import _capi as C
from bosss_b200 import operator as O
from bosss_b200 import problems as P
from bosss_b200 import timestepping as T
from oracle import oracle as orc

NAMED = ["ExplicitEuler", "ExplicitEuler2", "Middlepoint", "Heun2", "Heun", "RungeKutta3", "TVD3",
         "RungeKutta1901", "ThreeOverEight", "SSP54"]
ORDER = {"ExplicitEuler": 1, "ExplicitEuler2": 1, "Middlepoint": 2, "Heun2": 2, "Heun": 3, "RungeKutta3": 3,
         "TVD3": 3, "RungeKutta1901": 4, "ThreeOverEight": 4, "SSP54": 4}


@pytest.mark.parametrize("name", NAMED)
def test_named_scheme_order_conditions(name):
    s = getattr(T.RungeKuttaScheme, name)()
    a, b, c = s.a, s.b, s.c
    assert s.IsExplicit
    p = ORDER[name]
    conds = [(b.sum(), 1.0)]
    if p >= 2:
        conds.append((b @ c, 0.5))
    if p >= 3:
        conds += [(b @ c ** 2, 1 / 3), (b @ a @ c, 1 / 6)]
    if p >= 4:
        conds += [(b @ c ** 3, 1 / 4), (b @ (c * (a @ c)), 1 / 8), (b @ a @ c ** 2, 1 / 12), (b @ a @ a @ c, 1 / 24)]
    for got, want in conds:
        assert abs(got - want) < 1e-12, (name, got, want)


def test_scheme_validation():
    with pytest.raises(ValueError):
        T.RungeKuttaScheme([[0, 0], [1, 0]], [0.6, 0.5], [0, 1])   # b does not sum to 1
    with pytest.raises(ValueError):
        T.RungeKuttaScheme([[0, 0], [1, 0]], [0.5, 0.5], [0, 0.5])   # c != row sums
    assert T.RungeKutta.SchemeFactory(T.RungeKuttaSchemes.TVD3).Stages == 3
    with pytest.raises(NotImplementedError):
        T.RungeKutta.SchemeFactory("SSP54")


def _taylor(A, y, dt, order):
    out, term = y.copy(), y.copy()
    for m in range(1, order + 1):
        term = (-dt / m) * (A @ term)
        out += term
    return out


@pytest.mark.parametrize("name,order", [("RungeKutta1901", 4), ("ExplicitEuler", 1), ("Heun2", 2)])
def test_oracle_rk_equals_taylor_polynomial_on_linear_operator(name, order):
    # for du/dt = -A u, an explicit s-stage scheme of order p = s (s <= 4) gives exactly the
    # degree-p Taylor polynomial of exp(-dt A)
    pr = P.transport2d(n=4, k=2, seed=3)
    opd, gd = pr.descs()
    A = orc.jacobian_dense(opd, gd, pr.U)
    assert np.allclose(orc.evaluate(opd, gd, pr.U), A @ pr.U, rtol=0, atol=1e-12)
    s = getattr(T.RungeKuttaScheme, name)()
    dt = 0.01
    y1 = orc.rk_steps(opd, gd, pr.U, s.a, s.b, s.c, dt)
    ref = _taylor(A, pr.U, dt, order)
    assert np.max(np.abs(y1 - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))


def test_rk_abi_rejects_bad_arguments():
    L = C.lib()
    n = ctypes.c_int64()
    assert L.bosss_b200_rk_work_size(None, 3, ctypes.byref(n)) == C.ERR_BAD_ARG
    a = np.zeros(4)
    b = np.array([0.5, 0.5])
    c = np.zeros(2)
    assert L.bosss_b200_rk_steps_device(None, 2, C.ptr(a), C.ptr(b), C.ptr(c), 0.1, 1, 0.0, None, None, 1,
                                        None) == C.ERR_BAD_ARG


# ------------------------------------------------------------------------------- GPU


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b)))


@pytest.mark.gpu
@pytest.mark.parametrize("case,name,nsteps", [("euler", "TVD3", 3), ("euler", "RungeKutta1901", 2),
                                              ("transport", "SSP54", 4), ("advdiff", "Heun", 3)])
def test_rk_device_matches_oracle(case, name, nsteps):
    if case == "euler":
        pr = P.euler3d(n=4, k=2, seed=11)
        dt = 2e-3
    elif case == "transport":
        pr = P.transport2d(n=8, k=3, seed=12)
        dt = 5e-3
    else:
        pr = P.advection_diffusion3d(n=4, k=2, seed=13)
        dt = 1e-4
    opd, gd = pr.descs()
    s = getattr(T.RungeKuttaScheme, name)()
    ref = orc.rk_steps(opd, gd, pr.U, s.a, s.b, s.c, dt, nsteps)
    ev = pr.evaluator()
    try:
        U = np.array(pr.U, copy=True)
        rk = T.RungeKutta(s, ev, U)
        rk.Perform(dt, nsteps)
        assert abs(rk.Time - nsteps * dt) < 1e-15
        assert _rel(U, ref) <= 1e-12, _rel(U, ref)
    finally:
        ev.Dispose()


@pytest.mark.gpu
def test_rk_graph_equals_plain_launches():
    import torch
    pr = P.euler3d(n=6, k=3, seed=21)
    ev = pr.evaluator()
    try:
        s = T.RungeKuttaScheme.RungeKutta1901()
        Ug = torch.tensor(pr.U, device="cuda")
        Up = Ug.clone()
        T.RungeKutta(s, ev, None).PerformDevice(Ug, 1e-3, nsteps=5, use_graph=True)
        T.RungeKutta(s, ev, None).PerformDevice(Up, 1e-3, nsteps=5, use_graph=False)
        torch.cuda.synchronize()
        assert torch.equal(Ug, Up)
        opd, gd = pr.descs()
        ref = orc.rk_steps(opd, gd, pr.U, s.a, s.b, s.c, 1e-3, 5)
        assert _rel(Ug.cpu().numpy(), ref) <= 1e-12
    finally:
        ev.Dispose()


@pytest.mark.gpu
def test_rk4_temporal_order_on_smooth_transport():
    # u0 = sin(2 pi x) sin(2 pi y) projected, periodic transport; errors against a run with a
    # 16x smaller step: halving dt reduces the RK4 error by about 2^4
    n, k = 8, 3
    g = O.Cartesian2DGrid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1), True, True)
    op = O.DifferentialOperator(["u"], [], ["R"], O.QuadOrderFunc.FixedOrder(2 * k + 1))
    op.EquationComponents["R"].Add(O.ScalarTransportFlux((1.0, 0.5), "u"))
    op.Commit()
    u, r = O.DGField(g, k, "u"), O.DGField(g, k, "R")
    nq = k + 2
    phi, W, xi = P.volume_basis(2, k, nq)
    h = 1.0 / n
    ij = g.cell_ijk()
    X = (ij[:, 0:1] + 0.5 + 0.5 * xi[None, :, 0]) * h
    Y = (ij[:, 1:2] + 0.5 + 0.5 * xi[None, :, 1]) * h
    U0 = P.project_nodal(2, k, nq, [h, h], np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y)).ravel()
    ev = op.GetEvaluatorEx([u], None, [r])
    try:
        Tend = 0.08

        def run(nsteps):
            U = np.array(U0, copy=True)
            T.RungeKutta(T.RungeKuttaScheme.RungeKutta1901(), ev, U).Perform(Tend / nsteps, nsteps)
            return U

        fine = run(32 * 16)
        e1 = np.linalg.norm(run(32) - fine)
        e2 = np.linalg.norm(run(64) - fine)
        rate = np.log2(e1 / e2)
        assert 3.6 < rate < 4.4, (e1, e2, rate)
    finally:
        ev.Dispose()
