"""XDG bulk evaluation with moment-fitted cut-cell rules (two-phase Poisson, sphere).

* the device weight solve equals numpy's minimum-norm least squares (what DGELSY returns)
  on the same node sets and moments;
* the species volumes integrated with the rules reproduce the sphere volume;
* the per-species evaluation equals the oracle's restatement given the same rules;
* the full-size case (128^3, k=2) builds its rules and evaluates both species.
"""
import numpy as np
import pytest

from bosss_b200 import operator as O
from bosss_b200 import problems as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def basis_at(dim, p, pts):
    L = [P._legendre_table(p, pts[:, d]) for d in range(dim)]
    cols = []
    for deg in range(p + 1):
        if dim == 3:
            for a in range(deg + 1):
                for b in range(deg - a + 1):
                    cols.append(L[0][:, a] * L[1][:, b] * L[2][:, deg - a - b])
        else:
            for a in range(deg + 1):
                cols.append(L[0][:, a] * L[1][:, deg - a])
    return np.array(cols)


def small_case(n=10, k=2):
    opA, opB, g, c, UA, UB = P.xdg_poisson3d(n=n, k=k, seed=4001)
    return opA, opB, g, c, UA, UB


@pytest.fixture(scope="module")
def xdg_small():
    opA, opB, g, c, UA, UB = small_case()
    X = O.XdgEvaluator(opA, opB, g, 2, c, 0.4)
    yield opA, opB, g, c, UA, UB, X
    X.Dispose()


def test_weight_solve_is_min_norm_lstsq(xdg_small):
    opA, opB, g, c, UA, UB, X = xdg_small
    for s in (0, 1):
        R = X.rules(s)
        inf = X.info(s)
        assert inf["cut_cells"] > 0 and inf["max_fit_residual"] < 1e-9, inf
        worst = 0.0
        for r, (cell, dim, d, side, deg) in enumerate(R["info"]):
            o0, o1 = R["offsets"][r], R["offsets"][r + 1]
            pts = R["nodes"][o0:o1, :dim if dim == 3 else 2]
            A = basis_at(3 if dim == 3 else 2, deg, pts)
            b = R["moments"][r, :A.shape[0]]
            w_np = np.linalg.lstsq(A, b, rcond=None)[0]
            w = R["weights"][o0:o1]
            worst = max(worst, np.linalg.norm(w - w_np) / max(np.linalg.norm(w_np), 1e-300))
        assert worst < 1e-9, worst


def test_rules_reproduce_sphere_volume(xdg_small):
    opA, opB, g, c, UA, UB, X = xdg_small
    h = 2.0 / 10
    detJ = (h / 2) ** 3
    vols = []
    for s in (0, 1):
        R = X.rules(s)
        v = np.sum(R["vol_flags"] == 1) * 8 * detJ
        for r, (cell, dim, d, side, deg) in enumerate(R["info"]):
            if dim == 3:
                v += R["weights"][R["offsets"][r]:R["offsets"][r + 1]].sum() * detJ
        vols.append(v)
    exact = 4.0 / 3.0 * np.pi * 0.4 ** 3
    assert abs(vols[0] - exact) < 1e-4 * exact, (vols[0], exact)
    assert abs(vols[0] + vols[1] - 8.0) < 1e-10


def test_xdg_evaluate_matches_oracle(xdg_small):
    opA, opB, g, c, UA, UB, X = xdg_small
    for s, (op, U) in enumerate([(opA, UA), (opB, UB)]):
        R = X.rules(s)
        ref = orc.xdg_evaluate(op.descriptor([2], [2], 3), g.desc(), R, U)
        out = np.full_like(U, 3.0)     # beta = 0 overwrites every cell
        X.Evaluate(s, 1.0, 0.0, out, U)
        assert rel(out, ref) <= 1e-12, (s, rel(out, ref))
        # cells without the species return 0
        absent = np.repeat(R["vol_flags"] == 0, 10)
        assert np.all(out[absent] == 0.0)
        # out = beta * out + alpha * Op(U) on every cell, inside and outside the species' band
        prev = np.random.default_rng(5 + s).uniform(-1, 1, U.size)
        out = prev.copy()
        X.Evaluate(s, 0.5, 0.25, out, U)
        assert rel(out, 0.25 * prev + 0.5 * ref) <= 1e-12
        assert np.array_equal(out[absent], 0.25 * prev[absent])


def test_xdg_full_size():
    import torch
    opA, opB, g, c, UA, UB = P.xdg_poisson3d(n=128, k=2, seed=4000)
    with O.XdgEvaluator(opA, opB, g, 2, c, 0.4) as X:
        infA, infB = X.info(0), X.info(1)
        assert 5000 < infA["cut_cells"] < 20000
        assert infA["min_nodes"] >= 1 and infA["max_nodes"] <= 128
        for s, U in ((0, UA), (1, UB)):
            Ud = torch.from_numpy(U).cuda()
            out = torch.zeros_like(Ud)
            X.Evaluate(s, 1.0, 0.0, out, Ud)
            torch.cuda.synchronize()
            assert torch.isfinite(out).all()
