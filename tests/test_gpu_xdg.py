"""XDG bulk evaluation with moment-fitted cut-cell rules (two-phase Poisson, sphere).

* the device weight solve equals numpy's minimum-norm least squares (what DGELSY returns)
  on the same node sets and moments;
* the species volumes integrated with the rules reproduce the sphere volume;
* the per-species evaluation equals the oracle's restatement given the same rules and
  species cell length scales;
* the default species length scales equal species volume / (interface area + the species'
  face areas) recomputed here from the rules (MultiphaseAgglomerator.LengthScaleAgg without
  agglomeration), and caller-supplied (e.g. agglomerated) scales take effect;
* the full-size case (128^3, k=2): both species equal the oracle with the same rules.
"""
import numpy as np
import pytest

from bosss_b200 import _capi as C
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
        ref = orc.xdg_evaluate(op.descriptor([2], [2], 3), g.desc(), R, U, length_scales=X.length_scales(s))
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


def test_xdg_masked_slab_equals_masked_generic():
    """The species masks are read by both bulk kernels: the default handles (slab residual for
    the 3D SIP bulk) and handles forced onto the generic tile give the same species residuals."""
    opA, opB, g, c, UA, UB = small_case(n=12)
    with O.XdgEvaluator(opA, opB, g, 2, c, 0.4) as Xs, O.XdgEvaluator(opA, opB, g, 2, c, 0.4,
                                                                      kernel=C.KERNEL_GENERIC) as Xg:
        for s, U in enumerate((UA, UB)):
            a, b = np.zeros_like(U), np.zeros_like(U)
            Xs.Evaluate(s, 1.0, 0.0, a, U)
            Xg.Evaluate(s, 1.0, 0.0, b, U)
            assert rel(a, b) <= 1e-13, (s, rel(a, b))


def test_xdg_evaluation_is_bitwise_reproducible(xdg_small):
    """Cut items reduce in a fixed order (no atomics), so repeated evaluations give the same
    bits, bulk and interface term."""
    import torch
    opA, opB, g, c, UA, UB, X = xdg_small
    X.SetInterface(1.0, 10.0, 4.0, X.SIP, 6)
    outs = []
    for _ in range(3):
        a, b = torch.zeros(UA.size, dtype=torch.float64, device="cuda"), torch.zeros(UB.size, dtype=torch.float64, device="cuda")
        uA, uB = torch.from_numpy(UA).cuda(), torch.from_numpy(UB).cuda()
        X.Evaluate(0, 1.0, 0.0, a, uA)
        X.Evaluate(1, 1.0, 0.0, b, uB)
        X.EvaluateInterface(1.0, uA, uB, a, b)
        torch.cuda.synchronize()
        outs.append((a.cpu(), b.cpu()))
    for a, b in outs[1:]:
        assert torch.equal(a, outs[0][0]) and torch.equal(b, outs[0][1])


def test_saye_rules_evaluate_and_volume():
    """Saye-type rules (rule family 1, 8 Gauss nodes per direction and piece): the species-A
    rules plus the full cells give the ball volume to 1e-9 (the moment-fitted family: 1e-4,
    the accuracy of its subdivided moment integration), and the evaluation with these rules
    equals the oracle's with the same rules."""
    opA, opB, g, c, UA, UB = small_case()
    with O.XdgEvaluator(opA, opB, g, 2, c, 0.4, rule=C.XDG_RULE_SAYE, cut_nodes_1d=8) as X:
        h = 2.0 / 10
        detJ = (h / 2) ** 3
        R0 = X.rules(0)
        v = np.sum(R0["vol_flags"] == 1) * 8 * detJ
        for r, (cell, dim, d, side, deg) in enumerate(R0["info"]):
            if dim == 3:
                v += R0["weights"][R0["offsets"][r]:R0["offsets"][r + 1]].sum() * detJ
        exact = 4.0 / 3.0 * np.pi * 0.4 ** 3
        assert abs(v - exact) <= 1e-9 * exact, (v, exact)
        for s, (op, U) in enumerate([(opA, UA), (opB, UB)]):
            R = X.rules(s)
            ref = orc.xdg_evaluate(op.descriptor([2], [2], 3), g.desc(), R, U, length_scales=X.length_scales(s))
            out = np.zeros_like(U)
            X.Evaluate(s, 1.0, 0.0, out, U)
            assert rel(out, ref) <= 1e-12, (s, rel(out, ref))


def test_xdg_full_size_matches_oracle():
    """The full 128^3, k=2 case: both species against the oracle with the same rules."""
    import torch
    opA, opB, g, c, UA, UB = P.xdg_poisson3d(n=128, k=2, seed=4000)
    with O.XdgEvaluator(opA, opB, g, 2, c, 0.4) as X:
        infA, infB = X.info(0), X.info(1)
        assert 5000 < infA["cut_cells"] < 20000
        assert infA["min_nodes"] >= 1 and infA["max_nodes"] <= 128
        for s, (op, U) in enumerate([(opA, UA), (opB, UB)]):
            Ud = torch.from_numpy(U).cuda()
            out = torch.zeros_like(Ud)
            X.Evaluate(s, 1.0, 0.0, out, Ud)
            torch.cuda.synchronize()
            ref = orc.xdg_evaluate(op.descriptor([2], [2], 3), g.desc(), X.rules(s), U,
                                   length_scales=X.length_scales(s))
            assert rel(out.cpu().numpy(), ref) <= 1e-12, (s, rel(out.cpu().numpy(), ref))


def _default_length_scales(X, s, n):
    """Independent recomputation from the rules: V / (A_interface + sum of the species' face areas)."""
    R = X.rules(s)
    h = 2.0 / n
    J = n ** 3
    vol = h ** 3
    V = np.where(R["vol_flags"] == 1, vol, 0.0)
    fa = np.where(R["face_flags"].reshape(J, 6) == 1, h * h, 0.0)
    stride = [n * n, n, 1]
    for r, (cell, dim, d, side, deg) in enumerate(R["info"]):
        sw = R["weights"][R["offsets"][r]:R["offsets"][r + 1]].sum()
        if dim == 3:
            V[cell] = sw * (h / 2) ** 3
        else:
            a = sw * (h / 2) ** 2
            fa[cell, 2 * d + side] = a
            i = (cell // stride[d]) % n
            i2 = i + (1 if side else -1)
            if 0 <= i2 < n:
                fa[cell + (1 if side else -1) * stride[d], 2 * d + (1 - side)] = a
    X.SetInterface(1.0, 10.0, 4.0, X.SIP, nodes_1d=6)
    IR = X.interface_rules()
    ia = np.zeros(J)
    for r, cell in enumerate(IR["cells"]):
        ia[cell] += IR["weights"][IR["offsets"][r]:IR["offsets"][r + 1]].sum()
    S = ia + fa.sum(axis=1)
    L = np.full(J, np.nan)
    m = R["vol_flags"] != 0
    L[m] = np.maximum(V[m] / S[m], 2.220446049250313e-16 * h)
    return L, V, m


def test_default_length_scales_from_rules(xdg_small):
    opA, opB, g, c, UA, UB, X = xdg_small
    for s in (0, 1):
        L, V, m = _default_length_scales(X, s, 10)
        got = X.length_scales(s)
        assert np.array_equal(np.isnan(got), ~m)
        assert np.allclose(got[m], L[m], rtol=1e-13, atol=0)
        # uncut cells of the species: h^3 / (6 h^2); cut cells differ from the uncut value
        h = 0.2
        uncut = (X.rules(s)["vol_flags"] == 1)
        assert np.allclose(got[uncut], h / 6, rtol=1e-14)
        cut = X.rules(s)["vol_flags"] == 2
        assert np.abs(got[cut] - h / 6).max() > 0.1 * h / 6


def test_caller_length_scales_take_effect(xdg_small):
    """Caller-supplied (e.g. agglomerated) length scales: GPU == oracle with the same scales,
    different from the defaults' result; None restores the defaults."""
    opA, opB, g, c, UA, UB, X = xdg_small
    s = 0
    R = X.rules(s)
    base = X.length_scales(s)
    L = np.where(np.isnan(base), np.nan, np.random.default_rng(3).uniform(0.01, 0.05, base.size))
    try:
        X.set_length_scales(s, L)
        assert np.array_equal(np.nan_to_num(X.length_scales(s), nan=-1), np.nan_to_num(L, nan=-1))
        ref = orc.xdg_evaluate(opA.descriptor([2], [2], 3), g.desc(), R, UA, length_scales=L)
        out = np.zeros_like(UA)
        X.Evaluate(s, 1.0, 0.0, out, UA)
        assert rel(out, ref) <= 1e-12
        ref0 = orc.xdg_evaluate(opA.descriptor([2], [2], 3), g.desc(), R, UA, length_scales=base)
        assert rel(ref, ref0) > 1e-3
        bad = L.copy()
        bad[np.flatnonzero(~np.isnan(L))[0]] = 0.0
        with pytest.raises(Exception):
            X.set_length_scales(s, bad)
    finally:
        X.set_length_scales(s, None)
    assert np.array_equal(np.nan_to_num(X.length_scales(s), nan=-1), np.nan_to_num(base, nan=-1))
