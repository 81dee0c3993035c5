"""Level-set interface term of the two-phase Poisson problem (XLaplace_Interface over the
sphere surface, NECQuadratureLevelSet):

* the surface rules reproduce the sphere's area, int (x - c).N dS = 3 |ball| and int N dS = 0;
* the device evaluation (host-buffer and device entry points) equals the oracle's
  restatement given the same rules (SIP and SWIP), relative L2 <= 1e-12;
* the full-size case (128^3, k=2) builds its rules and evaluates.
"""
import math

import numpy as np
import pytest

from bosss_b200 import operator as O
from bosss_b200 import problems as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

R0 = 0.4


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def node_vectors(g):
    return [np.linspace(g.lo[d], g.hi[d], g.n[d] + 1) for d in range(3)]


def surface_moments(g, c, rules):
    h = np.array([(g.hi[d] - g.lo[d]) / g.n[d] for d in range(3)])
    lo = np.array(g.lo)
    cells = rules["cells"]
    ijk = np.stack([cells // (g.n[1] * g.n[2]), (cells // g.n[2]) % g.n[1], cells % g.n[2]], axis=1)
    cnt = np.diff(rules["offsets"])
    base = np.repeat(lo + ijk * h, cnt, axis=0)
    x = base + 0.5 * (rules["nodes"] + 1.0) * h
    w, N = rules["weights"], rules["normals"]
    area = w.sum()
    xn = (w * ((x - c) * N).sum(axis=1)).sum()
    nsum = np.abs(w @ N).max()
    return area, xn, nsum


@pytest.mark.parametrize("n,k,nodes_1d,tol", [(10, 2, 8, 1e-6), (16, 2, 6, 1e-5)])
def test_surface_rules_known_answers(n, k, nodes_1d, tol):
    opA, opB, g, c, UA, UB = P.xdg_poisson3d(n=n, k=k, seed=4002)
    with O.XdgEvaluator(opA, opB, g, k, c, R0) as X:
        X.SetInterface(1.0, 10.0, 4.0, X.SIP, nodes_1d)
        rules = X.interface_rules()
        assert len(rules["cells"]) > 0
        area, xn, nsum = surface_moments(g, np.asarray(c), rules)
        assert abs(area / (4 * math.pi * R0 ** 2) - 1) < tol
        assert abs(xn / (4 * math.pi * R0 ** 3) - 1) < tol
        assert nsum < tol * area
        # every cut cell of the bulk rules with a surface piece appears once
        assert len(np.unique(rules["cells"])) == len(rules["cells"])


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("n", [8, 11])
def test_interface_matches_oracle(mode, n):
    k = 2   # the two-phase Poisson bulk operator (Gauss order 5) is instantiated for k = 2
    import torch
    opA, opB, g, c, UA, UB = P.xdg_poisson3d(n=n, k=k, seed=4003 + n)
    with O.XdgEvaluator(opA, opB, g, k, c, R0) as X:
        X.SetInterface(1.0, 10.0, 4.0, mode, 5)
        rules = X.interface_rules()
        lens = (X.length_scales(0), X.length_scales(1))
        refA, refB = orc.xdg_interface(node_vectors(g), g.periodic, k, rules, UA, UB, 1.0, 10.0, 4.0, mode, alpha=0.7,
                                       length_scales=lens)
        # host-buffer entry point: adds to the given outputs
        oA = np.full(UA.size, 0.25)
        oB = np.full(UB.size, -0.5)
        X.EvaluateInterface(0.7, UA, UB, oA, oB)
        assert rel(oA - 0.25, refA) <= 1e-12
        assert rel(oB + 0.5, refB) <= 1e-12
        # device entry point
        dUA, dUB = torch.from_numpy(UA).cuda(), torch.from_numpy(UB).cuda()
        dA, dB = torch.zeros_like(dUA), torch.zeros_like(dUB)
        X.EvaluateInterface(0.7, dUA, dUB, dA, dB)
        torch.cuda.synchronize()
        assert rel(dA.cpu().numpy(), refA) <= 1e-12
        assert rel(dB.cpu().numpy(), refB) <= 1e-12


def test_interface_full_size():
    import time
    import torch
    opA, opB, g, c, UA, UB = P.xdg_poisson3d(n=128, k=2, seed=4000)
    with O.XdgEvaluator(opA, opB, g, 2, c, R0) as X:
        t0 = time.perf_counter()
        X.SetInterface(1.0, 10.0, 4.0, X.SIP, 6)
        t_setup = time.perf_counter() - t0
        rules = X.interface_rules()
        area, xn, _ = surface_moments(g, np.asarray(c), rules)
        assert abs(area / (4 * math.pi * R0 ** 2) - 1) < 1e-6
        dUA, dUB = torch.from_numpy(UA).cuda(), torch.from_numpy(UB).cuda()
        dA, dB = torch.zeros_like(dUA), torch.zeros_like(dUB)
        X.EvaluateInterface(1.0, dUA, dUB, dA, dB)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        X.EvaluateInterface(1.0, dUA, dUB, dA, dB)
        e1.record()
        torch.cuda.synchronize()
        # linearity in alpha: the second call added the same amount again
        A1 = dA.cpu().numpy()
        dA.zero_()
        X.EvaluateInterface(2.0, dUA, dUB, dA, dB)
        assert rel(dA.cpu().numpy(), A1) <= 1e-13
        print("interface 128^3 k=2: %d cut cells, %d nodes, setup %.2f s, evaluation %.3f ms"
              % (len(rules["cells"]), rules["weights"].size, t_setup, e0.elapsed_time(e1)))
