"""The CNS viscous SIPG operator (OptimizedSIPG fluxes, Sutherland viscosity, supersonic-inlet
boundary state) on the GPU against the reference's own stored operator outputs.

``SIPGConsistency.cs:87-160`` evaluates the operator once on the 3x3 grid of ``Control``
(``:165-225``) and checks every DOF against ``SIPGConsistencyRefSolution_p{1,2,3}.txt`` to
1e-11; the same check here, on the device, through the C-ABI: the operator registered through
the mirror, the boundary-state table filled at the library's boundary nodes from the
primitive boundary values (what SupersonicInlet.GetBoundaryState returns there). Also: the
device result equals the oracle's (relative L2 <= 1e-12), JVP / VJP equal the oracle's exact
products, and an evaluation without the table is rejected.
"""
import numpy as np
import pytest

import cns_sipg_case as S
from bosss_b200 import _capi as C
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("p", [1, 2, 3])
def test_gpu_reproduces_reference_sipg_consistency_output(p):
    op, g, dom, cod = S.problem(p)
    opd, gd, U, bnd = S.case(p)
    with op.GetEvaluatorEx(dom, None, cod) as ev:
        xb = ev.boundary_nodes()
        assert np.allclose(xb, S.boundary_nodes(gd, p), rtol=0, atol=1e-14)   # same numbering as the oracle's
        out = np.zeros(ev.n_codomain)
        with pytest.raises(C.BosssError) as ei:
            ev.Evaluate(1.0, 0.0, out, U)        # no boundary-state table yet
        assert ei.value.code == C.ERR_BAD_ARG
        ev.SetBoundaryState(S.conservative(xb[:, 0], xb[:, 1]))
        ev.Evaluate(1.0, 0.0, out, U)
        ref = S.reference_values(p)
        # SIPGConsistency.cs:155-158: |refSol[i] - output[i]| < 1e-11 for every DOF
        assert np.abs(out - ref).max() < 1e-11, np.abs(out - ref).max()
        assert rel(out, orc.evaluate(opd, gd, U, bnd=bnd)) <= 1e-12
        r = np.random.default_rng(p)
        V = r.uniform(-1, 1, U.size)
        W = r.uniform(-1, 1, U.size)
        assert rel(ev.jvp(U, V), orc.jvp(opd, gd, U, V, bnd=bnd)) <= 1e-12
        assert rel(ev.vjp(U, W), orc.vjp(opd, gd, U, W, bnd=bnd)) <= 1e-12
