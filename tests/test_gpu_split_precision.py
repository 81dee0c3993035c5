"""Split-precision residual (BOSSS_PRECISION_SPLIT_FP32): volume contractions on the tensor
cores (tcgen05 kind::i8, exact 8-bit slices, FP64 recombination), fluxes and faces in FP64.

Bars: relative L2 <= 1e-10 against the FP64 oracle at the full Euler 32^3 k=3 size and
against the device's plain FP64 path (the precision target of the split path; measured
7e-12: the slicing drops terms below 2^-48 of the row scale, and the volume terms largely
cancel with the face terms in the residual), alpha/beta accumulation, partial last tiles,
host-buffer entry point, JVP / VJP unchanged, unsupported operators rejected.
"""
import numpy as np
import pytest

from bosss_b200 import _capi as C
from bosss_b200 import problems as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _residual(pr, precision, alpha=1.0, beta=0.0, out0=None):
    with pr.evaluator(device=0, precision=precision) as ev:
        out = np.zeros(ev.n_codomain) if out0 is None else out0.copy()
        ev.Evaluate(alpha, beta, out, pr.U)
    return out


def test_split_residual_full_size_matches_oracle():
    pr = P.euler3d(n=32, k=3, seed=2000)
    opd, gd = pr.descs()
    ref = orc.evaluate(opd, gd, pr.U)
    R = _residual(pr, C.PRECISION_SPLIT_FP32)
    assert rel(R, ref) <= 1e-10
    R64 = _residual(pr, C.PRECISION_FP64)
    assert rel(R, R64) <= 1e-10


@pytest.mark.parametrize("n", [7, 5, 3])
def test_split_residual_small_grids(n):
    # 7^3 = 343, 5^3 = 125, 3^3 = 27 cells: tiles of 25 cells, partial last tiles
    pr = P.euler3d(n=n, k=3, seed=2100 + n)
    opd, gd = pr.descs()
    ref = orc.evaluate(opd, gd, pr.U)
    R = _residual(pr, C.PRECISION_SPLIT_FP32)
    assert rel(R, ref) <= 1e-10


def test_split_alpha_beta_semantics():
    pr = P.euler3d(n=6, k=3, seed=2201)
    opd, gd = pr.descs()
    ref = orc.evaluate(opd, gd, pr.U)
    out0 = np.random.default_rng(5).uniform(-1, 1, ref.size)
    R = _residual(pr, C.PRECISION_SPLIT_FP32, alpha=0.5, beta=-1.5, out0=out0)
    assert rel(R, 0.5 * ref - 1.5 * out0) <= 1e-10


def test_split_device_entry_and_unchanged_derivatives():
    import torch
    pr = P.euler3d(n=8, k=3, seed=2202)
    opd, gd = pr.descs()
    ref = orc.evaluate(opd, gd, pr.U)
    V = np.random.default_rng(6).uniform(-1, 1, pr.n_dofs)
    with pr.evaluator(device=0, precision=C.PRECISION_SPLIT_FP32) as ev, pr.evaluator(device=0) as e64:
        U = torch.from_numpy(pr.U).cuda()
        out = torch.zeros_like(U)
        ev.Evaluate(1.0, 0.0, out, U)
        torch.cuda.synchronize()
        assert rel(out.cpu().numpy(), ref) <= 1e-10
        # JVP / VJP stay on the FP64 kernels: identical to the plain handle's
        assert np.array_equal(ev.jvp(pr.U, V), e64.jvp(pr.U, V))
        assert np.array_equal(ev.vjp(pr.U, V), e64.vjp(pr.U, V))


def test_split_rejects_unsupported_operators():
    import ctypes
    # scalar SIP operator: no split-precision path
    pr = P.nonlinear_diffusion3d(n=4, k=2, seed=1)
    with pytest.raises(C.BosssError) as ei:
        pr.evaluator(device=0, precision=C.PRECISION_SPLIT_FP32)
    assert ei.value.code == C.ERR_BAD_ARG
    # Euler with 3 Gauss nodes per direction (quadrature order 5), and degree 2 with 4 nodes
    for k, qo in ((2, 5), (2, 7)):
        pr = P.euler3d(n=4, k=k, seed=2, quad_order=qo)
        with pytest.raises(C.BosssError) as ei:
            pr.evaluator(device=0, precision=C.PRECISION_SPLIT_FP32)
        assert ei.value.code == C.ERR_BAD_ARG
