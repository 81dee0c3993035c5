"""The oracle's restatement of the level-set interface term (XLaplace_Interface), on a
hand-built planar surface rule in one cell (CPU only):

* the form is a symmetric bilinear form of (uA, uB) and (vA, vB), so the assembled 2Np x 2Np
  matrix is symmetric;
* consistency: for uA = uB = u (no jump) and mu_A = mu_B = mu the rows of species A hold
  mu * int grad(u).N phi_n dS and those of B the negative;
* the penalty scales with the jump only.
"""
import numpy as np
import pytest

from oracle import oracle as orc


def plane_rule(nq=4, h=0.5, z=0.1):
    """Surface z = const through one cell [0,h]^3 (normal +e_z), tensor Gauss rule."""
    x, w = np.polynomial.legendre.leggauss(nq)
    xi = []
    wt = []
    zt = 2.0 * z / h - 1.0
    for i in range(nq):
        for j in range(nq):
            xi.append((x[i], x[j], zt))
            wt.append(w[i] * w[j] * (0.5 * h) ** 2)
    q = len(wt)
    return {"cells": np.array([0]), "offsets": np.array([0, q]), "nodes": np.array(xi), "weights": np.array(wt),
            "normals": np.tile([0.0, 0.0, 1.0], (q, 1))}


NODES = [np.array([0.0, 0.5])] * 3


@pytest.mark.parametrize("mode", [0, 1])
def test_interface_form_is_symmetric(mode):
    k = 2
    Np = 10
    R = plane_rule()
    M = np.zeros((2 * Np, 2 * Np))
    for c in range(2 * Np):
        e = np.zeros(2 * Np)
        e[c] = 1.0
        oA, oB = orc.xdg_interface(NODES, [False] * 3, k, R, e[:Np], e[Np:], 1.0, 10.0, 4.0, mode)
        M[:, c] = np.concatenate([oA, oB])
    assert np.abs(M - M.T).max() <= 1e-12 * np.abs(M).max()
    # the penalty part is negative semi-definite (Ret -= pen (uA-uB)(vA-vB)) and the
    # consistency/symmetry parts vanish on constants: constant u on both sides gives 0
    const = np.zeros(2 * Np)
    const[0] = const[Np] = 1.0
    assert np.abs(M @ const).max() <= 1e-12 * np.abs(M).max()


def test_interface_consistency_without_jump():
    k = 2
    Np = 10
    R = plane_rule(nq=5)
    rng = np.random.default_rng(7)
    u = rng.uniform(-1, 1, Np)
    mu = 3.0
    oA, oB = orc.xdg_interface(NODES, [False] * 3, k, R, u, u, mu, mu, 4.0, 1)
    # direct: mu * sum_q w grad(u).e_z phi_n with the oracle basis
    phi, dphi = orc.basis_eval(3, k, R["nodes"])
    sc = 1.0 / np.sqrt(0.25 ** 3)
    gz = (u @ dphi[:, :, 2]) * sc * 4.0
    ref = mu * (phi * sc) @ (R["weights"] * gz)
    assert np.allclose(oA, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    assert np.allclose(oB, -ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
