"""Saye-type cut-cell rules (``bosss_b200_saye_rule``, host computation, no GPU needed).

Known answers: over every cell of a grid cut by the sphere phi = |x - c| - r, the species
rules plus the full cells reproduce the ball volume 4/3 pi r^3 and the volume of the box
minus the ball; polynomial moments of a single cut cell agree with a brute-force
integration by fine subdivision; face rules reproduce the disc area where the face plane
cuts the sphere, converging exponentially in the Gauss nodes per piece (5: ~3e-8,
8: ~3e-12, 10: ~1e-14 relative); species A + species B = the whole cell.
"""
import ctypes
import math

import numpy as np
import pytest

from bosss_b200 import _capi as C


def rule(center, h, dim, direction, species, c, r, q=5):
    ls = C.LevelSetDesc()
    ls.type = C.LEVELSET_SPHERE
    for i, v in enumerate(list(c) + [r]):
        ls.params[i] = float(v)
    cen = np.ascontiguousarray(center, dtype=np.float64)
    hh = np.ascontiguousarray(h, dtype=np.float64)
    n = ctypes.c_int64()
    C.check(C.lib().bosss_b200_saye_rule(ctypes.byref(ls), dim, direction, species, C.ptr(cen), C.ptr(hh), q,
                                         ctypes.byref(n), None, None))
    nodes = np.zeros(3 * n.value)
    w = np.zeros(n.value)
    C.check(C.lib().bosss_b200_saye_rule(ctypes.byref(ls), dim, direction, species, C.ptr(cen), C.ptr(hh), q,
                                         ctypes.byref(n), C.ptr(nodes), C.ptr(w)))
    return nodes.reshape(-1, 3), w


def test_ball_volume_from_cut_and_full_cells():
    c, r, n = np.array([0.013, -0.021, 0.007]), 0.4, 12
    h = 2.0 / n
    vol_in = vol_out = 0.0
    for i in range(n):
        for j in range(n):
            for k in range(n):
                lo = -1.0 + h * np.array([i, j, k])
                near = np.clip(c, lo, lo + h)
                dmin = np.linalg.norm(near - c)
                dmax = np.linalg.norm(np.maximum(np.abs(lo - c), np.abs(lo + h - c)))
                if dmax <= r:
                    vol_in += h ** 3
                elif dmin >= r:
                    vol_out += h ** 3
                else:
                    for sp in (-1, 1):
                        _, w = rule(lo + h / 2, [h] * 3, 3, 0, sp, c, r, q=8)
                        if sp < 0:
                            vol_in += w.sum() * (h / 2) ** 3
                        else:
                            vol_out += w.sum() * (h / 2) ** 3
    ball = 4.0 / 3.0 * math.pi * r ** 3
    assert abs(vol_in - ball) <= 1e-9 * ball
    assert abs(vol_in + vol_out - 8.0) <= 1e-12


def test_cut_cell_moments_match_subdivision():
    c, r = np.array([0.0, 0.0, 0.0]), 0.4
    center, h = np.array([0.31, 0.12, 0.2]), np.array([0.2, 0.2, 0.2])
    # brute force: 80^3 midpoint cells with a 3-point Gauss rule each, inside the sphere only
    m = 80
    g, gw = np.polynomial.legendre.leggauss(3)
    t = (np.arange(m) + 0.5) / m * 2 - 1
    sub = (np.add.outer(t, g / m)).ravel()
    wsub = np.tile(gw / m, m)
    X, Y, Z = np.meshgrid(sub, sub, sub, indexing="ij")
    W = np.einsum("i,j,k->ijk", wsub, wsub, wsub)
    P = np.stack([X, Y, Z], -1)
    inside = np.linalg.norm(center + 0.5 * h * P - c, axis=-1) < r
    nodes, w = rule(center, h, 3, 0, -1, c, r, q=6)
    for (a, b, cc) in [(0, 0, 0), (1, 0, 0), (0, 2, 1), (2, 1, 1), (3, 0, 1)]:
        brute = (W * inside * X ** a * Y ** b * Z ** cc).sum()
        saye = (w * nodes[:, 0] ** a * nodes[:, 1] ** b * nodes[:, 2] ** cc).sum()
        assert abs(saye - brute) <= 2e-4 * max(abs(brute), 1e-3), (a, b, cc, saye, brute)


@pytest.mark.parametrize("direction", [0, 1, 2])
def test_face_rule_disc_area_and_complement(direction):
    c, r = np.array([0.0, 0.0, 0.0]), 0.4
    # a face normal to `direction` at distance 0.1 from the centre, covering the whole disc
    center = np.zeros(3)
    center[direction] = 0.1
    h = np.array([1.0, 1.0, 1.0])
    disc = math.pi * (r * r - 0.1 * 0.1)
    errs = []
    for q in (4, 6, 8):
        _, wA = rule(center, h, 2, direction, -1, c, r, q=q)
        _, wB = rule(center, h, 2, direction, +1, c, r, q=q)
        errs.append(abs(wA.sum() * 0.25 - disc) / disc)
        assert abs((wA.sum() + wB.sum()) - 4.0) <= 1e-12
    assert errs[2] <= 1e-10 and errs[1] < 0.05 * errs[0] and errs[2] < 0.05 * errs[1], errs


def test_rejects_bad_arguments():
    ls = C.LevelSetDesc()
    ls.type = C.LEVELSET_SPHERE
    ls.params[3] = 0.4
    cen = np.zeros(3)
    hh = np.ones(3)
    n = ctypes.c_int64()
    rc = C.lib().bosss_b200_saye_rule(ctypes.byref(ls), 4, 0, -1, C.ptr(cen), C.ptr(hh), 5, ctypes.byref(n), None, None)
    assert rc == C.ERR_BAD_ARG
