"""ctypes wrapper of the CPU FP64 oracle ``oracle/_build/libdg_oracle.so``.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` -- never by the ``bosss_b200`` package. It
takes the same descriptors as the C-ABI (``include/bosss_b200.h``).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libdg_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        L.orc_evaluate.argtypes = [P, P, P, ctypes.c_double, ctypes.c_double, P, P]
        L.orc_jvp.argtypes = [P, P, P, P, P, P]
        L.orc_vjp.argtypes = [P, P, P, P, P, P]
        L.orc_jacobian_blocks.argtypes = [P, P, P, P, P, P]
        L.orc_boundary_nodes.argtypes = [P, P, P]
        L.orc_set_boundary_kinds.argtypes = [P]
        L.orc_bsr_spmv.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, P, P, P, ctypes.c_double, P,
                                   ctypes.c_double, P]
        L.orc_sizes.argtypes = [P, P, P, P, P]
        L.orc_gauss_rule.argtypes = [ctypes.c_int, P, P]
        L.orc_basis_eval.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]
        L.orc_basis_monomials.argtypes = [ctypes.c_int, ctypes.c_int, P, P]
        L.orc_threads.argtypes = [ctypes.c_int]
        L.orc_xdg_evaluate.argtypes = [P, P, P, P, ctypes.c_int64, P, P, P, P, P, P, P]
        L.orc_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(rc):
    if rc != 0:
        buf = ctypes.create_string_buffer(512)
        lib().orc_last_error(buf, 512)
        raise RuntimeError("oracle error %d: %s" % (rc, buf.value.decode()))


def threads(n=0):
    """Set (n > 0) and return the OpenMP thread count of the oracle."""
    return lib().orc_threads(n)


def sizes(opd, gd):
    nd, nc, nq = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    _check(lib().orc_sizes(ctypes.byref(opd), ctypes.byref(gd), ctypes.byref(nd), ctypes.byref(nc),
                           ctypes.byref(nq)))
    return nd.value, nc.value, nq.value


def _bnd(opd, gd, bnd):
    """Boundary-state table argument: None, or the outer values of every domain variable at
    every boundary face node (``boundary_nodes`` order), shape (nodes, n_domain)."""
    if bnd is None:
        return None, None
    b = np.ascontiguousarray(bnd, dtype=np.float64)
    assert b.shape == (n_boundary_nodes(opd, gd), opd.n_domain), b.shape
    return b, _p(b)


class boundary_kinds:
    """Context: boundary-condition kinds (0 table state, 1 outlet, 2 slip wall) per boundary
    face node for the oracle calls inside the block."""

    def __init__(self, kinds):
        self.kinds = None if kinds is None else np.ascontiguousarray(kinds, dtype=np.int32)

    def __enter__(self):
        lib().orc_set_boundary_kinds(None if self.kinds is None else _p(self.kinds))
        return self

    def __exit__(self, *a):
        lib().orc_set_boundary_kinds(None)


def n_boundary_nodes(opd, gd):
    n = ctypes.c_int64()
    _check(lib().orc_boundary_nodes(ctypes.byref(opd), ctypes.byref(gd), ctypes.byref(n)))
    return n.value


def evaluate(opd, gd, U, alpha=1.0, beta=0.0, out=None, bnd=None):
    nd, nc, _ = sizes(opd, gd)
    U = np.ascontiguousarray(U, dtype=np.float64)
    assert U.shape == (nd,)
    out = np.zeros(nc) if out is None else np.array(out, dtype=np.float64, copy=True)
    keep, bp = _bnd(opd, gd, bnd)
    _check(lib().orc_evaluate(ctypes.byref(opd), ctypes.byref(gd), bp, alpha, beta, _p(U), _p(out)))
    return out


def jvp(opd, gd, U, V, bnd=None):
    nd, nc, _ = sizes(opd, gd)
    U = np.ascontiguousarray(U, dtype=np.float64)
    V = np.ascontiguousarray(V, dtype=np.float64)
    out = np.zeros(nc)
    keep, bp = _bnd(opd, gd, bnd)
    _check(lib().orc_jvp(ctypes.byref(opd), ctypes.byref(gd), bp, _p(U), _p(V), _p(out)))
    return out


def vjp(opd, gd, U, W, bnd=None):
    """Exact adjoint product J(U)^T W (gradient of W . Op(U), differentiated node by node)."""
    nd, nc, _ = sizes(opd, gd)
    U = np.ascontiguousarray(U, dtype=np.float64)
    W = np.ascontiguousarray(W, dtype=np.float64)
    assert U.shape == (nd,) and W.shape == (nc,)
    out = np.zeros(nd)
    keep, bp = _bnd(opd, gd, bnd)
    _check(lib().orc_vjp(ctypes.byref(opd), ctypes.byref(gd), bp, _p(U), _p(W), _p(out)))
    return out


def jacobian_dense(opd, gd, U, bnd=None):
    """Exact Jacobian (dense, small problems only) assembled from the oracle's
    cell-block Jacobian."""
    nd, nc, _ = sizes(opd, gd)
    D = gd.dim
    J = int(np.prod([gd.n[d] for d in range(D)]))
    Nd, Nc = nd // J, nc // J
    NB = 1 + 2 * D
    blocks = np.zeros(J * NB * Nc * Nd)
    nbr = np.zeros(J * NB, dtype=np.int32)
    U = np.ascontiguousarray(U, dtype=np.float64)
    keep, bp = _bnd(opd, gd, bnd)
    _check(lib().orc_jacobian_blocks(ctypes.byref(opd), ctypes.byref(gd), bp, _p(U), _p(blocks), _p(nbr)))
    blocks = blocks.reshape(J, NB, Nc, Nd)
    nbr = nbr.reshape(J, NB)
    A = np.zeros((nc, nd))
    for j in range(J):
        seen = set()
        for b in range(NB):
            jc = nbr[j, b]
            if jc < 0 or jc in seen:
                continue
            seen.add(jc)
            A[j * Nc:(j + 1) * Nc, jc * Nd:(jc + 1) * Nd] = blocks[j, b]
    return A


def jacobian_blocks(opd, gd, U, bnd=None):
    """Cell-block Jacobian: (blocks[J, 1+2D, Nc, Nd], nbr[J, 1+2D])."""
    nd, nc, _ = sizes(opd, gd)
    D = gd.dim
    J = int(np.prod([gd.n[d] for d in range(D)]))
    Nd, Nc = nd // J, nc // J
    NB = 1 + 2 * D
    blocks = np.zeros(J * NB * Nc * Nd)
    nbr = np.zeros(J * NB, dtype=np.int32)
    U = np.ascontiguousarray(U, dtype=np.float64)
    keep, bp = _bnd(opd, gd, bnd)
    _check(lib().orc_jacobian_blocks(ctypes.byref(opd), ctypes.byref(gd), bp, _p(U), _p(blocks), _p(nbr)))
    return blocks.reshape(J, NB, Nc, Nd), nbr.reshape(J, NB)


def gauss_rule(n):
    x, w = np.zeros(n), np.zeros(n)
    lib().orc_gauss_rule(n, _p(x), _p(w))
    return x, w


def basis_eval(D, k, pts):
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, D)
    npts = pts.shape[0]
    from math import comb
    Np = comb(k + D, D)
    phi = np.zeros(Np * npts)
    dphi = np.zeros(Np * npts * D)
    lib().orc_basis_eval(D, k, npts, _p(pts), _p(phi), _p(dphi))
    return phi.reshape(Np, npts), dphi.reshape(Np, npts, D)


def basis_monomials(D, k):
    """List per polynomial of (coef, exponents) terms of the oracle's basis."""
    from math import comb
    Np = comb(k + D, D)
    T = (k + 1) ** D
    coef = np.zeros(Np * T)
    exps = np.zeros(Np * T * 3, dtype=np.int32)
    lib().orc_basis_monomials(D, k, _p(coef), _p(exps))
    coef = coef.reshape(Np, T)
    exps = exps.reshape(Np, T, 3)
    out = []
    for p in range(Np):
        out.append([(coef[p, t], tuple(exps[p, t, :D])) for t in range(T) if coef[p, t] != 0.0])
    return out


def xdg_evaluate(opd, gd, rules, U, length_scales=None):
    """XDG bulk evaluation of one species with given rules (flags, cut items, nodes, weights).
    ``length_scales``: the species' cell length scales of the SIP penalty (one per cell,
    ``CoefficientSet.CellLengthScales`` of the species, XLaplace.cs:104-113, ipLaplace.cs:131-141);
    None: the uncut grid's (Vol / (surface / 2))."""
    nd, nc, _ = sizes(opd, gd)
    U = np.ascontiguousarray(U, dtype=np.float64)
    out = np.zeros(nc)
    info = np.ascontiguousarray(rules["info"], dtype=np.int64)
    ls = None if length_scales is None else np.ascontiguousarray(length_scales, dtype=np.float64)
    _check(lib().orc_xdg_evaluate(ctypes.byref(opd), ctypes.byref(gd), _p(np.ascontiguousarray(rules["vol_flags"])),
                                  _p(np.ascontiguousarray(rules["face_flags"])), len(info), _p(info),
                                  _p(np.ascontiguousarray(rules["offsets"], dtype=np.int64)),
                                  _p(np.ascontiguousarray(rules["nodes"])), _p(np.ascontiguousarray(rules["weights"])),
                                  None if ls is None else _p(ls), _p(U), _p(out)))
    return out


def rk_steps(opd, gd, U, a, b, c, dt, nsteps=1):
    """Explicit Runge-Kutta steps of du/dt = -Op(u) on the oracle evaluator, restating
    RungeKutta.Perform / PerformStage (TimeStepping/RungeKutta.cs:242-313): k_s = Op(u_s) into a
    cleared k (ExplicitEuler.ComputeChangeRate, ExplicitEuler.cs:223-229), u_s = y0 -
    dt*sum_{r<s} a[s,r] k_r, y1 = y0 - dt*sum_s b[s] k_s."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64).ravel()
    S = b.size
    a = a.reshape(S, S)
    y = np.array(U, dtype=np.float64, copy=True)
    for _ in range(nsteps):
        k = []
        for s in range(S):
            u = y.copy()
            for r in range(s):
                if a[s, r] != 0.0:
                    u += -dt * a[s, r] * k[r]
            k.append(evaluate(opd, gd, u, 1.0, 1.0, np.zeros_like(u)))
        upd = np.zeros_like(y)
        for s in range(S):
            if b[s] != 0.0:
                upd += -b[s] * dt * k[s]
        y = y + upd
    return y


def xdg_interface(nodes_xyz, periodic, k, rules, UA, UB, muA, muB, penalty_base, mode, alpha=1.0,
                  length_scales=None):
    """Level-set interface term, restated from XLaplace_Interface.InnerEdgeForm
    (XNSECommon/XLaplace.cs:229-297, GetPenalty :261-297, ComputeScaling :302-322,
    CoefficientUpdate :331-341) and the two-species scatter of
    NECQuadratureLevelSet.SaveIntegrationResults (NECQuadratureLevelSet.cs:622-661): for every
    cut cell and surface node, Ret(vA, vB) with (vA, vB) = (phi_n, 0) is added to species A's
    row n and with (0, phi_n) to species B's. Basis values come from the oracle's own basis
    (monomial representation); the surface rule is given. ``length_scales`` = (species A,
    species B) cell length scales: the penalty size factor is max(1 / len_A[j], 1 / len_B[j])
    of the cut cell j (GetPenalty, XLaplace.cs:261-297); None: the uncut cell's
    (Vol / (surface / 2), boundary faces counted twice). Returns (outA, outB)."""
    from math import comb
    h = [float(x[1] - x[0]) for x in nodes_xyz]
    n = [len(x) - 1 for x in nodes_xyz]
    Np = comb(k + 3, 3)
    detJ = np.prod([0.5 * hh for hh in h])
    sc = 1.0 / np.sqrt(detJ)
    if mode == 0:   # SWIP
        omA, omB = muB / (muA + muB), muA / (muA + muB)
        pen_mu = 2.0 * muA * muB / (muA + muB)
    else:           # SIP
        omA = omB = 0.5
        pen_mu = max(abs(muA), abs(muB)) * np.sign(muA)
    pdeg = max((k + 1.0) * (k + 3.0) / 3.0, (k + 1.0) ** 2)
    outA = np.zeros_like(np.asarray(UA, dtype=np.float64))
    outB = np.zeros_like(outA)
    cells, offs = rules["cells"], rules["offsets"]
    for r, cell in enumerate(cells):
        ijk = (cell // (n[1] * n[2]), (cell // n[2]) % n[1], cell % n[2])
        if length_scales is None:
            cj = 0.0
            for d in range(3):
                nb = 0 if periodic[d] else int(ijk[d] == 0) + int(ijk[d] == n[d] - 1)
                cj += (2.0 + nb) / h[d]
            size = 0.5 * cj
        else:
            size = max(1.0 / length_scales[0][cell], 1.0 / length_scales[1][cell])
        pen = penalty_base * pdeg * pen_mu * size
        sl = slice(offs[r], offs[r + 1])
        phi, dphi = basis_eval(3, k, rules["nodes"][sl])          # (Np, q), (Np, q, 3)
        N = rules["normals"][sl]
        w = rules["weights"][sl]
        phi = phi * sc
        gn = np.einsum("nqd,qd->nq", dphi * (sc * 2.0 / np.array(h)), N)   # grad(phi_n) . N
        cA, cB = UA[cell * Np:(cell + 1) * Np], UB[cell * Np:(cell + 1) * Np]
        uA, uB = cA @ phi, cB @ phi
        gA, gB = cA @ gn, cB @ gn
        jump = uA - uB
        flux = muA * omA * gA + muB * omB * gB
        retA = (flux - pen * jump) * phi + muA * omA * gn * jump      # vA = phi_n, vB = 0
        retB = -(flux - pen * jump) * phi + muB * omB * gn * jump     # vA = 0, vB = phi_n
        outA[cell * Np:(cell + 1) * Np] += alpha * (retA @ w)
        outB[cell * Np:(cell + 1) * Np] += alpha * (retB @ w)
    return outA, outB


def bsr_spmv(row_ptr, col_idx, values, alpha, x, beta, y):
    """BlockMsrMatrix.SpMV restated: y = beta*y + alpha*A*x; values[nnz, row_block, col_block]."""
    rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
    ci = np.ascontiguousarray(col_idx, dtype=np.int32)
    v = np.ascontiguousarray(values, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.array(y, dtype=np.float64, copy=True)
    assert v.ndim == 3 and y.size == (len(rp) - 1) * v.shape[1]
    lib().orc_bsr_spmv(len(rp) - 1, v.shape[1], v.shape[2], _p(rp), _p(ci), _p(v), alpha, _p(x), beta, _p(y))
    return y
