"""GPU parity of the sm_100a path against the CPU FP64 oracle, through the C-ABI.

Tolerances (FP64 plain path): relative L2 error <= 1e-12 against the oracle for
residuals, JVPs and VJPs at the small sizes and at the full config sizes (C1 64^2 k=2,
C2 32^3 k=3, C3 48^3 k=2 / 24^3 k=3 / 16^3 k=4); the VJP also against the transpose of
the oracle's assembled Jacobian (small grids) and through the adjoint identity
w.(J v) = (J^T w).v.
"""
import ctypes

import numpy as np
import pytest

from bosss_b200 import _capi as C
from bosss_b200 import operator as O
from bosss_b200 import problems as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


SMALL = [
    ("transport2d_8x6_k2", lambda: P.transport2d(n=8, k=2, seed=21)),
    ("transport2d_nonper_k3", lambda: P.transport2d(n=5, k=3, seed=22, periodic=False)),
    ("euler3d_4_k1", lambda: P.euler3d(n=4, k=1, seed=23)),
    ("euler3d_3_k3", lambda: P.euler3d(n=3, k=3, seed=24)),
    ("sip3d_4_k2", lambda: P.nonlinear_diffusion3d(n=4, k=2, seed=25)),
    ("sip3d_3_k3", lambda: P.nonlinear_diffusion3d(n=3, k=3, seed=26)),
    ("sip3d_3_k4", lambda: P.nonlinear_diffusion3d(n=3, k=4, seed=27)),
    ("sip3d_src_k2", lambda: P.nonlinear_diffusion3d(n=3, k=2, seed=28, source=1.5)),
    ("advdiff3d_4_k2", lambda: P.advection_diffusion3d(n=4, k=2, seed=29)),
    ("advdiff3d_3_k1_nonper", lambda: P.advection_diffusion3d(n=3, k=1, seed=30, periodic=False)),
    ("advdiff3d_3_k4", lambda: P.advection_diffusion3d(n=3, k=4, seed=31)),
]


@pytest.mark.parametrize("name,make", SMALL, ids=[s[0] for s in SMALL])
def test_residual_small(name, make):
    pr = make()
    ref = orc.evaluate(*pr.descs(), pr.U)
    with pr.evaluator() as ev:
        out = np.zeros(ev.n_codomain)
        ev.Evaluate(1.0, 0.0, out, pr.U)
    assert rel(out, ref) <= TOL, rel(out, ref)


@pytest.mark.parametrize("name,make", SMALL, ids=[s[0] for s in SMALL])
def test_jvp_small(name, make):
    pr = make()
    V = np.random.default_rng(1).uniform(-1, 1, pr.n_dofs)
    ref = orc.jvp(*pr.descs(), pr.U, V)
    with pr.evaluator() as ev:
        out = ev.jvp(pr.U, V)
    assert rel(out, ref) <= TOL, rel(out, ref)


@pytest.mark.parametrize("name,make", SMALL, ids=[s[0] for s in SMALL])
def test_vjp_is_transposed_jacobian(name, make):
    pr = make()
    opd, gd = pr.descs()
    A = orc.jacobian_dense(opd, gd, pr.U)
    W = np.random.default_rng(2).uniform(-1, 1, A.shape[0])
    ref = A.T @ W
    with pr.evaluator() as ev:
        out = ev.vjp(pr.U, W)
    assert rel(out, ref) <= TOL, rel(out, ref)


EULER_VARIANTS = [(k, kern) for k in (1, 2, 3, 4) for kern in (C.KERNEL_GENERIC, C.KERNEL_SLAB, C.KERNEL_FACES)]
_KNAME = {C.KERNEL_GENERIC: "generic", C.KERNEL_SLAB: "slab", C.KERNEL_FACES: "faces"}


@pytest.mark.parametrize("k,kernel", EULER_VARIANTS, ids=["k%d_%s" % (k, _KNAME[v]) for k, v in EULER_VARIANTS])
def test_euler_kernel_variants(k, kernel):
    """The 3D kernels (generic fused, register-blocked slab, slab volume + face-once face
    kernels) against the oracle: residual with alpha/beta, JVP, and VJP vs the transposed
    Jacobian."""
    pr = P.euler3d(n=3, k=k, seed=50 + k)
    opd, gd = pr.descs()
    r = np.random.default_rng(8)
    V = r.uniform(-1, 1, pr.n_dofs)
    W = r.uniform(-1, 1, pr.n_dofs)
    out0 = r.uniform(-1, 1, pr.n_dofs)
    ref = orc.evaluate(opd, gd, pr.U, alpha=0.5, beta=-1.5, out=out0)
    jref = orc.jvp(opd, gd, pr.U, V)
    A = orc.jacobian_dense(opd, gd, pr.U) if k <= 2 else None
    with pr.evaluator(kernel=kernel) as ev:
        out = out0.copy()
        ev.Evaluate(0.5, -1.5, out, pr.U)
        jv = ev.jvp(pr.U, V)
        jtw = ev.vjp(pr.U, W)
    assert rel(out, ref) <= TOL
    assert rel(jv, jref) <= TOL
    if A is not None:
        assert rel(jtw, A.T @ W) <= TOL
    assert abs(W @ jv - jtw @ V) <= 1e-12 * np.linalg.norm(W) * np.linalg.norm(jv)


def test_euler_full_size_slab_matches_generic():
    pr = P.euler3d(n=32, k=3, seed=2000)
    W = np.random.default_rng(9).uniform(-1, 1, pr.n_dofs)
    with pr.evaluator(kernel=C.KERNEL_GENERIC) as e1, pr.evaluator(kernel=C.KERNEL_SLAB) as e2, \
            pr.evaluator(kernel=C.KERNEL_FACES) as e3:
        r1, r2, r3 = np.zeros(pr.n_dofs), np.zeros(pr.n_dofs), np.zeros(pr.n_dofs)
        e1.Evaluate(1.0, 0.0, r1, pr.U)
        e2.Evaluate(1.0, 0.0, r2, pr.U)
        e3.Evaluate(1.0, 0.0, r3, pr.U)
        g1, g2, g3 = e1.vjp(pr.U, W), e2.vjp(pr.U, W), e3.vjp(pr.U, W)
    assert rel(r2, r1) <= TOL and rel(g2, g1) <= TOL
    assert rel(r3, r1) <= TOL and rel(g3, g1) <= TOL


def test_face_once_cell_ranges_match_whole_grid():
    """Face-once evaluation on cell ranges (each range computes the faces its cells need):
    three ranges one after the other equal the whole-grid launch, residual and VJP."""
    import torch
    pr = P.euler3d(n=6, k=3, seed=2301)
    W = np.random.default_rng(10).uniform(-1, 1, pr.n_dofs)
    with pr.evaluator(kernel=C.KERNEL_FACES) as ev:
        U = torch.from_numpy(pr.U).cuda()
        Wd = torch.from_numpy(W).cuda()
        whole_r, whole_g = torch.zeros_like(U), torch.zeros_like(U)
        part_r, part_g = torch.zeros_like(U), torch.zeros_like(U)
        L = C.lib()
        legacy = ctypes.c_void_p(C.CUDA_STREAM_LEGACY)
        J = pr.grid.NoOfCells
        C.check(L.bosss_b200_apply_device(ev.handle, C.MODE_RESIDUAL, 1.0, 0.0, C.ptr(U), None, C.ptr(whole_r), 0.0,
                                          0, J, legacy))
        C.check(L.bosss_b200_apply_device(ev.handle, C.MODE_VJP, 1.0, 0.0, C.ptr(U), C.ptr(Wd), C.ptr(whole_g), 0.0,
                                          0, J, legacy))
        for a, b in ((0, 72), (72, 150), (150, J)):
            C.check(L.bosss_b200_apply_device(ev.handle, C.MODE_RESIDUAL, 1.0, 0.0, C.ptr(U), None, C.ptr(part_r),
                                              0.0, a, b, legacy))
            C.check(L.bosss_b200_apply_device(ev.handle, C.MODE_VJP, 1.0, 0.0, C.ptr(U), C.ptr(Wd), C.ptr(part_g),
                                              0.0, a, b, legacy))
        torch.cuda.synchronize()
    assert torch.equal(whole_r, part_r) and torch.equal(whole_g, part_g)
    ref = orc.evaluate(*pr.descs(), pr.U)
    assert rel(whole_r.cpu().numpy(), ref) <= TOL
    assert rel(whole_g.cpu().numpy(), orc.vjp(*pr.descs(), pr.U, W)) <= TOL


def _transport3d(n, k, seed, periodic):
    g = O.Cartesian3DGrid(*[np.linspace(0, 1, n + 1)] * 3, periodic, periodic, periodic)
    op = O.DifferentialOperator(["u"], [], ["R"], O.QuadOrderFunc.FixedOrder(2 * k + 1))
    op.EquationComponents["R"].Add(O.ScalarTransportFlux((0.7, -0.4, 0.3), "u"))
    op.Commit()
    U = np.random.default_rng(seed).uniform(-1, 1, g.NoOfCells * O.np_of(3, k))
    return P.Problem("transport3d", op, g, [O.DGField(g, k, "u")], [O.DGField(g, k, "R")], U, {})


SCALAR3D = ([("transport_k%d_%s" % (k, "per" if per else "bnd"), (lambda k=k, per=per: _transport3d(3, k, 60 + k, per)))
             for k in (0, 1, 2, 3, 4) for per in (True, False)]
            + [("sip_k%d" % k, (lambda k=k: P.nonlinear_diffusion3d(n=3, k=k, seed=70 + k, source=0.5)))
               for k in (1, 2, 3, 4)]
            + [("advdiff_k%d_%s" % (k, "per" if per else "bnd"),
                (lambda k=k, per=per: P.advection_diffusion3d(n=3, k=k, seed=80 + k, periodic=per)))
               for k in (1, 2, 3, 4) for per in (True, False)])


@pytest.mark.parametrize("name,make", SCALAR3D, ids=[s[0] for s in SCALAR3D])
@pytest.mark.parametrize("kernel", [C.KERNEL_GENERIC, C.KERNEL_SLAB], ids=["generic", "slab"])
def test_scalar3d_kernel_variants(name, make, kernel):
    """Both 3D kernels on the scalar family (transport, SIP with nu(u) and source,
    advection-diffusion; periodic and boundary grids): residual with alpha/beta and JVP
    against the oracle, VJP against the transposed oracle Jacobian."""
    pr = make()
    opd, gd = pr.descs()
    r = np.random.default_rng(11)
    V = r.uniform(-1, 1, pr.n_dofs)
    W = r.uniform(-1, 1, pr.n_dofs)
    out0 = r.uniform(-1, 1, pr.n_dofs)
    ref = orc.evaluate(opd, gd, pr.U, alpha=0.5, beta=-1.5, out=out0)
    jref = orc.jvp(opd, gd, pr.U, V)
    A = orc.jacobian_dense(opd, gd, pr.U)
    with pr.evaluator(kernel=kernel) as ev:
        out = out0.copy()
        ev.Evaluate(0.5, -1.5, out, pr.U)
        jv = ev.jvp(pr.U, V)
        jtw = ev.vjp(pr.U, W)
    assert rel(out, ref) <= TOL, rel(out, ref)
    assert rel(jv, jref) <= TOL, rel(jv, jref)
    assert rel(jtw, A.T @ W) <= TOL, rel(jtw, A.T @ W)


def test_sip_full_size_slab_matches_generic():
    pr = P.nonlinear_diffusion3d(n=48, k=2, seed=3000)
    r = np.random.default_rng(9)
    V, W = r.uniform(-1, 1, pr.n_dofs), r.uniform(-1, 1, pr.n_dofs)
    with pr.evaluator(kernel=C.KERNEL_GENERIC) as e1, pr.evaluator(kernel=C.KERNEL_SLAB) as e2:
        r1, r2 = np.zeros(pr.n_dofs), np.zeros(pr.n_dofs)
        e1.Evaluate(1.0, 0.0, r1, pr.U)
        e2.Evaluate(1.0, 0.0, r2, pr.U)
        assert rel(r2, r1) <= TOL
        assert rel(e2.jvp(pr.U, V), e1.jvp(pr.U, V)) <= TOL
        assert rel(e2.vjp(pr.U, W), e1.vjp(pr.U, W)) <= TOL


def test_alpha_beta_semantics():
    pr = P.euler3d(n=3, k=2, seed=40)
    r = np.random.default_rng(3)
    out0 = r.uniform(-1, 1, pr.n_dofs)
    ref = orc.evaluate(*pr.descs(), pr.U, alpha=-0.7, beta=0.3, out=out0)
    with pr.evaluator() as ev:
        out = out0.copy()
        ev.Evaluate(-0.7, 0.3, out, pr.U)
    assert rel(out, ref) <= TOL


def test_globalid_cell_order():
    """Same operator on the GlobalID cell numbering gives the permuted residual."""
    a = P.advection_diffusion3d(n=4, k=2, seed=41, periodic=False)
    g2 = O.Cartesian3DGrid(np.linspace(0, 1, 5), np.linspace(0, 1, 5), np.linspace(0, 1, 5),
                           False, False, False, cell_order=C.CELLS_GLOBALID)
    ijk1, ijk2 = a.grid.cell_ijk(), g2.cell_ijk()
    pos = {tuple(t): i for i, t in enumerate(ijk1)}
    perm = np.array([pos[tuple(t)] for t in ijk2])
    Np = a.dom[0].Np
    U2 = a.U.reshape(-1, Np)[perm].ravel()
    dom2 = [O.DGField(g2, 2, "u")]
    cod2 = [O.DGField(g2, 2, "R")]
    with a.evaluator() as e1, a.op.GetEvaluatorEx(dom2, None, cod2) as e2:
        r1 = np.zeros(e1.n_codomain)
        r2 = np.zeros(e2.n_codomain)
        e1.Evaluate(1.0, 0.0, r1, a.U)
        e2.Evaluate(1.0, 0.0, r2, U2)
    assert rel(r2, r1.reshape(-1, Np)[perm].ravel()) <= TOL


FULL = [
    ("C1_transport2d_64x64_k2", lambda: P.transport2d(n=64, k=2, seed=1000)),
    ("C2_euler3d_32_k3", lambda: P.euler3d(n=32, k=3, seed=2000)),
    ("C3_sip3d_48_k2", lambda: P.nonlinear_diffusion3d(n=48, k=2, seed=3000)),
    ("C3_sip3d_24_k3", lambda: P.nonlinear_diffusion3d(n=24, k=3, seed=3001)),
    ("C3_sip3d_16_k4", lambda: P.nonlinear_diffusion3d(n=16, k=4, seed=3002)),
]


@pytest.mark.parametrize("name,make", FULL, ids=[s[0] for s in FULL])
def test_residual_full_size(name, make):
    pr = make()
    ref = orc.evaluate(*pr.descs(), pr.U)
    with pr.evaluator() as ev:
        out = np.zeros(ev.n_codomain)
        ev.Evaluate(1.0, 0.0, out, pr.U)
    assert rel(out, ref) <= TOL, rel(out, ref)


@pytest.mark.parametrize("name,make", FULL[:3], ids=[s[0] for s in FULL[:3]])
def test_adjoint_identity_full_size(name, make):
    """w.(J v) == (J^T w).v at full size (size-independent property)."""
    pr = make()
    r = np.random.default_rng(4)
    V = r.uniform(-1, 1, pr.n_dofs)
    W = r.uniform(-1, 1, pr.n_dofs)
    with pr.evaluator() as ev:
        jv = ev.jvp(pr.U, V)
        jtw = ev.vjp(pr.U, W)
    a, b = W @ jv, jtw @ V
    assert abs(a - b) <= 1e-11 * (np.linalg.norm(W) * np.linalg.norm(jv)), (a, b)


@pytest.mark.parametrize("name,make", FULL, ids=[s[0] for s in FULL])
def test_jvp_vjp_full_size_match_oracle(name, make):
    """J V and J^T W at the full config sizes against the oracle's exact products (the
    oracle's VJP differentiates W . Op(U) node by node, edge-centric, with dense tables)."""
    pr = make()
    opd, gd = pr.descs()
    r = np.random.default_rng(5)
    V = r.uniform(-1, 1, pr.n_dofs)
    W = r.uniform(-1, 1, pr.n_dofs)
    ref_jv = orc.jvp(opd, gd, pr.U, V)
    ref_jtw = orc.vjp(opd, gd, pr.U, W)
    with pr.evaluator() as ev:
        jv = ev.jvp(pr.U, V)
        jtw = ev.vjp(pr.U, W)
    assert rel(jv, ref_jv) <= TOL, rel(jv, ref_jv)
    assert rel(jtw, ref_jtw) <= TOL, rel(jtw, ref_jtw)


def test_jvp_matches_central_fd_full_size():
    """Central FD with eps = 1e-6 at full size, a sanity check of the linearisation.
    Coefficients of the orthonormal basis carry the scaling (2/h)^1.5 ~ 940 on the
    48^3 grid, so eps = 1e-6 moves u by ~1e-3 and central FD is accurate to ~1e-6
    only; in addition the SIP penalty picks nuMax = |nuA| > |nuB| ? nuA : nuB
    (ipLaplace.cs:181), a kink where FD is not a derivative. The exact comparison
    is test_jvp_full_size_matches_oracle."""
    pr = P.nonlinear_diffusion3d(n=48, k=2, seed=3000)
    V = np.random.default_rng(5).uniform(-1, 1, pr.n_dofs)
    eps = 1e-6
    with pr.evaluator() as ev:
        jv = ev.jvp(pr.U, V)
        fp = np.zeros(ev.n_codomain)
        fm = np.zeros(ev.n_codomain)
        ev.Evaluate(1.0, 0.0, fp, pr.U + eps * V)
        ev.Evaluate(1.0, 0.0, fm, pr.U - eps * V)
    fd = (fp - fm) / (2 * eps)
    # with the oracle's exact JVP on this state, FD(eps=1e-6) shows: median 1.0e-7 (the
    # eps^2 truncation term), 90th percentile 1.4e-5, 99.9th 3.4e-3 (kink)
    err = np.abs(jv - fd) / np.max(np.abs(jv))
    assert np.median(err) < 1e-6
    assert np.percentile(err, 90) < 1e-4
    assert np.percentile(err, 99.9) < 1e-2


def test_device_resident_path_matches_host_path():
    import torch
    pr = P.euler3d(n=8, k=2, seed=42)
    with pr.evaluator() as ev:
        out_h = np.zeros(ev.n_codomain)
        ev.Evaluate(1.0, 0.0, out_h, pr.U)
        U = torch.from_numpy(pr.U).cuda()
        out_d = torch.zeros(ev.n_codomain, dtype=torch.float64, device="cuda")
        ev.Evaluate(1.0, 0.0, out_d, U)
        torch.cuda.synchronize()
    assert np.array_equal(out_d.cpu().numpy(), out_h)


def test_check_nan_option():
    pr = P.euler3d(n=3, k=1, seed=43)
    U = pr.U.copy()
    U[5] = np.nan
    with pr.evaluator(check_nan=True) as ev:
        out = np.zeros(ev.n_codomain)
        with pytest.raises(C.BosssError) as ei:
            ev.Evaluate(1.0, 0.0, out, U)
        assert ei.value.code == C.ERR_NAN


def _bsr_from_dense_blocks(blocks, nbr):
    J, NB, Nc, Nd = blocks.shape
    rowptr = [0]
    cols, vals = [], []
    for j in range(J):
        seen = set()
        for b in range(NB):
            c = int(nbr[j, b])
            if c < 0 or c in seen:
                continue
            seen.add(c)
            cols.append(c)
            vals.append(blocks[j, b])
        rowptr.append(len(cols))
    return (np.array(rowptr, dtype=np.int64), np.array(cols, dtype=np.int32),
            np.ascontiguousarray(np.array(vals)).ravel())


def test_block_sparse_spmv_matches_dense():
    pr = P.nonlinear_diffusion3d(n=4, k=2, seed=44)
    opd, gd = pr.descs()
    blocks, nbr = orc.jacobian_blocks(opd, gd, pr.U)
    rp, ci, vals = _bsr_from_dense_blocks(blocks, nbr)
    Adense = orc.jacobian_dense(opd, gd, pr.U)
    J, NB, Nc, Nd = blocks.shape
    A = ctypes.c_void_p()
    C.check(C.lib().bosss_b200_bsr_create(J, J, Nc, Nd, C.ptr(rp), C.ptr(ci), C.ptr(vals), 0, ctypes.byref(A)))
    try:
        r = np.random.default_rng(7)
        x = r.uniform(-1, 1, J * Nd)
        y0 = r.uniform(-1, 1, J * Nc)
        y = y0.copy()
        C.check(C.lib().bosss_b200_bsr_spmv(A, 0.5, C.ptr(x), -2.0, C.ptr(y)))
        ref = 0.5 * Adense @ x - 2.0 * y0
        assert rel(y, ref) <= TOL
        # read back
        nnzb = ctypes.c_int64()
        C.check(C.lib().bosss_b200_bsr_get(A, None, None, None, None, ctypes.byref(nnzb), None, None, None))
        v2 = np.zeros(nnzb.value * Nc * Nd)
        C.check(C.lib().bosss_b200_bsr_get(A, None, None, None, None, None, None, None, C.ptr(v2)))
        assert np.array_equal(v2, vals)
    finally:
        C.lib().bosss_b200_bsr_destroy(A)


@pytest.mark.parametrize("case", ["euler_32", "sip_48_dirichlet", "advdiff_globalid"])
def test_host_pipeline_matches_device_path(case):
    """The host-buffer entry points stream their inputs and outputs by chunks of planes; the
    results equal the device-resident entry points' (residual with alpha/beta, JVP, VJP)."""
    import torch
    if case == "euler_32":
        pr = P.euler3d(n=32, k=3, seed=2000)
    elif case == "sip_48_dirichlet":
        pr = P.nonlinear_diffusion3d(n=48, k=2, seed=3000, source=1.0)
    else:
        n = 40
        g = O.Cartesian3DGrid(*[np.linspace(0, 1, n + 1)] * 3, True, False, True, cell_order=C.CELLS_GLOBALID)
        base = P.advection_diffusion3d(n=4, k=3, seed=5)
        U = np.random.default_rng(6).uniform(-1, 1, g.NoOfCells * O.np_of(3, 3))
        pr = P.Problem("advdiff_gid", base.op, g, [O.DGField(g, 3, "u")], [O.DGField(g, 3, "R")], U, {})
    r = np.random.default_rng(12)
    V = r.uniform(-1, 1, pr.n_dofs)
    out0 = r.uniform(-1, 1, pr.n_dofs)
    with pr.evaluator() as ev:
        host_r = out0.copy()
        ev.Evaluate(0.5, -1.5, host_r, pr.U)
        host_jv = ev.jvp(pr.U, V)
        host_g = ev.vjp(pr.U, V)
        Ud, Vd = torch.from_numpy(pr.U).cuda(), torch.from_numpy(V).cuda()
        dev_r = torch.from_numpy(out0).cuda()
        ev.Evaluate(0.5, -1.5, dev_r, Ud)
        dev_jv = ev.jvp(Ud, Vd)
        dev_g = ev.vjp(Ud, Vd)
        torch.cuda.synchronize()
    with pr.evaluator() as ev:
        comb_r, comb_g = ev.residual_vjp(pr.U, V, R=out0.copy(), alpha=0.5, beta=-1.5)
    for a, b in ((host_r, dev_r), (host_jv, dev_jv), (host_g, dev_g), (comb_r, dev_r), (comb_g, dev_g)):
        b = b.cpu().numpy()
        assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b))


def test_block_sparse_spmv_full_c3_pattern():
    """BlockMsrMatrix.SpMV at the C3 Jacobian's block pattern (48^3, k = 2: 110,592 block rows,
    7 blocks of 10 x 10 inside) against the oracle's restatement, y = beta*y + alpha*A*x."""
    pytest.importorskip("torch")
    rp, ci, vals = P.hex_block_pattern(48, 10)
    nbr = len(rp) - 1
    r = np.random.default_rng(12)
    x = r.uniform(-1, 1, nbr * 10)
    y0 = r.uniform(-1, 1, nbr * 10)
    ref = orc.bsr_spmv(rp, ci, vals, 0.5, x, -2.0, y0)
    A = O.BlockMsrMatrix.from_blocks(nbr, nbr, rp, ci, vals)
    try:
        y = A.SpMV(0.5, x, -2.0, y0.copy())
        assert rel(y, ref) <= 1e-14, rel(y, ref)
        y = A.SpMV(1.0, x, 0.0, np.full_like(y0, np.nan))   # beta = 0 overwrites
        assert rel(y, orc.bsr_spmv(rp, ci, vals, 1.0, x, 0.0, y0)) <= 1e-14
    finally:
        A.Dispose()


@pytest.mark.parametrize("shape", ["ragged_rectangular", "one_wide_row"])
def test_block_sparse_spmv_irregular_patterns(shape):
    """SpMV on patterns away from the Cartesian one: ragged rows, rectangular blocks, more
    block columns than rows and empty rows (sliced-ELL copy with zero padding), and a pattern
    with one very wide row (the ELL padding would not pay: the block-row kernel)."""
    r = np.random.default_rng(13)
    nbr, nbc, br, bc = (300, 410, 3, 5) if shape == "ragged_rectangular" else (200, 200, 4, 4)
    rows = []
    for i in range(nbr):
        if shape == "ragged_rectangular":
            k = 4 if r.random() < 0.9 else int(r.integers(0, 4))   # some short and empty rows
        else:
            k = 150 if i == 7 else 2
        rows.append(np.sort(r.choice(nbc, size=k, replace=False)))
    rp = np.zeros(nbr + 1, dtype=np.int64)
    rp[1:] = np.cumsum([len(c) for c in rows])
    ci = np.concatenate(rows).astype(np.int32)
    vals = r.uniform(-1, 1, (len(ci), br, bc))
    x = r.uniform(-1, 1, nbc * bc)
    y0 = r.uniform(-1, 1, nbr * br)
    ref = orc.bsr_spmv(rp, ci, vals, 0.5, x, -2.0, y0)
    A = O.BlockMsrMatrix.from_blocks(nbr, nbc, rp, ci, vals)
    try:
        y = A.SpMV(0.5, x, -2.0, y0.copy())
        assert rel(y, ref) <= 1e-14
    finally:
        A.Dispose()
