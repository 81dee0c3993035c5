"""The multigrid V-cycle's algorithm on the CPU (numpy restatement ``pmg_reference``, the
oracle's cell-block Jacobian of the nonlinear diffusion operator): as a preconditioner of
GMRES it needs a third of block-Jacobi's iterations at 8^3, and its iteration count grows
less from 4^3 to 8^3 than block-Jacobi's (which doubles with 1/h; at 12^3 -> 24^3 the V-cycle's
count is flat, 94 -> 99 to 1e-8, too slow a case for this suite)."""
import numpy as np
import scipy.sparse.linalg as spla

import pmg_reference as PR
from bosss_b200 import problems as P
from oracle import oracle as orc


def _system(n, k):
    pr = P.nonlinear_diffusion3d(n=n, k=k, seed=3000, source=1.0)
    opd, gd = pr.descs()
    B, nbr = orc.jacobian_blocks(opd, gd, pr.U)
    J, NB, m, _ = B.shape
    rp = np.zeros(J + 1, dtype=np.int64)
    ci, vals = [], []
    for i in range(J):
        cols = [int(c) for c in nbr[i] if c >= 0]
        for s_, c in enumerate(nbr[i]):
            if c >= 0:
                ci.append(int(c))
                vals.append(B[i, s_])
        rp[i + 1] = rp[i] + len(cols)
    vals = np.array(vals)
    ci = np.array(ci)
    A = PR.bsr_to_csr(rp, ci, vals)
    rhs = -orc.evaluate(opd, gd, pr.U)
    ijk = np.stack(np.unravel_index(np.arange(J), (n, n, n)), axis=1)
    return A, rhs, rp, ci, vals, ijk


def _iters(A, rhs, M):
    it = [0]

    def cb(_):
        it[0] += 1
    N = A.shape[0]
    x, info = spla.gmres(A, rhs, M=spla.LinearOperator((N, N), matvec=M), rtol=1e-6, restart=50, maxiter=40,
                         callback=cb, callback_type="pr_norm")
    assert info == 0
    assert np.linalg.norm(rhs - A @ x) <= 1e-6 * np.linalg.norm(rhs) * 1.01
    return it[0]


def test_vcycle_iterations_do_not_grow_with_the_grid():
    counts = {}
    for n in (4, 8):
        A, rhs, rp, ci, vals, ijk = _system(n, 2)
        V = PR.VCycle(rp, ci, vals, 3, 2, [n, n, n], ijk)
        J, m = len(rp) - 1, vals.shape[1]
        Dinv = np.linalg.inv(np.stack([vals[rp[i]] for i in range(J)]))

        def bj(v):
            return np.einsum("jab,jb->ja", Dinv, v.reshape(J, m)).ravel()
        counts[n] = (_iters(A, rhs, V.apply), _iters(A, rhs, bj))
    (mg4, bj4), (mg8, bj8) = counts[4], counts[8]
    assert mg8 * 3 <= bj8, counts
    assert bj8 >= 2 * bj4, counts
    assert mg8 / mg4 <= 0.8 * bj8 / bj4, counts
