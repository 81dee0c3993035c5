"""Plain numpy restatement of the multigrid V-cycle of ``bosss_b200_pmg_*`` (test helper).

Same algorithm as the device cycle, written with dense / scipy-sparse matrices:

* p-levels of degree K, K-1, ..., 1: the leading Np(k) x Np(k) sub-block of every cell block
  (hierarchical orthonormal basis); x = Dinv b, restriction of b - A x to the next level's
  modes, coarse solve, prolongation by zero padding, x += Dinv (b - A x);
* the piecewise-constant level (the blocks' (0, 0) entries) and its aggregates of 2x2x2 cells
  (ceil(n/2) per direction, Galerkin P^T A P with piecewise-constant P): two damped Jacobi
  sweeps (omega 0.7) from x = 0, restriction of the residual by aggregate sums, coarse solve,
  x += P x_c, two more sweeps;
* coarsest level (<= 100 unknowns): the dense inverse, or 40 Jacobi sweeps if it is singular.
"""
import numpy as np
import scipy.sparse as sp

OMEGA = 0.7
NU_H = 2
COARSE_MAX = 100
COARSE_SWEEPS = 40


def np_of(D, k):
    return (k + 1) * (k + 2) // 2 if D == 2 else (k + 1) * (k + 2) * (k + 3) // 6


def bsr_to_csr(rp, ci, vals):
    J, m = len(rp) - 1, vals.shape[1]
    rows, cols, data = [], [], []
    r = np.arange(m)
    for i in range(J):
        for b in range(rp[i], rp[i + 1]):
            j = ci[b]
            rows.append(np.repeat(i * m + r, m))
            cols.append(np.tile(j * m + r, m))
            data.append(vals[b].ravel())
    return sp.csr_matrix((np.concatenate(data), (np.concatenate(rows), np.concatenate(cols))), shape=(J * m, J * m))


def gauss_jordan(A):
    """Inverse by Gauss-Jordan with partial pivoting; None when a pivot is below 1e-12 of the
    largest entry (the device's singularity rule)."""
    A = np.array(A, dtype=np.float64)
    N = A.shape[0]
    I = np.eye(N)
    tiny = 1e-12 * np.abs(A).max()
    for k in range(N):
        p = k + int(np.argmax(np.abs(A[k:, k])))
        if not abs(A[p, k]) > tiny:
            return None
        A[[k, p]] = A[[p, k]]
        I[[k, p]] = I[[p, k]]
        d = A[k, k]
        A[k] /= d
        I[k] /= d
        f = A[:, k].copy()
        f[k] = 0.0
        A -= np.outer(f, A[k])
        I -= np.outer(f, I[k])
    return I


class VCycle:
    def __init__(self, rp, ci, vals, D, K, n, cell_ijk):
        """rp, ci, vals: the cell-block Jacobian (blocks [b, row, col]); n: cells per direction;
        cell_ijk: (J, D) integer cell indices of the cell order."""
        self.J = len(rp) - 1
        self.P = []
        for k in range(K, 0, -1):
            m = np_of(D, k)
            A = bsr_to_csr(rp, ci, vals[:, :m, :m])
            diag = np.stack([vals[rp[i], :m, :m] for i in range(self.J)])
            self.P.append({"m": m, "A": A, "Dinv": np.linalg.inv(diag)})
        A0 = bsr_to_csr(rp, ci, vals[:, :1, :1]).tocsr()
        self.H = [{"A": A0, "P": None}]
        ijk = np.asarray(cell_ijk).reshape(self.J, -1)
        dims = list(n)
        while self.H[-1]["A"].shape[0] > COARSE_MAX and max(dims) > 1:
            cdims = [(x + 1) // 2 for x in dims]
            agg = np.ravel_multi_index(tuple(ijk[:, d] // 2 for d in range(len(dims))), cdims)
            nf = self.H[-1]["A"].shape[0]
            Pm = sp.csr_matrix((np.ones(nf), (np.arange(nf), agg)), shape=(nf, int(np.prod(cdims))))
            Ac = (Pm.T @ self.H[-1]["A"] @ Pm).tocsr()
            self.H[-1]["Pnext"] = Pm
            self.H.append({"A": Ac})
            # cell indices of the aggregates, in their own lexicographic order
            ijk = np.stack(np.unravel_index(np.arange(int(np.prod(cdims))), cdims), axis=1)
            dims = cdims
        Ac = self.H[-1]["A"].toarray()
        self.coarse_inv = gauss_jordan(Ac) if Ac.shape[0] <= COARSE_MAX else None

    def _jacobi(self, A, b, x):
        d = A.diagonal()
        return x + OMEGA * (b - A @ x) / d

    def _cycle_h(self, l, b):
        L = self.H[l]
        A = L["A"]
        if l == len(self.H) - 1:
            if self.coarse_inv is not None:
                return self.coarse_inv @ b
            x = OMEGA * b / A.diagonal()
            for _ in range(COARSE_SWEEPS - 1):
                x = self._jacobi(A, b, x)
            return x
        x = OMEGA * b / A.diagonal()
        for _ in range(NU_H - 1):
            x = self._jacobi(A, b, x)
        Pm = L["Pnext"]
        xc = self._cycle_h(l + 1, Pm.T @ (b - A @ x))
        x = x + Pm @ xc
        for _ in range(NU_H):
            x = self._jacobi(A, b, x)
        return x

    def _bdiag(self, L, r):
        return np.einsum("jab,jb->ja", L["Dinv"], r.reshape(self.J, L["m"])).ravel()

    def _cycle_p(self, l, b):
        L = self.P[l]
        m = L["m"]
        x = self._bdiag(L, b)
        r = (b - L["A"] @ x).reshape(self.J, m)
        last = l == len(self.P) - 1
        mc = 1 if last else self.P[l + 1]["m"]
        bc = r[:, :mc].ravel()
        xc = self._cycle_h(0, bc) if last else self._cycle_p(l + 1, bc)
        x = x.reshape(self.J, m).copy()
        x[:, :mc] += xc.reshape(self.J, mc)
        x = x.ravel()
        return x + self._bdiag(L, b - L["A"] @ x)

    def apply(self, b):
        return self._cycle_p(0, b) if self.P else self._cycle_h(0, b)
