"""NumPy restatement of the coarse inverse of the two-level preconditioner
(test infrastructure).

Restates the blocked in-place Gauss-Jordan inversion with partial pivoting of
urban-sph_a100_b200/csrc/coarse.cu (k_gj_pivot, k_gj_pivot_row,
k_gj_panel_elim, k_gj_swap_rows, k_gj_copy_rows, k_gj_update) and the host
step of coarse_build that puts the inverse's columns back in order: per
panel of `panel` columns, every pivot column is swept inside the panel
(pivot = the largest |W[r, k]| for r >= k, lowest row on ties; the rows
swapped and the pivot row scaled in the panel's columns; every other row
eliminated in them), then the panel's row interchanges are applied to the
other columns and those columns take the rank-`panel` update
W[:, J] = (pivot rows zeroed) W[:, J] + N Bk.  Column c of the inverse is
column col[c] of W, col being the identity with the swaps (k, piv[k])
applied for k = m-1 down to 0.
"""
import numpy as np


def blocked_gauss_jordan(A, panel=64):
    """Returns (inverse, pivots) of the square matrix A."""
    W = np.array(A, dtype=np.float64, copy=True)
    m = W.shape[0]
    piv = np.zeros(m, dtype=np.int64)
    for k0 in range(0, m, panel):
        kb = min(panel, m - k0)
        K = slice(k0, k0 + kb)
        for k in range(k0, k0 + kb):
            col = np.abs(W[k:, k])
            p = k + int(np.argmax(col))          # first maximum: the lowest row
            if not col[p - k] > 0:
                raise np.linalg.LinAlgError("singular coarse operator")
            piv[k] = p
            a, b = W[k, K].copy(), W[p, K].copy()
            if p != k:
                W[p, K] = a
            inv = 1.0 / b[k - k0]
            W[k, K] = b * inv
            W[k, k] = inv
            rk = W[k, K].copy()
            for i in range(m):
                if i == k:
                    continue
                f = W[i, k]
                if f == 0.0:
                    continue
                row = W[i, K] - f * rk
                row[k - k0] = -f * rk[k - k0]
                W[i, K] = row
        if kb < m:
            J = np.ones(m, dtype=bool)
            J[K] = False
            for k in range(k0, k0 + kb):
                p = piv[k]
                if p != k:
                    t = W[k, J].copy()
                    W[k, J] = W[p, J]
                    W[p, J] = t
            Bk = W[K, :].copy()
            N = W[:, K].copy()
            base = W.copy()
            base[K, :] = 0.0
            W[:, J] = base[:, J] + (N @ Bk)[:, J]
    col = np.arange(m)
    for k in range(m - 1, -1, -1):
        p = piv[k]
        col[k], col[p] = col[p], col[k]
    return W[:, col], piv
