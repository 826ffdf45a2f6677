"""CPU restatement of the window-pivoted LU schedule of csrc/lu.cu (the FP32 and BF16
factorisations), in the library's storage: S is the column-major A, T = S^T is
factored with row pivoting (column pivoting of S), U in S's lower triangle and the
unit multipliers in its strict upper triangle.  The test replays the launch order --
window factorisation of each 32-wide sub-panel within its 32 x 32 diagonal block,
interchanges on the panel's rows, TRSM and GEMM restricted to the panel's diagonal
block, the panel's interchanges on every other row at once, the 128 x 128 inverses of
the diagonal block's triangles (the lower one through the unit-upper inverse of
(Lu^T)), the full triangle inverses assembled from them block column by block column,
and the two TRSMs as single products B := W^{-1} B and Y = X U^{-1} -- and checks
P T = L U in FP64."""
import numpy as np
import pytest


def _unit_upper_inv(U):
    k = U.shape[0]
    return np.linalg.inv(np.triu(U, 1) + np.eye(k))


def window_lu(A, nb=512, W=32, B=128):
    n = A.shape[0]
    S = A.copy()
    piv = np.zeros(n, dtype=int)
    for j0 in range(0, n, nb):
        jb = min(nb, n - j0)
        t0 = j0 + jb
        cend = t0  # the sub-panels stop at the panel's diagonal block
        for r0 in range(j0, t0, W):
            w = min(W, t0 - r0)
            D = S[r0:r0 + w, r0:r0 + w].T.copy()  # D[c, j] = S[r0 + j, r0 + c]
            p_loc = []
            for t in range(w):
                p = t + int(np.argmax(np.abs(D[t:, t])))
                p_loc.append(p)
                D[[t, p], :] = D[[p, t], :]
                l = D[t + 1:, t] / D[t, t]
                D[t + 1:, t] = l
                D[t + 1:, t + 1:] -= np.outer(l, D[t, t + 1:])
            X = S[r0:r0 + w, r0 + w:cend].copy()  # the sub-panel's other block columns
            for t in range(w):
                X[t] /= D[t, t]
                X[t + 1:] -= np.outer(D[t, t + 1:], X[t])
            S[r0:r0 + w, r0 + w:cend] = X
            piv[r0:r0 + w] = r0 + np.array(p_loc)
            # the panel's rows only, except in the last panel (no permutation after it)
            rows = list(range(j0 if t0 < n else 0, r0)) + list(range(r0 + w, t0 if t0 < n else n))
            for t in range(w):
                a, b = r0 + t, piv[r0 + t]
                if a != b:
                    S[np.ix_(rows, [a, b])] = S[np.ix_(rows, [b, a])]
            S[r0:r0 + w, r0:r0 + w] = D.T
            q0 = r0 + w
            if t0 > q0:
                S[q0:t0, r0:r0 + w] = S[q0:t0, r0:r0 + w] @ _unit_upper_inv(S[r0:r0 + w, r0:r0 + w])
                S[q0:t0, q0:cend] -= S[q0:t0, r0:r0 + w] @ S[r0:r0 + w, q0:cend]
        if t0 < n:
            rows = list(range(0, j0)) + list(range(t0, n))  # permute_panel_kernel
            perm = np.arange(jb)
            for t in range(jb):
                p = piv[j0 + t] - j0
                perm[[t, p]] = perm[[p, t]]
            S[np.ix_(rows, j0 + np.arange(jb))] = S[np.ix_(rows, j0 + perm)]
            Dg = S[j0:t0, j0:t0]
            # 128-block inverses (panel_inv_f32_kernel): unit upper, and the lower
            # triangle's through the unit-upper inverse of (Lu^T)
            Vu, Wl = [], []
            for b0 in range(0, jb, B):
                bb = min(B, jb - b0)
                Vu.append(_unit_upper_inv(Dg[b0:b0 + bb, b0:b0 + bb]))
                Wbb = np.tril(Dg[b0:b0 + bb, b0:b0 + bb])
                rd = np.diag(Wbb)
                Wl.append(_unit_upper_inv(Wbb.T / rd[:, None]).T / rd[:, None])
            # the full inverses, block column by block column
            XU = np.zeros((jb, jb))
            XL = np.zeros((jb, jb))
            for k, b0 in enumerate(range(0, jb, B)):
                bb = min(B, jb - b0)
                XU[b0:b0 + bb, b0:b0 + bb] = Vu[k]
                XL[b0:b0 + bb, b0:b0 + bb] = Wl[k]
                if b0:
                    XU[:b0, b0:b0 + bb] = -(XU[:b0, :b0] @ Dg[:b0, b0:b0 + bb]) @ Vu[k]
                    XL[b0:b0 + bb, :b0] = -Wl[k] @ (Dg[b0:b0 + bb, :b0] @ XL[:b0, :b0])
            S[j0:t0, t0:] = XL @ S[j0:t0, t0:]  # B := W^{-1} B
            Y = S[t0:, j0:t0] @ XU  # Y = X U^{-1}
            S[t0:, j0:t0] = Y
            S[t0:, t0:] -= Y @ S[j0:t0, t0:]
    return S, piv


@pytest.mark.parametrize("n,nb", [(700, 512), (1300, 1024), (700, 256)])
def test_window_pivoted_schedule_factors_the_matrix(n, nb):
    """Panels of 512, 1024 and 256 with a ragged last panel and last 128-block."""
    rng = np.random.default_rng(1)
    A = rng.standard_normal((n, n)) + 4.0 * np.eye(n)
    S, piv = window_lu(A, nb=nb)
    assert np.all((piv >= np.arange(n) // 32 * 32) & (piv < np.minimum(np.arange(n) // 32 * 32 + 32, n)))
    T = A.T.copy()
    for i in range(n):  # P T with P = tau_0 tau_1 ... applied in order
        T[[i, piv[i]]] = T[[piv[i], i]]
    L = np.triu(S, 1).T + np.eye(n)
    U = np.tril(S).T
    assert np.abs(T - L @ U).max() <= 1e-11 * np.abs(A).max()
