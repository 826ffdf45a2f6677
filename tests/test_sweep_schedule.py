"""CPU restatement of the block-inverse triangular sweeps of csrc/lu.cu
(`sweep_inv_kernel`, `diag_inv_kernel`), the mixed-precision modes' preconditioner
solve, on factors in the library's storage.

T = A^T = P L U is factored in place in S (the column-major A): U in S's lower
triangle, the unit multipliers in its strict upper triangle.  So A = U^T L^T P^T and
A x = b is solved as
  forward:  tril(S) y = b          (blocks first to last, diag_inv's "lower" inverses)
  backward: (striu(S) + I) z = y   (blocks last to first, the unit-upper inverses)
  x = P z                          (permute_kernel with the gather form of P).
A sweep over 128-row blocks runs as one cooperative launch of G CTAs: step s solves
block k(s) and is owned by CTA s mod G, which keeps the partial right-hand sides w of
its blocks; once block s is published, every CTA subtracts the tiles S(k(sx), k(s)) y_s
from its blocks sx > s, the owner of step s + 1 first, which then solves
y_{s+1} = Dinv_{s+1} w_{s+1}.  The restatement replays that order for several G and
checks the sweeps and the whole solve against LAPACK.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from test_lu_schedule import window_lu  # noqa: E402

NB = 128  # kSolveBlock


def sweep_inv(S, b, upper, G):
    n = S.shape[0]
    nblk = (n + NB - 1) // NB
    blocks = [slice(k * NB, min(n, (k + 1) * NB)) for k in range(nblk)]

    def bidx(s):
        return nblk - 1 - s if upper else s

    def dinv(k):  # diag_inv_kernel: the inverse of the block's triangle
        D = S[blocks[k], blocks[k]]
        M = np.triu(D, 1) + np.eye(D.shape[0]) if upper else np.tril(D)
        return np.linalg.inv(M)

    w = {s: b[blocks[bidx(s)]].copy() for s in range(nblk)}  # owned by CTA s % G
    y = {0: dinv(bidx(0)) @ w[0]}
    for s in range(nblk - 1):
        for g in range(G):
            first = s + 1 + (g - (s + 1)) % G  # this CTA's first step after s
            for sx in range(first, nblk, G):
                w[sx] -= S[blocks[bidx(sx)], blocks[bidx(s)]] @ y[s]
                if sx == s + 1:  # the owner of the next step solves it at once
                    y[sx] = dinv(bidx(sx)) @ w[sx]
    x = np.empty(n)
    for s in range(nblk):
        x[blocks[bidx(s)]] = y[s]
    return x


@pytest.mark.parametrize("n,G", [(1000, 1), (1000, 3), (1000, 148), (300, 7), (129, 2)])
def test_block_inverse_sweeps_solve_the_triangles(n, G):
    rng = np.random.default_rng(3)
    S = rng.standard_normal((n, n)) / np.sqrt(n) + 3.0 * np.eye(n)
    b = rng.standard_normal(n)
    y = sweep_inv(S, b, upper=False, G=G)
    assert np.abs(np.tril(S) @ y - b).max() <= 1e-12 * np.abs(b).max()
    z = sweep_inv(S, y, upper=True, G=G)
    assert np.abs((np.triu(S, 1) + np.eye(n)) @ z - y).max() <= 1e-12 * np.abs(y).max()


@pytest.mark.parametrize("n,nb", [(700, 256), (1000, 512)])
def test_sweeps_solve_the_factored_system(n, nb):
    rng = np.random.default_rng(4)
    A = rng.standard_normal((n, n)) / np.sqrt(n) + 2.0 * np.eye(n)
    b = rng.standard_normal(n)
    S, piv = window_lu(A, nb=nb)
    z = sweep_inv(S, sweep_inv(S, b, upper=False, G=148), upper=True, G=148)
    x = z.copy()
    for i in range(n - 1, -1, -1):  # x = P z, P = tau_0 tau_1 ... tau_{n-1}
        x[[i, piv[i]]] = x[[piv[i], i]]
    x_ref = np.linalg.solve(A, b)
    assert np.abs(x - x_ref).max() <= 1e-10 * np.abs(x_ref).max()
