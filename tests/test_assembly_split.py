"""CPU restatement of the split last wave of the regular assembly (csrc/assembly.cu:
`plan_tail`, the pieces of `ghmat_regular_kernel`, `tail_merge_cols_kernel`,
`tail_merge_fd_kernel`), on the element batches of a real mesh.

The tiles past the last full wave of 148 CTAs run as pp pieces each, piece p over the
batches [nb p / pp, nb (p + 1) / pp); piece 0 adds into A as an unsplit tile does,
pieces >= 1 add into scratch whose columns are the piece's node slots, and the merges
add the pieces' columns (summed in piece order) and their FI / diagonal partial sums.
The restatement checks the plan (piece count, a partition of the batches, slots for
every node a piece touches) and that the merged columns of A equal the unsplit sums
(the FI and diagonal partial sums merge the same way, one row each).
"""
import numpy as np
import pytest

from bem3d_elastostatic_b200.mesh import uniaxial_cube

KBATCH, MAX_PIECES, SMS = 8, 8, 148


def build_batches(n, ne, nconec, kconec):
    """context.cu build_batches: elements in order into the first of the 32 most recent
    not-full batches that holds none of their nodes."""
    batches, node_batches, open_ = [], [[] for _ in range(n)], []
    for e in range(ne):
        nodes = kconec[:nconec[e], e] - 1
        chosen = next((b for b in open_ if not any(b in node_batches[v] for v in nodes)), -1)
        if chosen < 0:
            chosen = len(batches)
            batches.append([])
            open_.append(chosen)
            if len(open_) > 32:
                open_.pop(0)
        batches[chosen].append(e)
        for v in nodes:
            node_batches[v].append(chosen)
        if len(batches[chosen]) == KBATCH:
            open_.remove(chosen)
    return batches


def plan(tiles, nbatches):
    rem = tiles % SMS
    if rem == 0:
        return 1, tiles
    return max(1, min(MAX_PIECES, SMS // rem, nbatches)), tiles - rem


def piece_slots(batches, nconec, kconec, n, pp):
    nb = len(batches)
    slots = []
    for p in range(1, pp):
        b0, b1 = nb * p // pp, nb * (p + 1) // pp
        nodes = sorted({int(v) - 1 for b in batches[b0:b1] for e in b for v in kconec[:nconec[e], e]})
        sl = np.full(n, -1)
        sl[nodes] = np.arange(len(nodes))
        slots.append(sl)
    return slots


@pytest.mark.parametrize("m", [2, 4, 8])
def test_split_wave_plan_and_merge(m):
    mesh = uniaxial_cube(m)
    n, ne = mesh.n, mesh.ne
    nconec = np.asarray(mesh.nconec)
    kconec = np.asarray(mesh.kconec)  # (9, ne), 1-based
    assert kconec.shape == (9, ne)
    batches = build_batches(n, ne, nconec, kconec)
    nb = len(batches)
    tiles = (n + 31) // 32
    pp, tail0 = plan(tiles, nb)
    assert 2 <= pp <= MAX_PIECES and tail0 + (tiles - tail0) * pp <= 2 * SMS
    # the pieces partition the batch list
    ranges = [(nb * p // pp, nb * (p + 1) // pp) for p in range(pp)]
    assert ranges[0][0] == 0 and ranges[-1][1] == nb
    assert all(ranges[i][1] == ranges[i + 1][0] for i in range(pp - 1))
    slots = piece_slots(batches, nconec, kconec, n, pp)

    # a synthetic element block per (collocation row, element, node of the element, dof)
    def block(rows, e, k, ld):
        return np.sin(0.37 * rows + 1.3 * e + 0.7 * k + 0.11 * ld)

    ndof = 3 * n
    A_ref = np.zeros((ndof, ndof))
    A = np.zeros((ndof, ndof))
    for t in range(tail0, tiles):
        rows = np.arange(96 * t, min(ndof, 96 * t + 96))  # the tile's rows of A
        scratch = [np.zeros((96, 3 * int((slots[p - 1] >= 0).sum()))) for p in range(1, pp)]
        for p, (b0, b1) in enumerate(ranges):
            for b in range(b0, b1):
                for e in batches[b]:
                    for k in range(nconec[e]):
                        node = kconec[k, e] - 1
                        for ld in range(3):
                            v = block(rows, e, k, ld)
                            A_ref[rows, 3 * node + ld] += v
                            if p == 0:
                                A[rows, 3 * node + ld] += v
                            else:
                                sl = slots[p - 1][node]
                                assert sl >= 0  # every node of the piece's elements has a slot
                                scratch[p - 1][:rows.size, 3 * sl + ld] += v
        # tail_merge_cols_kernel: per (node, dof) column segment, pieces summed in order
        for node in range(n):
            for ld in range(3):
                acc, hit = np.zeros(96), False
                for p in range(1, pp):
                    sl = slots[p - 1][node]
                    if sl >= 0:
                        acc += scratch[p - 1][:, 3 * sl + ld]
                        hit = True
                if hit:
                    A[rows, 3 * node + ld] += acc[:rows.size]
    assert np.abs(A - A_ref).max() <= 1e-12 * np.abs(A_ref).max()
