"""Batched systems (bem_batch_*) against the oracle, system by system and load case
by load case: A and FI as the single-system assembly, solutions to the FP64 bar."""
import numpy as np
import pytest

import oracle as O
from bem3d_elastostatic_b200.mesh import box_batch, loaded_box

pytestmark = pytest.mark.gpu


def _oracle_case(mesh, bc):
    mesh.bc = np.asfortranarray(bc)
    orc = O.Oracle(mesh)
    A, FI = orc.ghmat8()
    x, info = orc.solve(A.copy(order="F"), FI)
    assert info == 0
    return A, FI, x


@pytest.fixture(scope="module")
def small_batch():
    rng = np.random.default_rng(7)
    systems = [loaded_box(1.0, 0.7, 1.3, 1, 0.3, 1.0, rng.standard_normal((3, 3))),
               loaded_box(0.6, 1.8, 0.9, 2, 0.12, 1.0, rng.standard_normal((3, 3))),
               loaded_box(1.5, 1.5, 0.5, 3, 0.41, 1.0, rng.standard_normal((3, 3))),
               loaded_box(1.0, 1.0, 1.0, 2, 0.25, 2.0, rng.standard_normal((3, 3)))]
    return systems


def test_batch_assembly_and_fp32_ir(small_batch):
    from bem3d_elastostatic_b200.api import Batch

    b = Batch()
    for mesh, bcs in small_batch:
        b.add(mesh, bcs)
    b.assemble()
    info = b.solve("fp32-ir", tol=1e-14, max_iter=8)
    assert info["singular"] == 0 and info["lu_threads"] in (256, 512)
    for i, (mesh, bcs) in enumerate(small_batch):
        A, F = b.system(i)
        x = b.solution(i)
        for r, bc in enumerate(bcs):
            Ar, Fr, xr = _oracle_case(mesh, bc)
            rowmax = np.abs(Ar).max(axis=1, keepdims=True)
            assert (np.abs(A - Ar) / rowmax).max() <= 1e-12, (i, r)
            assert np.abs(F[:, r] - Fr).max() <= 1e-12 * np.abs(Fr).max(), (i, r)
            err = np.abs(x[:, r] - xr).max() / np.abs(xr).max()
            assert err <= 1e-10, (i, r, err)
    assert info["max_backward_error"] <= 1e-14
    b.close()


def test_batch_fp64_and_graph_replay(small_batch):
    from bem3d_elastostatic_b200.api import Batch

    b = Batch()
    for mesh, bcs in small_batch:
        b.add(mesh, bcs)
    b.assemble()
    b.solve("fp64")
    x1 = [b.solution(i) for i in range(len(small_batch))]
    b.solve("fp64")  # the captured graph replayed
    for i, (mesh, bcs) in enumerate(small_batch):
        x2 = b.solution(i)
        assert np.array_equal(x1[i], x2)
        _, _, xr = _oracle_case(mesh, bcs[1])
        assert np.abs(x2[:, 1] - xr).max() <= 1e-10 * np.abs(xr).max()
    b.close()


def test_batch_rejects_inconsistent_supports():
    from bem3d_elastostatic_b200 import _lib
    from bem3d_elastostatic_b200.api import Batch

    mesh, bcs = loaded_box(1.0, 1.0, 1.0, 2, 0.3)
    bc = bcs[0].copy(order="F")
    # two bottom elements prescribe different u_z at a shared node
    bottom = [e for e in range(mesh.ne) if mesh.kode[3 * e + 2] == 0]
    bc[2::3, bottom[0]] = 1e-3
    b = Batch()
    with pytest.raises(_lib.BemError):
        b.add(mesh, [bc])
    b.close()


def test_box_batch_sizes():
    systems = box_batch(16, loads=2)
    assert all(len(bcs) == 2 for _, bcs in systems)
    assert all(78 <= m.ndof <= 2598 for m, _ in systems)
