"""The two work decompositions that change how the hot path is scheduled, checked against
the plain form on the GPU, through the C ABI.

* CTA pairs (`umma_pair_kernel`, tcgen05.mma.cta_group::2): every tensor-core product
  of more than 128 rows runs as 256 x 256 tiles on clusters of two CTAs.  The products
  are the same BF16 terms accumulated in the same order as on single CTAs, so both
  mixed-precision solutions must be bitwise equal to the ones with BEM_UMMA_PAIR=0
  (read once per process, hence the two child processes).
* The split last wave of the regular assembly: the tiles past the last full wave run as
  pieces over shares of the element batches, merged from scratch in piece order.  The
  sums are reordered, so A and FI agree with the unsplit assembly (BEM_ASM_SPLIT=0) to
  rounding, row by row; a wrong scratch slot or merge would show at O(1).  At 4,614 DOF
  all 49 tiles are split (3 pieces each).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from bem3d_elastostatic_b200.mesh import uniaxial_cube

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_SOLVE = """
import sys
import numpy as np
sys.path.insert(0, sys.argv[2])
from bem3d_elastostatic_b200.api import Quadesth
from bem3d_elastostatic_b200.mesh import uniaxial_cube
q = Quadesth(uniaxial_cube(8))
q.precompute_element_geometry()
q.ghmat8()
xs = [q.solve_linear_system(p, tol=1e-14, max_iter=60) for p in ("bf16-ir", "fp32-ir")]
np.save(sys.argv[1], np.stack(xs))
q.close()
"""


def _solve_child(tmp_path, name, env_extra):
    out = str(tmp_path / f"{name}.npy")
    env = dict(os.environ, **env_extra)
    subprocess.run([sys.executable, "-c", _SOLVE, out, ROOT], env=env, check=True, timeout=600)
    return np.load(out)


def test_cta_pair_products_are_bitwise_equal_to_single_cta(tmp_path):
    pair = _solve_child(tmp_path, "pair", {"BEM_UMMA_PAIR": "1"})
    single = _solve_child(tmp_path, "single", {"BEM_UMMA_PAIR": "0"})
    assert pair.shape == single.shape == (2, 4614)
    assert np.array_equal(pair, single)


def test_split_assembly_wave_matches_the_unsplit_one(monkeypatch):
    from bem3d_elastostatic_b200.api import Quadesth

    mesh = uniaxial_cube(8)
    q = Quadesth(mesh)
    try:
        q.precompute_element_geometry()
        monkeypatch.setenv("BEM_ASM_SPLIT", "1")
        q.ghmat8()
        A1, F1 = q.system_rows(0, mesh.n)
        monkeypatch.setenv("BEM_ASM_SPLIT", "0")
        q.ghmat8()
        A0, F0 = q.system_rows(0, mesh.n)
    finally:
        q.close()
    rowmax = np.abs(A0).max(axis=1)
    assert np.all(np.abs(A1 - A0).max(axis=1) <= 1e-13 * rowmax)
    assert np.abs(F1 - F0).max() <= 1e-13 * np.abs(F0).max()
