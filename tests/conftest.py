import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cube8_mesh():
    import zlib

    import numpy as np

    from bem3d_elastostatic_b200.mesh import read_quadesth

    g = np.load(os.path.join(ROOT, "tests", "golden", "cube8_golden.npz"))
    text = zlib.decompress(g["cube8_zlib"].tobytes()).decode()
    return read_quadesth(text, is_text=True)


@pytest.fixture(scope="session")
def cube8_golden():
    import numpy as np

    return np.load(os.path.join(ROOT, "tests", "golden", "cube8_golden.npz"))["internal_points"]


@pytest.fixture(scope="session")
def cube8_oracle_solution(cube8_mesh):
    """The oracle's full run on the reference's own input (cached per session)."""
    import oracle as O

    orc = O.Oracle(cube8_mesh)
    return orc, orc.run()
