"""Result writers (bem3d_elastostatic_b200/output.py) against the reference's own
output text and against the parsing rules of its post-processing script."""
import os

import numpy as np

import oracle as O
from bem3d_elastostatic_b200.mesh import cube_grid_points, uniaxial_cube
from bem3d_elastostatic_b200.output import fortran_e, fortran_g, write_all, write_internal_points


def test_fortran_edit_descriptors():
    assert fortran_e(0.7874, 15, 7) == "  0.7874000E+00"
    assert fortran_e(-5.847155e-07, 15, 7) == " -0.5847155E-06"
    assert fortran_e(0.0, 15, 7) == "  0.0000000E+00"
    assert fortran_e(99.99983, 15, 7) == "  0.9999983E+02"
    assert fortran_e(1.0e100, 15, 7) == "  0.1000000+101"
    assert fortran_e(2.0e-4, 18, 8) == "    0.20000000E-03"
    assert fortran_g(1.0, 14, 7) == "  1.000000    "
    assert fortran_g(0.3, 14, 7) == " 0.3000000    "
    assert fortran_g(250000.0, 12, 5) == " 0.25000E+06"


def test_internal_points_text_matches_reference(cube8_golden):
    """Formatting the values of the reference's internal_points.dat reproduces its
    first 30 rows and its header byte for byte."""
    import zlib  # noqa: F401  (the fixture module decompresses the input)

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "cube8_golden.npz"))
    head = bytes(d["internal_points_head"]).decode().splitlines()
    rows = np.array([[float(v) for v in line.split()] for line in head[9:]])
    path = "/tmp/_ip_fmt_check.dat" if not os.environ.get("TMPDIR") else os.path.join(
        os.environ["TMPDIR"], "_ip_fmt_check.dat")
    write_internal_points(path, rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4:7].T, rows[:, 7:13].T,
                          rows[:, 13], rows[:, 14:17].T)
    got = open(path).read().splitlines()
    got[1] = head[1]  # the total count line carries this file's 30, not 1965
    assert got == head
    os.remove(path)


def _posproc_sections(path):
    """The section rules of the reference's parse_cube8_out (posproc.py:26-84): 4-field
    lines after 'BOUNDARY NODES COORDINATES', 'BOUNDARY NODES DISPLACEMENTS' and
    'INTERNAL POINTS DISPLACEMENTS'."""
    coords, disp, internal = {}, {}, {}
    section = None
    for line in open(path):
        s = line.strip()
        if not s:
            continue
        if "BOUNDARY NODES COORDINATES" in s:
            section = "COORDS"
            continue
        if "ELEMENT CONNECTIVITIES" in s:
            section = "CONNECT"
            continue
        if "BOUNDARY NODES DISPLACEMENTS" in s:
            section = "DISP"
            continue
        if "BOUNDARY ELEMENTS TRACTIONS" in s:
            section = "TRACTIONS"
            continue
        if "INTERNAL POINTS DISPLACEMENTS" in s:
            section = "INTERNAL"
            continue
        if "*" * 79 in s:
            if section == "INTERNAL":
                section = None
            continue
        p = s.split()
        if len(p) == 4 and p[0].isdigit():
            target = {"COORDS": coords, "DISP": disp, "INTERNAL": internal}.get(section)
            if target is not None:
                target[int(p[0])] = [float(v) for v in p[1:]]
    return coords, disp, internal


def test_result_files_read_back(tmp_path):
    mesh = uniaxial_cube(2, young=1.0, nu=0.3, points=cube_grid_points([0.25, 0.5, 0.75]))
    res = O.Oracle(mesh).run()
    paths = write_all(str(tmp_path), mesh, res)
    coords, disp, internal = _posproc_sections(paths["output"])
    assert len(coords) == mesh.n and len(disp) == mesh.n and len(internal) == mesh.l
    u = res["u"].reshape(-1, 3)
    got = np.array([disp[i + 1] for i in range(mesh.n)])
    assert np.abs(got - u).max() <= 5e-8 * np.abs(u).max()  # E18.8: 8 significant digits
    ip = np.loadtxt(paths["internal_points"])
    assert ip.shape == (mesh.l, 17)
    assert np.abs(ip[:, 9] - res["sigma"][2]).max() <= 1e-6 * np.abs(res["sigma"][2]).max()
    st = np.loadtxt(paths["stresses"])
    assert st.shape == (mesh.n, 14)
    assert np.abs(st[:, 6] - res["sigma_node"][2]).max() <= 1e-6
    dt = np.loadtxt(paths["disp_trac"])
    assert dt.shape == (6,)
