"""Generates tests/golden/cube8_golden.npz from the reference's shipped files.

Inputs (read here, in the build container, where the reference is mounted):
  cube8.dat            the reference's input for the 6 m cube (866 nodes, 216 quad9,
                       1965 internal points, tracked node 770)
  internal_points.dat  the reference's own output for that input
                       (stress_mod.f90:926-932 format: id, x, y, z, u(3), sigma(6),
                       von Mises, principal(3); E15.7)

Output: one compressed .npz with the input text (zlib), the output table and the
output file's first lines as text (its 9 header lines and 30 rows, for the writer's
format check), so the tests run where the reference is absent.  Run:
python tests/golden/make_golden.py
"""
import os
import sys
import zlib

import numpy as np

REF = os.environ.get("QUADESTH_REFERENCE", "/root/reference")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cube8_golden.npz")


def main():
    text = open(os.path.join(REF, "cube8.dat"), "rb").read()
    rows = []
    for line in open(os.path.join(REF, "internal_points.dat")):
        if line.startswith("#") or not line.strip():
            continue
        rows.append([float(v) for v in line.split()])
    table = np.array(rows, dtype=np.float64)
    assert table.shape == (1965, 17), table.shape
    head = "".join(open(os.path.join(REF, "internal_points.dat")).readlines()[:39]).encode()
    np.savez_compressed(OUT, cube8_zlib=np.frombuffer(zlib.compress(text, 9), dtype=np.uint8),
                        internal_points=table,
                        internal_points_head=np.frombuffer(head, dtype=np.uint8))
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    sys.exit(main())
