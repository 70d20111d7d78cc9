"""Writes the small input fixtures under tests/golden/.

box_10_8_6.geom: a 10 x 8 x 6 dipole box as an ADDA-style text dipole list
("x y z" per line, x fastest, '#' comments), the same dipole set as the
reference's test fixture DDA/box_10_8_6.geom.  tests/test_oracle.py checks
the equality against the reference file when the reference tree is present.
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def box_geom(nx=10, ny=8, nz=6):
    lines = ["#box dipole list", "#box size: %dx%dx%d" % (nx, ny, nz)]
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                lines.append("%d %d %d" % (x, y, z))
    return "\n".join(lines) + "\n"


if __name__ == "__main__":
    with open(os.path.join(HERE, "box_10_8_6.geom"), "w") as f:
        f.write(box_geom())
