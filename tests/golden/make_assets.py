"""Writes the small scene / mesh / patch files of tests/test_assets.py into
tests/golden/assets/ (project-authored test content: a unit cube and a
tetrahedron as OBJ, two bicubic patches in the bezmesh .dat layout, and a
.scene file that uses every command of the reference's scene format).

    python tests/golden/make_assets.py
"""
import os

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "assets")

CUBE = """# unit cube: 8 positions, 4 texture coordinates, 6 normals, 6 quads
o cube
v -0.5 -0.5 -0.5
v  0.5 -0.5 -0.5
v  0.5  0.5 -0.5
v -0.5  0.5 -0.5
v -0.5 -0.5  0.5
v  0.5 -0.5  0.5
v  0.5  0.5  0.5
v -0.5  0.5  0.5
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 -1
vn 0 0 1
vn 0 -1 0
vn 0 1 0
vn -1 0 0
vn 1 0 0
s off
f 1/1/1 4/4/1 3/3/1 2/2/1
f 5/1/2 6/2/2 7/3/2 8/4/2
f 1/1/3 2/2/3 6/3/3 5/4/3
f 4/1/4 8/2/4 7/3/4 3/4/4
f 1/1/5 5/2/5 8/3/5 4/4/5
f 2/1/6 3/2/6 7/3/6 6/4/6
"""

TETRA = """# tetrahedron without normals; the last face uses negative indices
v 0 0 0
v 1 0 0
v 0 1 0
v 0 0 1
f 1 3 2
f 1 2 4
f 1 4 3
f -3 -2 -1
"""


def patch_lines(z_of):
    rows = []
    for r in range(4):
        pts = []
        for c in range(4):
            x, y = c / 3.0 * 2.0 - 1.0, r / 3.0 * 2.0 - 1.0
            pts.append(f"{x:.6f} {y:.6f} {z_of(r, c):.6f}")
        rows.append(" ".join(pts))
    return rows


def main():
    os.makedirs(HERE, exist_ok=True)
    with open(os.path.join(HERE, "cube.obj"), "w") as f:
        f.write(CUBE)
    with open(os.path.join(HERE, "tetra.obj"), "w") as f:
        f.write(TETRA)
    with open(os.path.join(HERE, "two_patches.dat"), "w") as f:
        f.write("# two bicubic patches: a flat one and a bump\n")
        for z_of in (lambda r, c: 0.0, lambda r, c: 1.5 if (r in (1, 2) and c in (1, 2)) else -0.25):
            f.write('Patch "bicubic"\n')
            for line in patch_lines(z_of):
                f.write(line + "\n")
    with open(os.path.join(HERE, "test.scene"), "w") as f:
        f.write("""# every command of the scene format
camera [ 0 1 5 ] [ 0 0 0 ] [ 0 1 0 ]
camera_fov 50
zNear 0.1
zFar 50
light [ 2 3 4 ] [ 1 1 1 ] [ 1 1 1 ] 20
material [ 0.1 0.1 0.1 ] [ 0.8 0.2 0.2 ] [ 0 0 0 ] 1
meshAttribute subdivisions 2
translate [ 1 0 0 ]
rotate [ 0 1 0 ] 30
scale [ 2 2 2 ]
loadmesh cube.obj
reset
material [ 0 0 0 ] [ 0.2 0.8 0.2 ] [ 0 0 0 ] 1
translate [ -1 0 0 ]
loadmesh tetra.obj   # trailing comment
texture unused.png
reset
scale [ 0.5 0.5 0.5 ]
loadbez two_patches.dat
""")


if __name__ == "__main__":
    main()
