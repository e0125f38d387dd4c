"""Regenerates tests/golden/*.npz from the reference tree (run where the
reference is mounted; the committed .npz files are what the tests read):

    python tests/golden/make_fixtures.py <path of the buff-em source tree>

Fixtures
  ref_meshes.npz : the reference's own test meshes, as parsed gmsh arrays
                   (node ids, coordinates, tetrahedron node ids), from
                   src/unitTests/Sphere_48.vmsh, src/unitTests/Sphere_533.vmsh
                   (used with E10Sphere_533.buffgeo: eps = 10, omega = 0.1,
                   unit-test-LFField.cc:50-71) and
                   examples/MieScattering/Sphere_677.vmsh.
The tests rewrite these arrays as gmsh 2.2 text so the mesh reader (node
re-numbering, 1e-6 vertex merge) is exercised on the original data.
"""
import os
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
FILES = {
    "sphere48": "src/unitTests/Sphere_48.vmsh",
    "sphere533": "src/unitTests/Sphere_533.vmsh",
    "sphere677": "examples/MieScattering/Sphere_677.vmsh",
}


def parse(path):
    lines = open(path).read().splitlines()
    i = lines.index("$Nodes")
    nn = int(lines[i + 1])
    ids, xyz = [], []
    for ln in lines[i + 2:i + 2 + nn]:
        p = ln.split()
        ids.append(int(p[0]))
        xyz.append([float(v) for v in p[1:4]])
    j = lines.index("$Elements")
    ne = int(lines[j + 1])
    tets = []
    for ln in lines[j + 2:j + 2 + ne]:
        p = [int(v) for v in ln.split()]
        if p[1] == 4:
            ntags = p[2]
            tets.append(p[3 + ntags:3 + ntags + 4])
    return np.array(ids, np.int32), np.array(xyz), np.array(tets, np.int32)


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <path of the buff-em source tree>")
    ref = sys.argv[1]
    out = {}
    for name, rel in FILES.items():
        ids, xyz, tets = parse(os.path.join(ref, rel))
        out[name + "_ids"] = ids
        out[name + "_xyz"] = xyz
        out[name + "_tets"] = tets
    np.savez_compressed(os.path.join(OUT, "ref_meshes.npz"), **out)
    print("wrote", os.path.join(OUT, "ref_meshes.npz"))


if __name__ == "__main__":
    main()
