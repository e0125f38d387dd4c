"""Inputs of the reference-pinned golden cases (tests/golden/ref_libbuff.npz):
rebuilds each case's mesh files, material files and .buffgeo file exactly as
tests/golden/make_ref_fixtures.py wrote them for the reference's own code,
so that the oracle (CPU tests) and the library (GPU tests) run the same
inputs through their own parsers."""
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
TENSOR = [[4, 0.5, 0], [0.5, 6, 0], [0, 0, 9]]
WAVE = ([1, 0, 0], [0, 0, 1])


def load():
    """(cases, fixture) -- the case list as the generator stored it, and the
    npz with keys '<case>/<item>'."""
    d = np.load(os.path.join(GOLDEN, "ref_libbuff.npz"))
    return json.loads(str(d["cases"])), d


def mesh_file(spec, d):
    import meshgen
    if spec.startswith("ref:"):
        name = spec[4:]
        data = np.load(os.path.join(GOLDEN, "ref_meshes.npz"))
        ids, xyz, tets = data[name + "_ids"], data[name + "_xyz"], data[name + "_tets"]
        path = os.path.join(d, name + ".vmsh")
        with open(path, "w") as f:
            f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(ids))
            for i, (x, y, z) in zip(ids, xyz):
                f.write("%d %.17g %.17g %.17g\n" % (i, x, y, z))
            f.write("$EndNodes\n$Elements\n%d\n" % len(tets))
            for k, t in enumerate(tets):
                f.write("%d 4 2 0 1 %d %d %d %d\n" % (k + 1, *t))
            f.write("$EndElements\n")
        return path
    parts = spec.split(":")
    n = int(parts[1])
    kw = dict(radius=1.0, jitter=0.0, seed=0)
    for p in parts[2:]:
        if p.startswith("R"):
            kw["radius"] = float(p[1:])
        elif p.startswith("jitter"):
            kw["jitter"] = float(p[6:])
        elif p.startswith("seed"):
            kw["seed"] = int(p[4:])
    tag = spec.replace(":", "_").replace(".", "p")
    return meshgen.sphere_vmsh(os.path.join(d, tag + ".vmsh"), n, **kw)


def material_line(obj, d, tag):
    m = obj["material"]
    if m == "const":
        e = complex(*obj["eps"])
        return "MATERIAL CONST_EPS_%.17g%+.17gi" % (e.real, e.imag)
    path = os.path.join(d, tag + ".svtensor")
    with open(path, "w") as f:
        if m == "tensor":
            for i, a in enumerate("XYZ"):
                for j, b in enumerate("XYZ"):
                    v = TENSOR[i][j]
                    if v == 0 and i != j:
                        continue
                    f.write("Eps%s%s = %.17g%s\n" % (a, b, v, " + 0.1*i" if i == j else ""))
        elif m == "janus":
            f.write("Eps = 4 + 0.2*i + (8 + 0.8*i)*step(-z)\n")
        elif m == "gauss":
            c = obj["center"]
            f.write("cx = %.17g\ncy = %.17g\ncz = %.17g\n" % tuple(c))
            f.write("Eps = 3 + 0.1*i + 1.5*exp(-((x-cx)^2 + (y-cy)^2 + (z-cz)^2))\n")
    return "SVTENSOR " + path


def write_inputs(case, d):
    """Mesh files and the .buffgeo of a case; returns (buffgeo, meshes, displacements)."""
    objs = case["objects"]
    meshes = [mesh_file(o["mesh"], d) for o in objs]
    geo = os.path.join(d, case["name"] + ".buffgeo")
    with open(geo, "w") as f:
        for k, (o, m) in enumerate(zip(objs, meshes)):
            f.write("OBJECT Obj%d\n MESHFILE %s\n %s\n" % (k, m, material_line(o, d, "%s_obj%d" % (case["name"], k))))
            if "displaced" in o:
                f.write(" DISPLACED %.17g %.17g %.17g\n" % tuple(o["displaced"]))
            f.write("ENDOBJECT\n")
    disp = np.array([o.get("displaced", [0, 0, 0]) for o in objs], float)
    return geo, meshes, disp


def oracle_material(oracle, obj):
    m = obj["material"]
    if m == "const":
        return oracle.material(eps=complex(*obj["eps"]))
    if m == "tensor":
        return oracle.material(kind=oracle.MAT_CONST_TENSOR, tensor=np.array(TENSOR, complex) + 0.1j * np.eye(3))
    if m == "janus":
        return oracle.material(kind=oracle.MAT_JANUS_Z, eps=4 + 0.2j, eps2=12 + 1j)
    return oracle.material(kind=oracle.MAT_GAUSSIAN, eps=3 + 0.1j, amp=1.5, center=tuple(obj["center"]))


def close(got, want, rtol):
    """Entrywise |got - want| <= rtol (|want| + 1e-3 max|want|): relative to
    each entry, with a floor at a thousandth of the largest; returns
    (ok, worst ratio of the error to that bound)."""
    got, want = np.asarray(got), np.asarray(want)
    scale = np.abs(want).max()
    bound = rtol * (np.abs(want) + 1e-3 * scale)
    r = np.abs(got - want) / bound
    return bool((r <= 1).all()), float(r.max())
