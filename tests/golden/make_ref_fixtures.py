"""Generates tests/golden/ref_libbuff.npz from the reference's own libbuff
code (run where the reference is mounted; the committed .npz is what the
tests read):

    python tests/golden/make_ref_fixtures.py <path of the buff-em source tree>

How the reference is run: oracle/refpin/Makefile compiles 16 of the
reference's libbuff sources in place (SWGGeometry, SWGVolume, InitFaceList,
ReadGMSHFile, TetCR, Cubature, GMatrixElements, FIBBICache, VIEMatrix,
OverlapIntegrals, RHSVector, SVTensor, GetPFT, EMTPFT, OPFT, GetFields)
with project-written stand-ins for the SCUFF-EM surface they include
(oracle/refpin/shim.cc; SCUFF-EM is not vendored) into
oracle/_ref/libbuffref.so, and oracle/refpin/refdrv.cc calls it in the
reference drivers' order (buff-scatter.cc:236-347): SWGGeometry(.buffgeo),
AssembleVIEMatrix, AssembleRHSVector(PlaneWave), GetPFTMatrix, GetFields.

What comes from the reference's code: the mesh reader and face list (the
basis-function order), the far-field rule, the desingularised near-field
rule with its exp-relative series, the combination with the cached static
integrals, the 16x16 static rule for tetrahedron pairs sharing <= 1 vertex,
the V^-1 Gram blocks with SVTensor materials, the RHS, the EMT and overlap
power/force/torque and the scattered fields.

The static integrals of tetrahedron pairs sharing >= 2 vertices: the
reference computes them with its Taylor-Duffy code (TTaylorDuffy.cc, also
compiled in place) through an adaptive cubature library that is not
vendored; here that cubature is the project's own (Genz-Malik, shim.cc) and
the kernel functions K_n(X) are restated from the Taylor-Duffy paper.  Case
s48 runs it for every record at RelTol 1e-8 (the reference's default is
1e-6) and stores the singular records themselves ('td_pairs', 'td_records')
beside the matrices.  For the other cases (Taylor-Duffy at that tolerance
takes seconds per record) the records of the basis-function pairs that have
such a tetrahedron pair are written by the project's CPU oracle with its
refined singular rule, in the reference's cache file format, and loaded by
the reference's own FIBBICache::PreLoad through BUFF_CACHE_PATH; the
reference computes every other record itself.  Also restated rather than
the reference's: the plane wave (E = E0 exp(i k nHat.x), H = nHat x E / Z0,
k = Omega), the dyadic Green's functions of the field routine (CalcGC), and
the complex expression evaluator of the material files.

Cases (inputs are regenerated by the tests from the metadata stored beside
the outputs; meshes come from buff-em_b200/meshgen.py or the reference's own
test meshes in tests/golden/ref_meshes.npz; tests/refpin_cases.py writes
them, here and in the tests):
  s48       Sphere_48 (src/unitTests), CONST_EPS_10, omega 0.1 and 1.0,
            every near record by the reference (Taylor-Duffy at 1e-8):
            full matrices, RHS, LAPACK solution, EMT and overlap PFT,
            fields, and the 624 singular records
  s533      Sphere_533 with E10Sphere_533.buffgeo's eps = 10, omega = 0.1
            (unit-test-LFField.cc:50-71): 16 seeded rows, RHS, solution, PFT,
            fields
  n5        the small-sphere configuration: 5^3 cells (N = 1,350),
            eps = 4 + 0.2i, omega = 1: 12 seeded rows, RHS, solution, PFT
  n2tensor  2^3-cell sphere, SVTENSOR [[4,.5,0],[.5,6,0],[0,0,9]] + 0.1i,
            omega = 1 and 1 + 0.1i: full matrices
  n3janus   3^3-cell sphere jittered +-0.05 h (seed 2), SVTENSOR
            eps = 4 + 0.2i (z > 0) / 12 + 1i (z <= 0), omega = 1: 16 rows,
            RHS, solution, PFT, fields
  gauss2    two spheres (2^3 and 3^3 cells, radii 0.8 and 1.1, the second
            DISPLACED 0 0 2.4), SVTENSOR eps(x) = 3 + 1.5 exp(-|x - c|^2)
            + 0.1i about each centre, omega = 0.7: 16 rows, RHS, solution, PFT
"""
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import scipy.linalg as sl

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "buff-em_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from refpin_cases import WAVE, oracle_material, write_inputs  # noqa: E402

SIG = b"FIBBI_GCACHE\0"

CASES = [
    dict(name="s48", objects=[dict(mesh="ref:sphere48", material="const", eps=[10.0, 0.0])],
         omegas=[[0.1, 0.0], [1.0, 0.0]], rows=None, fields=True, taylor_duffy=[1e-8, 200000]),
    dict(name="s533", objects=[dict(mesh="ref:sphere533", material="const", eps=[10.0, 0.0])],
         omegas=[[0.1, 0.0]], rows=16, fields=True),
    dict(name="n5", objects=[dict(mesh="sphere:5", material="const", eps=[4.0, 0.2])],
         omegas=[[1.0, 0.0]], rows=12, fields=False),
    dict(name="n2tensor", objects=[dict(mesh="sphere:2", material="tensor")],
         omegas=[[1.0, 0.0], [1.0, 0.1]], rows=None, fields=False, solve=False),
    dict(name="n3janus", objects=[dict(mesh="sphere:3:jitter0.05:seed2", material="janus")],
         omegas=[[1.0, 0.0]], rows=16, fields=True),
    dict(name="gauss2", objects=[dict(mesh="sphere:2:R0.8", material="gauss", center=[0, 0, 0]),
                                 dict(mesh="sphere:3:R1.1", material="gauss", center=[0, 0, 2.4],
                                      displaced=[0, 0, 2.4])],
         omegas=[[0.7, 0.0]], rows=16, fields=False),
]


def ref_lib(ref):
    subprocess.run(["make", "-s", "-j", "8", "-C", os.path.join(ROOT, "oracle", "refpin"), "REF=" + ref], check=True)
    oracle.build()
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libbuffref.so"))
    P = C.c_void_p
    L.rp_geometry.restype = P
    L.rp_geometry.argtypes = [C.c_char_p]
    for f in ("rp_total_bfs", "rp_num_objects"):
        getattr(L, f).argtypes = [P]
    for f in ("rp_object_bfs", "rp_cache_size"):
        getattr(L, f).argtypes = [P, C.c_int]
    L.rp_faces.argtypes = [P, C.c_int, P]
    L.rp_vertices.argtypes = [P, C.c_int, P]
    L.rp_singular_pairs.argtypes = [P, C.c_int, P, C.c_int]
    L.rp_cache_key.argtypes = [P, C.c_int, C.c_int, C.c_int, P]
    L.rp_assemble.argtypes = [P, C.c_double, C.c_double, P]
    L.rp_rhs.argtypes = [P, C.c_double, C.c_double, P, P, P]
    L.rp_pft.argtypes = [P, P, C.c_double, C.c_double, P, P, C.c_int, P]
    L.rp_fields.argtypes = [P, P, C.c_double, C.c_double, C.c_int, P, P]
    L.rp_set_taylor_duffy.argtypes = [C.c_double, C.c_int]
    L.rp_fibbi.argtypes = [P, C.c_int, C.c_int, P, P]
    return L


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def run_case(L, case, d):
    objs = case["objects"]
    geo, meshes, disp = write_inputs(case, d)
    G = C.c_void_p(L.rp_geometry(geo.encode()))
    N = L.rp_total_bfs(G)
    nobj = L.rp_num_objects(G)
    out = {"N": np.array(N)}
    # near-field records for the pairs that need Taylor-Duffy, from the oracle
    Go = oracle.Geometry(meshes, [oracle_material(oracle, o) for o in objs], displacements=disp, nang=10, refine=True)
    assert Go.N == N, (Go.N, N)
    cachedir = os.path.join(d, "cache_" + case["name"])
    os.makedirs(cachedir, exist_ok=True)
    nrec = 0
    for k in range(nobj):
        nb = L.rp_object_bfs(G, k)
        faces = np.zeros((nb, 9), np.int32)
        L.rp_faces(G, k, ptr(faces))
        out["faces%d" % k] = faces
        cnt = L.rp_singular_pairs(G, k, None, 0)
        pairs = np.zeros((cnt, 2), np.int32)
        L.rp_singular_pairs(G, k, ptr(pairs), cnt)
        off = Go.off[k]
        base = os.path.splitext(os.path.basename(meshes[k]))[0]
        if "taylor_duffy" in case:
            # the reference computes every record itself, Taylor-Duffy included
            tol, maxe = case["taylor_duffy"]
            L.rp_set_taylor_duffy(tol, maxe)
            rec = np.zeros((cnt, 6))
            L.rp_fibbi(G, k, cnt, ptr(pairs), ptr(rec))
            out["td_pairs%d" % k] = pairs
            out["td_records%d" % k] = rec
            continue
        with open(os.path.join(cachedir, base + ".cache"), "wb") as f:
            f.write(SIG)
            key = np.zeros(27, np.float32)
            for a, b in pairs:
                L.rp_cache_key(G, k, int(a), int(b), ptr(key))
                f.write(key.tobytes())
                f.write(np.asarray(Go.fibbi(int(a + off), int(b + off)), np.float64).tobytes())
        nrec += cnt
    out["singular_records"] = np.array(0 if "taylor_duffy" in case else nrec)
    os.environ["BUFF_CACHE_PATH"] = cachedir
    rng = np.random.default_rng(len(case["name"]) * 7919 + N)
    rows = None if case["rows"] is None else np.sort(rng.choice(N, case["rows"], replace=False))
    if rows is not None:
        out["rows"] = rows
    E0 = np.array(WAVE[0], complex)
    nh = np.array(WAVE[1], float)
    for i, (wr, wi) in enumerate(case["omegas"]):
        flat = np.zeros(2 * N * N)
        L.rp_assemble(G, wr, wi, ptr(flat))
        A = flat.view(np.complex128).reshape(N, N, order="F")
        out["matrix%d" % i] = A if rows is None else A[rows]
        if case.get("solve", True):
            b = np.zeros(2 * N)
            L.rp_rhs(G, wr, wi, ptr(E0.view(np.float64)), ptr(nh), ptr(b))
            b = b.view(np.complex128)
            J = sl.lu_solve(sl.lu_factor(A), b)
            out["rhs%d" % i] = b
            out["solution%d" % i] = J
            for meth, tag in ((1, "pft_emt"), (0, "pft_overlap")):
                P = np.zeros(8 * nobj)
                L.rp_pft(G, ptr(J.view(np.float64)), wr, wi, ptr(E0.view(np.float64)), ptr(nh), meth, ptr(P))
                out["%s%d" % (tag, i)] = P.reshape(nobj, 8)
            if case.get("fields"):
                X = np.random.default_rng(5).normal(size=(8, 3))
                X *= (1.6 + np.arange(8)[:, None] * 0.5) / np.linalg.norm(X, axis=1, keepdims=True)
                F = np.zeros(2 * 6 * len(X))
                L.rp_fields(G, ptr(J.view(np.float64)), wr, wi, len(X), ptr(np.ascontiguousarray(X)), ptr(F))
                out["field_points%d" % i] = X
                out["fields%d" % i] = F.view(np.complex128).reshape(len(X), 6)
    for k in range(nobj):
        out["cache_records%d" % k] = np.array(L.rp_cache_size(G, k))
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_ref_fixtures.py <path of the buff-em source tree>")
    L = ref_lib(os.path.abspath(sys.argv[1]))
    result = {"cases": np.array(json.dumps(CASES))}
    with tempfile.TemporaryDirectory() as d:
        cwd = os.getcwd()
        os.chdir(d)      # the reference stores its caches beside the working directory
        try:
            for case in CASES:
                res = run_case(L, case, d)
                for k, v in res.items():
                    result[case["name"] + "/" + k] = v
                print(case["name"], "N =", int(res["N"]), "records from the oracle:", int(res["singular_records"]),
                      flush=True)
        finally:
            os.chdir(cwd)
    path = os.path.join(HERE, "ref_libbuff.npz")
    np.savez_compressed(path, **result)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
