"""The CUDA path against the reference's own libbuff code (needs a B200: -m gpu).

The inputs are the reference-pinned golden cases (tests/golden/ref_libbuff.npz,
made by tests/golden/make_ref_fixtures.py from the reference's libbuff
sources compiled in place), read through the library's own .buffgeo, mesh,
MATERIAL and SVTENSOR parsers -- the Janus and Gaussian eps(x) as SVTENSOR
expressions of position, compiled into device programs -- and, for those two,
once more through the material API with the same function of position.
The library runs its default refined singular rule; the reference ran its
own code throughout for case s48 (Taylor-Duffy at RelTol 1e-8 included) and,
in the other cases, with the oracle's refined static integrals for
tetrahedron pairs sharing >= 2 vertices.

Tolerances: face tables bit-exact; matrix entries 1e-10 per entry (relative,
floor 1e-3 of the largest; 3e-8 for s48, the Taylor-Duffy tolerance); the
device near-field records of s48 within 2e-8 of the reference's Taylor-Duffy
records (per kernel scale); RHS 1e-12; GPU LU solution 1e-10 in norm (2e-8
for s48); EMT power/force/torque 1e-9 per column plus 1e-11 of the largest
column (2e-8 for s48); overlap absorbed power likewise; scattered fields
1e-9 (2e-8 for s48).
"""
import tempfile

import numpy as np
import pytest

import buffem
import refpin_cases as rc

pytestmark = pytest.mark.gpu

CASES, FIX = rc.load()
NAMES = [c["name"] for c in CASES]


def tolerances(name):
    """(matrix, solution/fields/PFT) relative tolerances of a case."""
    return (3e-8, 2e-8) if name == "s48" else (1e-10, 1e-10)


def geometry(case, d, api=False):
    geo, meshes, disp = rc.write_inputs(case, d)
    if not api:
        return buffem.SWGGeometry(GeoFileName=geo)
    mats = []
    for o in case["objects"]:
        if o["material"] == "janus":
            mats.append(buffem.Material(kind=buffem.BG_MAT_JANUS_Z, eps=4 + 0.2j, eps2=12 + 1j))
        else:
            mats.append(buffem.Material(kind=buffem.BG_MAT_GAUSSIAN, eps=3 + 0.1j, amp=1.5,
                                        center=tuple(o["center"])))
    return buffem.SWGGeometry(meshfiles=meshes, materials=mats, displacements=disp)


@pytest.mark.parametrize("name", NAMES)
def test_case_matches_reference(name):
    case = CASES[NAMES.index(name)]
    with tempfile.TemporaryDirectory() as d:
        G = geometry(case, d)
        N = G.TotalBFs
        assert N == int(FIX[name + "/N"])
        for k in range(G.NumObjects):
            np.testing.assert_array_equal(G.faces(k), FIX["%s/faces%d" % (name, k)])
        rows = FIX[name + "/rows"] if (name + "/rows") in FIX.files else None
        pw = buffem.PlaneWave(*rc.WAVE)
        tm, ts = tolerances(name)
        if (name + "/td_pairs0") in FIX.files:
            # the device's near-field records against the reference's Taylor-Duffy ones
            pairs, data = G.near_data()
            lookup = {(int(a), int(b)): k for k, (a, b) in enumerate(np.asarray(pairs)[:, :2])}
            ref = FIX[name + "/td_records0"]
            got = np.array([np.asarray(data)[lookup[(int(a), int(b))]] for a, b in FIX[name + "/td_pairs0"]])
            err = np.zeros_like(ref)
            for k in range(6):
                sc = np.abs(ref[:, 2 * (k // 2):2 * (k // 2) + 2]).max()
                err[:, k] = np.abs(got[:, k] - ref[:, k]) / np.maximum(np.abs(ref[:, k]), 1e-3 * sc)
            assert err.max() < 2e-8, err.max()
        for i, (wr, wi) in enumerate(case["omegas"]):
            w = complex(wr, wi)
            M = G.AssembleVIEMatrix(w)
            A = M.download() if rows is None else M.rows(rows)
            ok, worst = rc.close(A, FIX["%s/matrix%d" % (name, i)], tm)
            assert ok, (name, i, "matrix", worst)
            if not case.get("solve", True):
                continue
            b = G.AssembleRHSVector(w, pw)
            ok, worst = rc.close(b, FIX["%s/rhs%d" % (name, i)], 1e-12)
            assert ok, (name, i, "rhs", worst)
            M.LUFactorize()
            J = b.copy()
            M.LUSolve(J)
            Jr = FIX["%s/solution%d" % (name, i)]
            err = np.linalg.norm(J - Jr) / np.linalg.norm(Jr)
            assert err <= ts, (name, i, "solution", err)
            tp = max(ts, 1e-9)
            P = G.GetPFTMatrix(Jr, w, pw, full=True)
            Pr = FIX["%s/pft_emt%d" % (name, i)]
            floor = 1e-11 * np.abs(Pr).max()
            assert np.all(np.abs(P - Pr) <= tp * np.abs(Pr) + floor), (name, i, P, Pr)
            Po = G.GetPFTMatrix(Jr, w, None, method=buffem.BG_PFT_OVERLAP)[:, 0]
            Pro = FIX["%s/pft_overlap%d" % (name, i)][:, 0]
            assert np.all(np.abs(Po - Pro) <= tp * np.abs(Pro) + floor), (name, i, Po, Pro)
            if ("%s/fields%d" % (name, i)) in FIX.files:
                X = FIX["%s/field_points%d" % (name, i)]
                F = G.GetFields(None, Jr, w, X)
                ok, worst = rc.close(F, FIX["%s/fields%d" % (name, i)], tp)
                assert ok, (name, i, "fields", worst)


@pytest.mark.parametrize("name", ["n3janus", "gauss2"])
def test_material_api_matches_svtensor_files(name):
    """The same eps(x) given through bg_material (Janus, Gaussian kinds) and
    as SVTENSOR expressions of position compiled for the device: the
    matrices agree to 1e-12 (the two evaluate the same function by different
    code)."""
    case = CASES[NAMES.index(name)]
    with tempfile.TemporaryDirectory() as d:
        w = complex(*case["omegas"][0])
        A1 = geometry(case, d).AssembleVIEMatrix(w).download()
        A2 = geometry(case, d, api=True).AssembleVIEMatrix(w).download()
        ok, worst = rc.close(A1, A2, 1e-12)
        assert ok, worst
