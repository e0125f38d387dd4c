"""The CPU oracle against the reference's own libbuff code (CPU, no GPU).

tests/golden/ref_libbuff.npz holds outputs of the reference's libbuff
sources compiled in place (tests/golden/make_ref_fixtures.py): the face
table (basis-function order), matrix entries, RHS, the LAPACK solution, EMT
and overlap power/force/torque and scattered fields, for the reference's own
test meshes, the small-sphere configuration (5^3 cells, N = 1,350) and
tensor, Janus and two-object Gaussian materials.  In case s48 every number
is the reference's own, its Taylor-Duffy static integrals included (run at
RelTol 1e-8, its default being 1e-6; the adaptive cubature under it is the
project's Genz-Malik rule, the cubature library being absent); in the other
cases the static integrals of tetrahedron pairs sharing >= 2 vertices were
given to the reference by the oracle (its refined rule, through the
reference's cache loader) and everything else is the reference's own
arithmetic.

Tolerances: face tables bit-exact; matrix entries 1e-12 and RHS 1e-12 per
entry (relative, floor 1e-3 of the largest) -- 3e-8 for s48, whose singular
integrals carry the Taylor-Duffy tolerance; singular near-field records
2e-8 of each kernel's scale; solution 1e-10 in norm (2e-8 for s48); PFT 1e-9
per column plus 1e-11 of the largest column (components that vanish by
symmetry are rounding noise: the reference's torques of s48 are 1e-7 of its
largest entry and differ between summation orders by ~3e-13 of it; 2e-8 for
s48); fields 1e-10 (2e-8 for s48).
"""
import tempfile

import numpy as np
import pytest
import scipy.linalg as sl

import refpin_cases as rc

CASES, FIX = rc.load()
NAMES = [c["name"] for c in CASES]
SMALL = {"s48", "n2tensor", "n3janus", "gauss2", "s533"}
# cases whose singular integrals are the reference's Taylor-Duffy at RelTol 1e-8
TD_CASES = {"s48"}


def tolerances(name):
    """(matrix, solution and fields, PFT) relative tolerances of a case."""
    return (3e-8, 2e-8, 2e-8) if name in TD_CASES else (1e-12, 1e-10, 1e-9)


def record_errors(got, ref):
    """Per-record error of 6-double near-field records relative to each
    kernel's magnitude (components 2k, 2k+1 share kernel r^(k-1)); floor
    1e-3 of the largest value of that kernel."""
    err = np.zeros_like(ref)
    for k in range(6):
        sc = np.abs(ref[:, 2 * (k // 2):2 * (k // 2) + 2]).max()
        err[:, k] = np.abs(got[:, k] - ref[:, k]) / np.maximum(np.abs(ref[:, k]), 1e-3 * sc)
    return err


def oracle_geometry(oracle_lib, case, d):
    geo, meshes, disp = rc.write_inputs(case, d)
    return oracle_lib.Geometry(meshes, [rc.oracle_material(oracle_lib, o) for o in case["objects"]],
                               displacements=disp, nang=10, refine=True)


@pytest.mark.parametrize("name", NAMES)
def test_face_order_matches_reference(name, oracle_lib):
    case = CASES[NAMES.index(name)]
    with tempfile.TemporaryDirectory() as d:
        Go = oracle_geometry(oracle_lib, case, d)
        assert Go.N == int(FIX[name + "/N"])
        for k in range(len(case["objects"])):
            np.testing.assert_array_equal(Go.faces(k), FIX["%s/faces%d" % (name, k)])


@pytest.mark.parametrize("name", [n for n in NAMES if n in SMALL])
def test_system_matches_reference(name, oracle_lib):
    case = CASES[NAMES.index(name)]
    with tempfile.TemporaryDirectory() as d:
        Go = oracle_geometry(oracle_lib, case, d)
        Go.cache_build()
        rows = FIX[name + "/rows"] if (name + "/rows") in FIX.files else None
        E0 = np.array(rc.WAVE[0], complex)
        nh = np.array(rc.WAVE[1], float)
        tm, ts, tp = tolerances(name)
        for i, (wr, wi) in enumerate(case["omegas"]):
            w = complex(wr, wi)
            A = Go.assemble(w)
            ref = FIX["%s/matrix%d" % (name, i)]
            ok, worst = rc.close(A if rows is None else A[rows], ref, tm)
            assert ok, (name, i, "matrix", worst)
            if case.get("solve", True):
                b = Go.rhs_planewave(w, E0, nh)
                ok, worst = rc.close(b, FIX["%s/rhs%d" % (name, i)], 1e-12)
                assert ok, (name, i, "rhs", worst)
                J = sl.lu_solve(sl.lu_factor(A), b)
                Jr = FIX["%s/solution%d" % (name, i)]
                assert np.linalg.norm(J - Jr) <= ts * np.linalg.norm(Jr)
                P = Go.pft_emt8(w, Jr, E0, nh)
                Pr = FIX["%s/pft_emt%d" % (name, i)]
                floor = 1e-11 * np.abs(Pr).max()
                assert np.all(np.abs(P - Pr) <= tp * np.abs(Pr) + floor), (name, i, P, Pr)
                Po = Go.pft_opft(w, Jr)
                Pro = FIX["%s/pft_overlap%d" % (name, i)][:, 0]
                assert np.all(np.abs(Po - Pro) <= tp * np.abs(Pro) + floor), (name, i, Po, Pro)
                if ("%s/fields%d" % (name, i)) in FIX.files:
                    X = FIX["%s/field_points%d" % (name, i)]
                    F = Go.get_fields(w, Jr, X)
                    ok, worst = rc.close(F, FIX["%s/fields%d" % (name, i)], max(ts, 1e-10))
                    assert ok, (name, i, "fields", worst)


def test_singular_records_match_reference_taylor_duffy(oracle_lib):
    """The near-field records of every basis-function pair of Sphere_48 that
    has a tetrahedron pair sharing >= 2 vertices, computed by the reference's
    own ComputeFIBBIData (Taylor-Duffy at RelTol 1e-8), against the oracle's
    refined singular rule: within 2e-8 of each kernel's scale (observed
    1.1e-8, the Taylor-Duffy tolerance)."""
    case = CASES[NAMES.index("s48")]
    with tempfile.TemporaryDirectory() as d:
        Go = oracle_geometry(oracle_lib, case, d)
        pairs, ref = FIX["s48/td_pairs0"], FIX["s48/td_records0"]
        assert len(pairs) == 624
        got = np.array([Go.fibbi(int(a), int(b)) for a, b in pairs])
        err = record_errors(got, ref)
        assert err.max() < 2e-8, err.max()


def test_small_sphere_configuration_rows(oracle_lib):
    """5^3 cells, N = 1,350, eps 4 + 0.2i, omega 1: the reference's rows,
    RHS and absorbed/scattered power for its own solution."""
    case = CASES[NAMES.index("n5")]
    with tempfile.TemporaryDirectory() as d:
        Go = oracle_geometry(oracle_lib, case, d)
        rows = FIX["n5/rows"]
        Go.cache_build(rows)
        R = Go.assemble_rows(1.0 + 0j, rows)     # the upper-triangle part b >= a of each row
        Rr = FIX["n5/matrix0"]
        for k, r in enumerate(rows):
            ok, worst = rc.close(R[k, r:], Rr[k, r:], 1e-12)
            assert ok, (int(r), worst)
        E0, nh = np.array(rc.WAVE[0], complex), np.array(rc.WAVE[1], float)
        ok, worst = rc.close(Go.rhs_planewave(1.0 + 0j, E0, nh), FIX["n5/rhs0"], 1e-12)
        assert ok, worst
        Pr = FIX["n5/pft_emt0"]
        P = Go.pft_emt(1.0 + 0j, FIX["n5/solution0"], E0, nh)
        np.testing.assert_allclose(P[0], Pr[0, :2], rtol=1e-9)
