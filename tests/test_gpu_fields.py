"""GetFields on the GPU (-m gpu) against the oracle's restatement of
SWGGeometry::GetFields (GetFields.cc:176-382), through the C-ABI.

Tolerance: 1e-10 of the largest field component at each point, E and H
separately (FP64 on both sides, the same quadrature points and rule choice,
summed per tetrahedron on the GPU and per basis function in the oracle).
At full size, properties that need no oracle: the curl equations by finite
differences and the scattered Poynting flux against the EMT scattered power.
"""
import numpy as np
import pytest
import scipy.linalg as sl

import buffem
from test_gpu_parity import pair

pytestmark = pytest.mark.gpu

Z0 = 376.73031346177


def points(rng, n, rmin, rmax, center=(0, 0, 0)):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    return np.asarray(center) + d * rng.uniform(rmin, rmax, size=(n, 1))


def fields_close(Fg, Fo, rtol=1e-10):
    for sl_ in (slice(0, 3), slice(3, 6)):
        scale = np.abs(Fo[:, sl_]).max(axis=1, keepdims=True)
        err = np.abs(Fg[:, sl_] - Fo[:, sl_]) / scale
        assert err.max() <= rtol, err.max()


@pytest.mark.parametrize("omega", [1.0, 0.7 + 0.02j])
def test_fields_parity_one_sphere(sphere, oracle_lib, omega):
    """Random currents on a jittered sphere, points inside the body, near
    its surface (both rules per tetrahedron) and far away (4-point rule
    only), with and without the incident wave, at a real and a complex
    frequency."""
    Gb, Go = pair(sphere(3, jitter=0.05, seed=4), buffem.Material(eps=4 + 0.2j),
                  oracle_lib.material(eps=4 + 0.2j), oracle_lib=oracle_lib)
    rng = np.random.default_rng(1)
    J = rng.normal(size=Gb.TotalBFs) + 1j * rng.normal(size=Gb.TotalBFs)
    X = np.vstack([points(rng, 20, 0.0, 0.9), points(rng, 40, 1.05, 4.0), points(rng, 20, 8.0, 30.0)])
    E0, nh = np.array([1, 0.4j, -0.3j], complex), np.array([0, 0.6, 0.8])
    for IF in (None, buffem.PlaneWave(E0, nh)):
        Fg = Gb.GetFields(IF, J, omega, X)
        Fo = Go.get_fields(complex(omega), J, X, None if IF is None else E0, None if IF is None else nh)
        fields_close(Fg, Fo)
    # incident field alone (J = 0 in the reference)
    Fg = Gb.GetFields(buffem.PlaneWave(E0, nh), None, omega, X)
    Fo = Go.get_fields(complex(omega), None, X, E0, nh)
    np.testing.assert_allclose(Fg, Fo, rtol=1e-13, atol=1e-15)
    assert Gb.GetFields(None, J, omega, np.zeros((0, 3))).shape == (0, 6)


def test_fields_parity_two_objects_solved(sphere, oracle_lib):
    """Solved currents of two displaced spheres of different meshes and
    materials; points between and around them."""
    disp = [[0, 0, 0], [0.3, 0, 2.4]]
    meshes = [sphere(2, radius=0.8), sphere(3, radius=1.0)]
    Gb, Go = pair(meshes, [buffem.Material(eps=4 + 0.2j), buffem.Material(eps=9 + 1j)],
                  [oracle_lib.material(eps=4 + 0.2j), oracle_lib.material(eps=9 + 1j)], disp=disp,
                  oracle_lib=oracle_lib)
    w = 1.3
    E0, nh = np.array([1, 0, 0], complex), np.array([0, 0, 1.0])
    J = sl.lu_solve(sl.lu_factor(Go.assemble(complex(w))), Go.rhs_planewave(complex(w), E0, nh))
    rng = np.random.default_rng(2)
    X = np.vstack([points(rng, 30, 0.85, 1.6), points(rng, 30, 1.05, 2.0, center=disp[1]),
                   points(rng, 40, 4.0, 20.0)])
    Fg = Gb.GetFields(buffem.PlaneWave(E0, nh), J, w, X)
    Fo = Go.get_fields(complex(w), J, X, E0, nh)
    fields_close(Fg, Fo)


def test_fields_many_points_split(sphere, oracle_lib):
    """Enough points that the tetrahedron blocks are lengthened (several
    tetrahedra per thread): the result does not depend on the split."""
    Gb, Go = pair(sphere(3), buffem.Material(eps=4 + 0.2j), oracle_lib.material(eps=4 + 0.2j),
                  oracle_lib=oracle_lib)
    rng = np.random.default_rng(3)
    J = rng.normal(size=Gb.TotalBFs) + 1j * rng.normal(size=Gb.TotalBFs)
    X = points(rng, 40000, 1.2, 6.0)
    Fg = Gb.GetFields(None, J, 1.0, X)
    idx = rng.choice(len(X), 200, replace=False)
    fields_close(Fg[idx], Go.get_fields(1.0 + 0j, J, X[idx]))
    F1 = Gb.GetFields(None, J, 1.0, X[idx])
    np.testing.assert_allclose(F1, Fg[idx], rtol=1e-12, atol=0)


def test_fields_full_size_properties(sphere):
    """A sphere of N = 25350 basis functions solved on the GPU: its fields
    satisfy curl E = i w Z0 H and curl H = -i w E / Z0 outside the body, the
    scattered flux is the same through two spheres, matches the EMT PScat of
    the same currents to 0.5% and the total flux matches minus the OPFT PAbs
    to 0.5%."""
    G = buffem.SWGGeometry(meshfiles=sphere(13), materials=buffem.Material(eps=4 + 0.2j))
    w = 1.0
    E0, nh = np.array([1, 0, 0], complex), np.array([0, 0, 1.0])
    IF = buffem.PlaneWave(E0, nh)
    A = G.AssembleVIEMatrix(w)
    b = G.AssembleRHSVector(w, IF)
    A.LUFactorize()
    J = A.LUSolve(b.copy())
    rng = np.random.default_rng(5)
    h = 1e-4
    # points where every basis function takes the 4-point rule: the rule
    # switch at |X - centroid| = 10 radius is a step that finite differences
    # would magnify
    for x in points(rng, 3, 2.5, 4.0):
        pts = [x] + [x + s * h * e for e in np.eye(3) for s in (1, -1)]
        F = G.GetFields(IF, J, w, np.array(pts))
        d = np.array([(F[1 + 2 * c] - F[2 + 2 * c]) / (2 * h) for c in range(3)])
        curl = lambda o: np.array([d[1, o + 2] - d[2, o + 1], d[2, o] - d[0, o + 2], d[0, o + 1] - d[1, o]])
        assert np.abs(curl(0) - 1j * w * Z0 * F[0, 3:]).max() <= 1e-6 * np.abs(curl(0)).max()
        assert np.abs(curl(3) + 1j * w / Z0 * F[0, :3]).max() <= 1e-6 * np.abs(curl(3)).max()

    def flux(R, inc):
        xq, wq = np.polynomial.legendre.leggauss(32)
        ph = np.linspace(0, 2 * np.pi, 64, endpoint=False)
        st = np.sqrt(1 - xq * xq)
        P = R * np.stack([np.outer(st, np.cos(ph)), np.outer(st, np.sin(ph)), np.outer(xq, np.ones(64))], -1)
        P = P.reshape(-1, 3)
        ws = np.repeat(wq, 64) * (2 * np.pi / 64) * R * R
        F = G.GetFields(IF if inc else None, J, w, P)
        S = 0.5 * np.real(np.cross(F[:, :3], np.conj(F[:, 3:])))
        return float(np.sum(ws * np.sum(S * P / R, axis=1)))
    f1, f2 = flux(1.5, False), flux(4.0, False)
    assert abs(f1 / f2 - 1) < 1e-6
    emt = G.GetPFTMatrix(J, w, IF)[0]
    assert abs(f2 / emt[1] - 1) < 5e-3, (f2, emt)
    opft = G.GetPFTMatrix(J, w, IF, method=buffem.BG_PFT_OVERLAP)[0]
    assert abs(-flux(4.0, True) / opft[0] - 1) < 5e-3
