"""Precision form: complex64 LU with tcgen05 (TF32) trailing updates plus FP64
iterative refinement against the complex128 matrix (-m gpu).

Tolerances: the refined solution must match LAPACK zgetrf's (scipy) to 1e-10
relative; the unrefined complex64 solve is only TF32-accurate (checked loosely,
< 1e-2 relative residual)."""
import numpy as np
import pytest
import scipy.linalg as sl

import buffem

pytestmark = pytest.mark.gpu


def vie_pair(path, eps, n_order=6):
    G = buffem.SWGGeometry(meshfiles=path, materials=buffem.Material(eps=eps), singular_order=n_order)
    return G


@pytest.mark.parametrize("n", [3, 5])
def test_mixed_solution_matches_fp64(sphere, n):
    G = vie_pair(sphere(n), 4 + 0.2j)
    w = 1.0
    A = G.AssembleVIEMatrix(w)
    Ah = A.download()
    F = G.AllocateVIEMatrix(buffem.BG_C64).convert_from(A)
    F.LUFactorize()
    B = np.zeros((G.TotalBFs, 3), complex, order="F")
    waves = [([1, 0, 0], [0, 0, 1]), ([0, 1, 0], [0, 0, 1]), ([0, 0, 1], [1, 0, 0])]
    for i, (E0, nh) in enumerate(waves):
        B[:, i] = G.AssembleRHSVector(w, buffem.PlaneWave(E0, nh))
    X, st = A.LUSolveRefined(F, B.copy(order="F"), tol=1e-13, maxit=40)
    Xo = sl.lu_solve(sl.lu_factor(Ah), B)
    err = np.linalg.norm(X - Xo) / np.linalg.norm(Xo)
    assert err < 1e-10, (err, st)
    assert st[1] <= 1e-13 and st[0] >= 1
    # the bare complex64 solve is TF32-accurate only
    x32 = B[:, 0].copy()
    F.LUSolve(x32)
    r = np.linalg.norm(Ah @ x32 - B[:, 0]) / np.linalg.norm(B[:, 0])
    assert r < 1e-2


def test_mixed_random_matrix_sizes():
    rng = np.random.default_rng(5)
    for N in (64, 300, 1000):
        A = rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N)) + N * np.eye(N) * 0.1
        from test_gpu_parity import RawMatrix
        M = RawMatrix(N)
        M.upload(A)
        F = M.G.AllocateVIEMatrix(buffem.BG_C64).convert_from(M.M)
        F.LUFactorize()
        b = rng.normal(size=(N, 2)) + 1j * rng.normal(size=(N, 2))
        X, st = M.M.LUSolveRefined(F, b, tol=1e-13, maxit=50)
        xo = np.linalg.solve(A, b)
        assert np.linalg.norm(X - xo) <= 1e-10 * np.linalg.norm(xo), (N, st)


def test_mixed_singular_reports_info():
    from test_gpu_parity import RawMatrix
    M = RawMatrix(50)
    A = np.eye(50, dtype=complex)
    A[:, 7] = 0
    M.upload(A)
    F = M.G.AllocateVIEMatrix(buffem.BG_C64).convert_from(M.M)
    with pytest.raises(buffem.BuffError) as e:
        F.LUFactorize()
    assert e.value.status == 8
