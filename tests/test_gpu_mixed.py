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


@pytest.mark.parametrize("N", [300, 2500])
def test_c64_factors_partial_pivoting(N):
    """The complex64 factorisation itself (cooperative panels over up to 79
    CTAs, TF32 trailing updates): P A = L U to TF32
    accuracy -- 4 sqrt(N) 2^-11 of |A| in Frobenius norm (observed 6.6e-3 at
    N = 300, against ~8e-3 expected from K = 300 reductions at TF32's unit
    roundoff; a wrong swap or update leaves O(1) errors) -- and partial
    pivoting by |re|+|im| bounds every multiplier by sqrt(2) in modulus."""
    rng = np.random.default_rng(11)
    A = (rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))).astype(np.complex128)
    from test_gpu_parity import RawMatrix
    M = RawMatrix(N)
    M.upload(A)
    F = M.G.AllocateVIEMatrix(buffem.BG_C64).convert_from(M.M)
    F.LUFactorize()
    LU = F.download().astype(np.complex128)
    piv = F.pivots() - 1
    L = np.tril(LU, -1) + np.eye(N)
    U = np.triu(LU)
    PA = A.copy()
    for i, p in enumerate(piv):
        PA[[i, p]] = PA[[p, i]]
    assert np.abs(np.tril(LU, -1)).max() <= np.sqrt(2) * (1 + 1e-6)
    assert np.linalg.norm(PA - L @ U) <= 4 * np.sqrt(N) * 2.0 ** -11 * np.linalg.norm(A)


@pytest.mark.parametrize("which", ["sphere3", "sphere677"])
def test_assemble_with_copy_matches_convert(sphere, ref_mesh, which):
    """bg_assemble_with_copy writes the complex64 copy in the assembly
    kernels themselves: the complex128 matrix is the plain assembly's and the
    copy equals its conversion, bit for bit (far, near and Gram entries; odd
    N with a padded complex64 leading dimension for Sphere_677)."""
    path = sphere(3) if which == "sphere3" else ref_mesh("sphere677")
    G = vie_pair(path, 4 + 0.2j)
    w = 0.8 + 0.05j
    A = G.AssembleVIEMatrix(w).download()
    M, F = G.AssembleVIEMatrixWithCopy(w)
    np.testing.assert_array_equal(M.download(), A)
    C = G.AllocateVIEMatrix(buffem.BG_C64).convert_from(M)
    np.testing.assert_array_equal(F.download(), C.download())
    np.testing.assert_array_equal(F.download(), A.astype(np.complex64))


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


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (70, 33, 17), (300, 130, 64), (513, 200, 1000), (2100, 300, 40),
                                   (4096, 300, 100), (8192, 600, 256)])
def test_cgemm_tf32_device(M, N, K):
    """C -= A B on the tcgen05 TF32 tensor cores (complex64): against the
    complex128 product of the same complex64 inputs, entrywise within
    2^-9 (|A| |B|)_ij plus FP32 rounding of C -- TF32 keeps 10 mantissa bits
    of each operand and accumulates in FP32.  The shapes cover ragged tiles,
    both tile widths (N <= 128 and N > 128) and more tiles than SMs, so the
    persistent CTAs cycle through both TMEM accumulators; the tile width
    (64, 128 or 256 columns) follows the shape, all three occur."""
    import torch
    rng = np.random.default_rng(M + 3 * N + 7 * K)
    A = (rng.normal(size=(M, K)) + 1j * rng.normal(size=(M, K))).astype(np.complex64)
    B = (rng.normal(size=(K, N)) + 1j * rng.normal(size=(K, N))).astype(np.complex64)
    Cm = (rng.normal(size=(M, N)) + 1j * rng.normal(size=(M, N))).astype(np.complex64)
    ldb = K + (K & 1)                 # B's columns on 16-byte boundaries (tensor map)
    Bp = np.zeros((N, ldb), np.complex64)
    Bp[:, :K] = B.T
    dA = torch.tensor(A.T.copy(), device="cuda")
    dB = torch.tensor(Bp, device="cuda")
    dC = torch.tensor(Cm.T.copy(), device="cuda")
    buffem.cgemm_sub_device(M, N, K, dA.data_ptr(), M, dB.data_ptr(), ldb, dC.data_ptr(), M)
    out = dC.cpu().numpy().T.astype(np.complex128)
    ref = Cm.astype(np.complex128) - A.astype(np.complex128) @ B.astype(np.complex128)
    bound = 2.0 ** -9 * (np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)) + 1e-6 * np.abs(Cm)
    assert np.all(np.abs(out - ref) <= bound), float((np.abs(out - ref) / bound).max())
