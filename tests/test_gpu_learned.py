"""Learned form on the GPU (-m gpu): FP64 GMRES against the LU solution, the
graph network's forward pass and gradients against the numpy oracle
(oracle/gnn_oracle.py), and the iteration gain of the trained preconditioner.

Tolerances: GMRES solutions match LAPACK zgetrf's (scipy) to 1e-9 relative at
a 1e-12 residual target; the network runs in FP32, so its outputs are checked
to 1e-4 and its gradients to 2e-3 of the largest gradient entry."""
import os
import sys

import numpy as np
import pytest
import scipy.linalg as sl

import buffem
import meshgen

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import gnn_oracle as go  # noqa: E402

pytestmark = pytest.mark.gpu

EPS = 6 + 0.5j


def setup(path, omega=1.0, eps=EPS):
    G = buffem.SWGGeometry(meshfiles=path, materials=buffem.Material(eps=eps))
    A = G.AssembleVIEMatrix(omega)
    B = np.zeros((G.TotalBFs, 2), complex, order="F")
    B[:, 0] = G.AssembleRHSVector(omega, buffem.PlaneWave([1, 0, 0], [0, 0, 1]))
    B[:, 1] = G.AssembleRHSVector(omega, buffem.PlaneWave([0, 1, 0], [1, 0, 0]))
    return G, A, B


@pytest.mark.parametrize("which", ["none", "jacobi"])
def test_gmres_matches_lu(sphere, which):
    G, A, B = setup(sphere(4))
    Ah = A.download()
    P = buffem.Preconditioner.jacobi(A) if which == "jacobi" else None
    X, st = buffem.GMRESSolve(A, B, P, tol=1e-12, restart=30, maxit=3000)
    Xo = sl.lu_solve(sl.lu_factor(Ah), B)
    err = np.linalg.norm(X - Xo) / np.linalg.norm(Xo)
    assert err < 1e-9, (err, st)
    assert st[1] <= 1e-12 and st[0] >= 1
    r = np.linalg.norm(Ah @ X - B) / np.linalg.norm(B)
    assert r < 1e-11


@pytest.mark.parametrize("which", ["none", "jacobi"])
def test_mixed_gmres_matches_lu(sphere, which):
    G, A, B = setup(sphere(5))
    Ah = A.download()
    F = G.AllocateVIEMatrix(buffem.BG_C64).convert_from(A)
    P = buffem.Preconditioner.jacobi(A) if which == "jacobi" else None
    X, st = buffem.GMRESSolveMixed(A, F, B, P, tol=1e-12, restart=40, maxit=3000, inner_tol=1e-5)
    Xo = sl.lu_solve(sl.lu_factor(Ah), B)
    err = np.linalg.norm(X - Xo) / np.linalg.norm(Xo)
    assert err < 1e-9, (err, st)
    assert st[1] <= 1e-12 and st[2] >= 2   # at least two refinement sweeps at this target


def test_gmres_random_system_restarts():
    from test_gpu_parity import RawMatrix
    rng = np.random.default_rng(3)
    N = 300
    Ah = rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N)) + 30 * np.eye(N)
    M = RawMatrix(N)
    M.upload(Ah)
    b = rng.normal(size=(N, 3)) + 1j * rng.normal(size=(N, 3))
    X, st = buffem.GMRESSolve(M.M, b, None, tol=1e-12, restart=8, maxit=2000)
    xo = np.linalg.solve(Ah, b)
    assert np.linalg.norm(X - xo) <= 1e-9 * np.linalg.norm(xo), st
    assert st[0] > 8   # several restart cycles ran


@pytest.mark.parametrize("N", [301, 1024])
def test_mixed_gmres_random_odd_and_aligned_sizes(N):
    """Odd N exercises the two-rows-per-thread complex64 matrix-vector tail;
    N = 1024 has no leading-dimension padding."""
    from test_gpu_parity import RawMatrix
    rng = np.random.default_rng(N)
    Ah = rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N)) + 3 * np.sqrt(N) * np.eye(N)
    M = RawMatrix(N)
    M.upload(Ah)
    F = M.G.AllocateVIEMatrix(buffem.BG_C64).convert_from(M.M)
    b = rng.normal(size=(N, 4)) + 1j * rng.normal(size=(N, 4))
    X, st = buffem.GMRESSolveMixed(M.M, F, b, None, tol=1e-12, restart=20, maxit=2000, inner_tol=1e-4)
    xo = np.linalg.solve(Ah, b)
    assert np.linalg.norm(X - xo) <= 1e-10 * np.linalg.norm(xo), st


def test_gmres_rejects_factored_matrix(sphere):
    G, A, B = setup(sphere(2))
    A.LUFactorize()
    with pytest.raises(buffem.BuffError) as e:
        buffem.GMRESSolve(A, B)
    assert e.value.status == buffem.BG_ERR_STATE


def test_untrained_network_is_jacobi(sphere):
    G, A, B = setup(sphere(3))
    net = buffem.GNN(seed=1)
    P = buffem.Preconditioner.learned(G, A, 1.0, net)
    rowptr, col, val = P.csr(G.TotalBFs)
    Ah = A.download()
    rows = np.repeat(np.arange(G.TotalBFs), np.diff(rowptr))
    diag = rows == col
    assert np.all(val[~diag] == 0)
    np.testing.assert_allclose(val[diag], 1.0 / np.diag(Ah), rtol=1e-15)


def _device_vs_oracle(G, A, net, omega, seed):
    faces = G.faces(0)
    rowptr_o, col_o, _ = go.pattern(faces)
    P = buffem.Preconditioner.learned(G, A, omega, net)
    rowptr, col, val = P.csr(G.TotalBFs)
    assert np.array_equal(rowptr, rowptr_o) and np.array_equal(col, col_o)
    return rowptr_o, col_o, val


def test_network_forward_and_gradients_match_oracle(sphere):
    n, omega = 3, 1.3
    G, A, B = setup(sphere(n), omega=omega)
    N = G.TotalBFs
    Ah = A.download()
    V, _ = meshgen.sphere_arrays(n)
    net = buffem.GNN(seed=7)
    rng = np.random.default_rng(11)
    flat = net.params()
    # give the readout non-zero weights so every layer carries gradient
    off, total = go.layout()
    for k in ("Wo", "bo"):
        o, m = off[k]
        flat[o:o + m] = rng.normal(scale=0.05, size=m).astype(np.float32)
    net.set_params(flat)
    faces = G.faces(0)
    rowptr, col, val = _device_vs_oracle(G, A, net, omega, 0)
    Pl = buffem.Preconditioner.learned(G, A, omega, net)
    rho1, smax = Pl.bound()
    F, Ef, ratio, dinv = go.features(V, faces, Ah, omega, rowptr, col)
    p = go.unpack(flat.astype(np.float64))
    m_o, c_o = go.forward(p, F, Ef, rowptr, col, ratio, dinv)
    assert abs(rho1 - c_o["rho_ref"]) <= 1e-9 * c_o["rho_ref"], (rho1, c_o["rho_ref"])
    assert abs(smax - c_o["smax"]) <= 1e-6 * c_o["smax"]
    scale = np.abs(m_o).max()
    assert np.abs(val - m_o).max() <= 1e-4 * scale
    # gradients (lr = 0: no update) on random probes plus a right-hand side,
    # and on probes pushed twice through the Jacobi error map
    Z = rng.normal(size=(N, 4)) + 1j * rng.normal(size=(N, 4))
    b = B[:, 0].copy()
    x = sl.lu_solve(sl.lu_factor(Ah), b)
    for power in (0, 2):
        loss = net.train_step(G, A, omega, Z, b, x, lam=0.5, lr=0.0, probe_power=power)
        g_dev = net.grads()
        Zp = Z.copy()
        for _ in range(power):
            Zp = Zp - Ah @ (dinv[:, None] * Zp)
            Zp *= np.sqrt(2 * N / np.sum(np.abs(Zp) ** 2, axis=0))
        L_o, g_o, _ = go.loss_and_grad(flat.astype(np.float64), F, Ef, rowptr, col, ratio, dinv, Ah, Zp, b, x, 0.5)
        assert abs(loss - L_o) <= 1e-4 * abs(L_o), (power, loss, L_o)
        g_dev = g_dev * loss          # the device descends log L
        err = np.abs(g_dev - g_o).max()
        assert err <= 2e-3 * np.abs(g_o).max(), (power, err, np.abs(g_o).max())
    np.testing.assert_array_equal(net.params(), flat)   # lr = 0 leaves the parameters alone


def test_trained_network_beats_jacobi(sphere):
    """A short training run on seeded small spheres (other jitters) lowers the
    GMRES step count below Jacobi's on a held-out sphere."""
    net = buffem.GNN(seed=3)
    rng = np.random.default_rng(0)
    train = []
    for s in range(4):
        G, A, B = setup(sphere(4, jitter=0.15, seed=100 + s), omega=1.0)
        x = sl.lu_solve(sl.lu_factor(A.download()), B[:, 0])
        train.append((G, A, B[:, 0].copy(), x))
    losses = []
    for it in range(120):
        G, A, b, x = train[it % len(train)]
        N = G.TotalBFs
        Z = rng.normal(size=(N, 8)) + 1j * rng.normal(size=(N, 8))
        losses.append(net.train_step(G, A, 1.0, Z, b, x, lam=1.0, lr=2e-3, probe_power=4 * (it % 2)))
    plain = losses[0::2]                      # steps on unmapped random probes
    assert np.mean(plain[-4:]) < np.mean(plain[:4]), (plain[:4], plain[-4:])
    G, A, B = setup(sphere(5, jitter=0.15, seed=7), omega=1.0)
    Pj = buffem.Preconditioner.jacobi(A)
    Pl = buffem.Preconditioner.learned(G, A, 1.0, net)
    _, sj = buffem.GMRESSolve(A, B, Pj, tol=1e-10, restart=50, maxit=3000)
    Xl, sl_ = buffem.GMRESSolve(A, B, Pl, tol=1e-10, restart=50, maxit=3000)
    assert sl_[1] <= 1e-10
    assert sl_[0] < sj[0], (sl_, sj)


def test_committed_weights_beat_jacobi(sphere):
    """The shipped weights (trained by buff-em_b200/train_gnn.py) take fewer
    GMRES steps than Jacobi on a sphere outside the training set."""
    G, A, B = setup(sphere(8, jitter=0.05, seed=31), omega=1.3)
    net = buffem.GNN.load()
    _, sj = buffem.GMRESSolve(A, B, buffem.Preconditioner.jacobi(A), tol=1e-10, restart=50, maxit=3000)
    _, sl_ = buffem.GMRESSolve(A, B, buffem.Preconditioner.learned(G, A, 1.3, net), tol=1e-10, restart=50,
                               maxit=3000)
    assert sl_[1] <= 1e-10 and sl_[0] < sj[0], (sl_, sj)


def test_lu_fallback_when_gmres_misses_tolerance(sphere):
    """With a Krylov budget far too small, the solve falls back to the LU path
    and still meets the tolerance; LU also checks the GMRES answer."""
    G, A, B = setup(sphere(5))
    Ah = A.download()
    Xo = sl.lu_solve(sl.lu_factor(Ah), B)
    F = G.AllocateVIEMatrix(buffem.BG_C64).convert_from(A)
    X, st = buffem.SolveLearned(A, F, B, buffem.Preconditioner.jacobi(A), tol=1e-11, restart=10, maxit=5)
    assert st[3] == 1 and st[1] <= 1e-11, st
    assert np.linalg.norm(X - Xo) <= 1e-9 * np.linalg.norm(Xo)
    F2 = G.AllocateVIEMatrix(buffem.BG_C64).convert_from(A)
    net = buffem.GNN.load()
    X2, st2 = buffem.SolveLearned(A, F2, B, buffem.Preconditioner.learned(G, A, 1.0, net), tol=1e-11)
    assert st2[3] == 0 and st2[1] <= 1e-11, st2
    assert np.linalg.norm(X2 - Xo) <= 1e-9 * np.linalg.norm(Xo)


@pytest.mark.parametrize("nrhs", [1, 2, 3, 4])
def test_symmetric_matvec_matches_full_product(ref_mesh, nrhs):
    """An assembled matrix is known to be symmetric, so its complex64 copy
    takes the upper-triangle matrix-vector product; the same numbers uploaded
    from the host are not known to be, and take the full product.  Both
    mixed solves match LAPACK's LU and each other, at an odd N that spans
    three 256-row tiles (the reference's Sphere_677 mesh)."""
    G = buffem.SWGGeometry(meshfiles=ref_mesh("sphere677"), materials=buffem.Material(eps=EPS))
    A = G.AssembleVIEMatrix(1.0)
    Ah = A.download()
    F = G.AllocateVIEMatrix(buffem.BG_C64).convert_from(A)
    Fu = G.AllocateVIEMatrix(buffem.BG_C64)
    Fu.upload(F.download())
    rng = np.random.default_rng(nrhs)
    B = np.asfortranarray(rng.normal(size=(G.TotalBFs, nrhs)) + 1j * rng.normal(size=(G.TotalBFs, nrhs)))
    Xo = sl.lu_solve(sl.lu_factor(Ah), B)
    Xs, ss = buffem.GMRESSolveMixed(A, F, B, None, tol=1e-12, restart=40, maxit=3000, inner_tol=1e-5)
    Xf, sf = buffem.GMRESSolveMixed(A, Fu, B, None, tol=1e-12, restart=40, maxit=3000, inner_tol=1e-5)
    for X, st in ((Xs, ss), (Xf, sf)):
        assert np.linalg.norm(X - Xo) <= 1e-9 * np.linalg.norm(Xo), st
    assert abs(ss[0] - sf[0]) <= max(3, 0.05 * sf[0]), (ss, sf)   # same Krylov work up to FP32 rounding
