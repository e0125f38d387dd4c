"""CPU checks of the graph-network oracle (oracle/gnn_oracle.py): its
hand-written backward pass against central finite differences of its forward
pass, on the VIE matrix of a small sphere assembled by the C oracle."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import gnn_oracle as go  # noqa: E402


@pytest.fixture(scope="module")
def small_system(sphere, oracle_lib):
    import meshgen
    import oracle
    n = 2
    G = oracle.Geometry([sphere(n)], [oracle.material(eps=6 + 0.5j)])
    A = G.assemble(1.1)
    faces = G.faces(0)
    V, _ = meshgen.sphere_arrays(n)
    rowptr, col, etr = go.pattern(faces)
    return A, faces, V, rowptr, col, etr


def test_pattern_is_symmetric_with_self_pairs(small_system):
    A, faces, V, rowptr, col, etr = small_system
    N = len(rowptr) - 1
    rows = np.repeat(np.arange(N), np.diff(rowptr))
    assert np.all(col[etr] == rows) and np.all(rows[etr] == col)
    assert np.all(np.diff(col)[np.diff(rows) == 0] > 0)        # sorted, unique per row
    assert set(zip(rows[rows == col], col[rows == col])) == {(i, i) for i in range(N)}


def test_untrained_network_is_jacobi(small_system):
    A, faces, V, rowptr, col, etr = small_system
    F, Ef, ratio, dinv = go.features(V, faces, A, 1.1, rowptr, col)
    _, total = go.layout()
    rng = np.random.default_rng(0)
    flat = rng.normal(scale=0.2, size=total)
    off, _ = go.layout()
    for k in ("Wo", "bo"):
        o, m = off[k]
        flat[o:o + m] = 0
    m, _ = go.forward(go.unpack(flat), F, Ef, rowptr, col, ratio, dinv)
    N = len(rowptr) - 1
    rows = np.repeat(np.arange(N), np.diff(rowptr))
    np.testing.assert_array_equal(m, np.where(rows == col, dinv[col], 0))


def test_backward_matches_finite_differences(small_system):
    A, faces, V, rowptr, col, etr = small_system
    N = A.shape[0]
    F, Ef, ratio, dinv = go.features(V, faces, A, 1.1, rowptr, col)
    rng = np.random.default_rng(1)
    _, total = go.layout()
    flat = rng.normal(scale=0.15, size=total)
    Z = rng.normal(size=(N, 3)) + 1j * rng.normal(size=(N, 3))
    b = rng.normal(size=N) + 1j * rng.normal(size=N)
    x = np.linalg.solve(A, b)
    L, g, _ = go.loss_and_grad(flat, F, Ef, rowptr, col, ratio, dinv, A, Z, b, x, 0.5)
    off, _ = go.layout()
    idx = []
    for k, (o, n) in off.items():           # a few live entries of every parameter block
        live = np.flatnonzero(g[o:o + n])
        assert live.size > 0, k
        idx += list(rng.choice(live, size=min(3, live.size), replace=False) + o)
    h = 1e-7                                # small enough not to cross ReLU kinks
    for k in idx:
        e = np.zeros(total)
        e[k] = h
        Lp = go.loss_and_grad(flat + e, F, Ef, rowptr, col, ratio, dinv, A, Z, b, x, 0.5)[0]
        Lm = go.loss_and_grad(flat - e, F, Ef, rowptr, col, ratio, dinv, A, Z, b, x, 0.5)[0]
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * (abs(g[k]) + 1e-3 * np.abs(g).max()), (k, fd, g[k])


def test_coefficient_bound_tracks_the_near_field_spectrum(small_system):
    """The power-iteration estimate of rho(K1) matches the dense eigenvalue
    computation, and a saturated readout gives s = smax on every edge."""
    A, faces, V, rowptr, col, etr = small_system
    N = A.shape[0]
    F, Ef, ratio, dinv = go.features(V, faces, A, 1.1, rowptr, col)
    rng = np.random.default_rng(2)
    _, total = go.layout()
    flat = rng.normal(scale=0.3, size=total)
    o, m = go.layout()[0]["Wo"]
    flat[o:o + m] = 0.0
    o, m = go.layout()[0]["bo"]
    flat[o:o + m] = [0.0, 0.0, 30.0, 0.0]    # c = 0 and s = smax on every edge
    mv, c = go.forward(go.unpack(flat), F, Ef, rowptr, col, ratio, dinv)
    rows = np.repeat(np.arange(N), np.diff(rowptr))
    K1 = np.zeros((N, N), complex)
    K1[rows, col] = np.where(rows != col, A[rows, col] / np.diag(A)[col], 0)
    rho1_true = np.abs(np.linalg.eigvals(K1)).max()
    assert abs(c["rho_ref"] - rho1_true) <= 0.1 * rho1_true, (c["rho_ref"], rho1_true)
    assert c["smax"] == go.SREL / max(c["rho_ref"], go.SREL)
    # m_ij = -smax r_ij / A_jj off the diagonal, 1 / A_jj on it
    off = rows != col
    np.testing.assert_allclose(mv[off], -c["smax"] * ratio[off] * dinv[col[off]], rtol=1e-12, atol=0)
    np.testing.assert_allclose(mv[~off], dinv[col[~off]], rtol=1e-12, atol=0)
