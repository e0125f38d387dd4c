"""GPU-vs-oracle parity through the C-ABI (needs a B200: -m gpu).

Tolerances: matrix entries and near-field integrals to 1e-10 relative
(FP64 on both sides, same quadrature rules, different summation order);
LU solutions to 1e-10 relative against LAPACK zgetrf (scipy); powers to 1e-9.
"""
import numpy as np
import pytest
import scipy.linalg as sl

import buffem

pytestmark = pytest.mark.gpu

ORDER = 6  # fixed singular-rule order used on both sides to keep the oracle fast


def entry_close(Mg, Mo, rtol=1e-10):
    scale = np.abs(Mo).max()
    err = np.abs(Mg - Mo)
    bad = err > rtol * np.abs(Mo) + 1e-13 * scale
    return (not bad.any()), float((err / (np.abs(Mo) + 1e-13 * scale)).max())


def pair(path_or_paths, mats_b, mats_o, disp=None, order=ORDER, oracle_lib=None, refine=False):
    """GPU and oracle geometries with the same singular rule: the fixed rule
    of the given order (refine=False, fast on the CPU) or the library's
    default refined rule (orders 10 and 12 with box refinement)."""
    paths = [path_or_paths] if isinstance(path_or_paths, str) else path_or_paths
    Gb = buffem.SWGGeometry(meshfiles=paths, materials=mats_b, displacements=disp, singular_order=order,
                            singular_refine=refine)
    Go = oracle_lib.Geometry(paths, mats_o, displacements=disp, nang=order, refine=refine)
    return Gb, Go


CASES = {
    "iso": dict(n=2, jit=0.0, omega=1.0, mat=("iso", 4 + 0.2j)),
    "tensor_complex_omega": dict(n=3, jit=0.05, omega=0.7 + 0.01j,
                                 mat=("tensor", [[4, .5, 0], [.5, 6, 0], [0, 0, 9]])),
    "janus": dict(n=3, jit=0.05, omega=1.3, mat=("janus", (4 + 0.2j, 12 + 1j))),
}


def mats(kind, val, oracle_lib, center=(0, 0, 0)):
    if kind == "iso":
        return buffem.Material(eps=val), oracle_lib.material(eps=val)
    if kind == "tensor":
        t = np.array(val, complex) + 0.1j * np.eye(3)
        return (buffem.Material(kind=buffem.BG_MAT_CONST_TENSOR, tensor=t),
                oracle_lib.material(kind=oracle_lib.MAT_CONST_TENSOR, tensor=t))
    if kind == "janus":
        return (buffem.Material(kind=buffem.BG_MAT_JANUS_Z, eps=val[0], eps2=val[1]),
                oracle_lib.material(kind=oracle_lib.MAT_JANUS_Z, eps=val[0], eps2=val[1]))
    if kind == "gauss":
        return (buffem.Material(kind=buffem.BG_MAT_GAUSSIAN, eps=3 + 0.1j, amp=1.5, center=center, width=1.0),
                oracle_lib.material(kind=oracle_lib.MAT_GAUSSIAN, eps=3 + 0.1j, amp=1.5, center=center, width=1.0))
    raise ValueError(kind)


@pytest.mark.parametrize("case", sorted(CASES))
def test_matrix_parity(case, sphere, oracle_lib):
    c = CASES[case]
    mb, mo = mats(*c["mat"], oracle_lib)
    Gb, Go = pair(sphere(c["n"], jitter=c["jit"], seed=7), mb, mo, oracle_lib=oracle_lib)
    M = Gb.AssembleVIEMatrix(c["omega"]).download()
    Mo = Go.assemble(complex(c["omega"]))
    ok, worst = entry_close(M, Mo)
    assert ok, worst
    assert np.array_equal(M, M.T)


def test_matrix_parity_reference_meshes(ref_mesh, oracle_lib):
    """unit-test-LFField configuration: E10Sphere_533 (eps = 10), omega = 0.1."""
    for name in ("sphere48", "sphere533"):
        Gb, Go = pair(ref_mesh(name), buffem.Material(eps=10.0), oracle_lib.material(eps=10.0),
                      oracle_lib=oracle_lib)
        ok, worst = entry_close(Gb.AssembleVIEMatrix(0.1).download(), Go.assemble(0.1 + 0j))
        assert ok, (name, worst)


def test_matrix_parity_default_order(sphere, oracle_lib):
    Gb, Go = pair(sphere(2), buffem.Material(eps=6 + 0.5j), oracle_lib.material(eps=6 + 0.5j), order=10,
                  oracle_lib=oracle_lib)
    ok, worst = entry_close(Gb.AssembleVIEMatrix(2.0).download(), Go.assemble(2.0 + 0j))
    assert ok, worst


def test_two_objects_gaussian(sphere, oracle_lib):
    p1, p2 = sphere(2, radius=1.0), sphere(2, radius=0.7)
    d = np.array([[0, 0, 0], [0, 0, 2.3]], float)
    mb1, mo1 = mats("gauss", None, oracle_lib, center=(0, 0, 0))
    mb2, mo2 = mats("gauss", None, oracle_lib, center=(0, 0, 2.3))
    Gb, Go = pair([p1, p2], [mb1, mb2], [mo1, mo2], disp=d, oracle_lib=oracle_lib)
    assert Gb.NumObjects == 2
    ok, worst = entry_close(Gb.AssembleVIEMatrix(0.5).download(), Go.assemble(0.5 + 0j))
    assert ok, worst


def test_near_field_cache_parity(sphere, oracle_lib):
    Gb, Go = pair(sphere(2, jitter=0.05, seed=1), buffem.Material(eps=4.0), oracle_lib.material(eps=4.0),
                  oracle_lib=oracle_lib)
    pairs, data = Gb.near_data()
    assert len(pairs) > 0
    ref = np.array([Go.fibbi(int(a), int(b)) for a, b in pairs])
    # the r^0 DivDiv column cancels to zero exactly (4 signed tet pairs of equal
    # value), so the absolute floor is taken over the whole table
    scale = np.abs(ref).max()
    assert np.all(np.abs(data - ref) <= 1e-10 * np.abs(ref) + 1e-13 * scale)


def test_rhs_parity(sphere, oracle_lib):
    Gb, Go = pair(sphere(3), buffem.Material(eps=4.0), oracle_lib.material(eps=4.0), oracle_lib=oracle_lib)
    for E0, nh, w in (([1, 0, 0], [0, 0, 1], 1.0), ([0, 1j, 0.5], [0.6, 0, 0.8], 0.8 + 0.02j)):
        E0 = np.array(E0, complex)
        nh = np.array(nh, float)
        vb = Gb.AssembleRHSVector(w, buffem.PlaneWave(E0, nh))
        vo = Go.rhs_planewave(complex(w), E0, nh)
        assert np.max(np.abs(vb - vo)) <= 1e-12 * np.abs(vo).max()


@pytest.mark.parametrize("N", [1, 7, 32, 33, 65, 130, 257, 700])
def test_lu_random_vs_zgetrf(N):
    rng = np.random.default_rng(N)
    A = rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))
    G = None
    lu, piv = sl.lu_factor(A)
    x_ref = sl.lu_solve((lu, piv), np.eye(N, 3, dtype=complex))
    import ctypes as C
    # a geometry-free matrix handle needs a geometry: use a 1x1-cell sphere only for its size
    pytest.importorskip("numpy")
    M = RawMatrix(N)
    M.upload(A)
    M.LUFactorize()
    assert np.array_equal(M.pivots() - 1, piv)
    F = M.download()
    assert np.max(np.abs(F - lu)) <= 1e-12 * np.abs(lu).max()
    B = np.asfortranarray(np.eye(N, 3, dtype=complex))
    M.LUSolve(B)
    assert np.linalg.norm(B - x_ref) <= 1e-10 * np.linalg.norm(x_ref)


class RawMatrix:
    """Device matrix of arbitrary size (for LU tests on non-VIE data)."""

    _geo = {}

    def __init__(self, N):
        import meshgen, tempfile, os
        # geometry with exactly N basis functions is not available for every N;
        # the matrix handle only needs N, so build it through a stub geometry
        # whose face count we overwrite via a chain of tetrahedra
        d = tempfile.mkdtemp()
        path = os.path.join(d, f"chain{N}.vmsh")
        _chain_mesh(path, N)
        self.G = buffem.SWGGeometry(meshfiles=path, materials=buffem.Material(eps=2.0))
        assert self.G.TotalBFs == N
        self.M = self.G.AllocateVIEMatrix()

    def upload(self, A):
        self.M.upload(A)

    def LUFactorize(self):
        self.M.LUFactorize()

    def pivots(self):
        return self.M.pivots()

    def download(self):
        return self.M.download()

    def LUSolve(self, B):
        return self.M.LUSolve(B)


def _chain_mesh(path, N):
    """N+1 tetrahedra glued face to face along a line: exactly N interior faces."""
    V = [(0, 0, 0), (1, 0, 0), (0, 1, 0)]
    tets = []
    for k in range(N + 1):
        z = 0.5 * (k + 1)
        V.append((0.3 * np.cos(k), 0.3 * np.sin(k), z))
        a, b, c, d = len(V) - 4, len(V) - 3, len(V) - 2, len(V) - 1
        tets.append((a, b, c, d))
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(V))
        for i, (x, y, z) in enumerate(V):
            f.write("%d %.17g %.17g %.17g\n" % (i + 1, x, y, z))
        f.write("$EndNodes\n$Elements\n%d\n" % len(tets))
        for i, t in enumerate(tets):
            f.write("%d 4 2 0 1 %d %d %d %d\n" % (i + 1, t[0] + 1, t[1] + 1, t[2] + 1, t[3] + 1))
        f.write("$EndElements\n")


def test_singular_matrix_reports_info():
    M = RawMatrix(40)
    A = np.eye(40, dtype=complex)
    A[:, 5] = 0
    M.upload(A)
    with pytest.raises(buffem.BuffError) as e:
        M.LUFactorize()
    assert e.value.status == 6


def test_solve_and_power_parity(sphere, oracle_lib):
    """config-1 physics on a smaller sphere: assemble, factor, solve 3 plane
    waves, EMT and overlap power -- GPU vs oracle + LAPACK."""
    mb, mo = buffem.Material(eps=4 + 0.2j), oracle_lib.material(eps=4 + 0.2j)
    Gb, Go = pair(sphere(3), mb, mo, oracle_lib=oracle_lib)
    w = 1.0
    M = Gb.AssembleVIEMatrix(w)
    Mo = Go.assemble(complex(w))
    lu = sl.lu_factor(Mo)
    M.LUFactorize()
    waves = [([1, 0, 0], [0, 0, 1]), ([0, 1, 0], [0, 0, 1]), ([0, 0, 1], [1, 0, 0])]
    B = np.zeros((Gb.TotalBFs, 3), complex, order="F")
    for i, (E0, nh) in enumerate(waves):
        B[:, i] = Gb.AssembleRHSVector(w, buffem.PlaneWave(E0, nh))
    Xo = sl.lu_solve(lu, B)
    X = B.copy(order="F")
    M.LUSolve(X)
    assert np.linalg.norm(X - Xo) <= 1e-10 * np.linalg.norm(Xo)
    for i, (E0, nh) in enumerate(waves):
        pw = buffem.PlaneWave(E0, nh)
        pb = Gb.GetPFTMatrix(X[:, i], w, pw)[0]
        po = Go.pft_emt(complex(w), Xo[:, i], np.array(E0, complex), np.array(nh, float))[0]
        np.testing.assert_allclose(pb, po, rtol=1e-9)
        ob = Gb.GetPFTMatrix(X[:, i], w, method=buffem.BG_PFT_OVERLAP)[0, 0]
        oo = Go.pft_opft(complex(w), Xo[:, i])[0]
        np.testing.assert_allclose(ob, oo, rtol=1e-9)


def test_full_size_properties(sphere):
    """n=8 sphere (N=5760): exact symmetry and a backward-stable solve."""
    G = buffem.SWGGeometry(meshfiles=sphere(8), materials=buffem.Material(eps=6 + 0.5j))
    M = G.AssembleVIEMatrix(1.0)
    A = M.download()
    assert np.array_equal(A, A.T)
    b = G.AssembleRHSVector(1.0, buffem.PlaneWave([1, 0, 0], [0, 0, 1]))
    M.LUFactorize()
    x = b.copy()
    M.LUSolve(x)
    r = A @ x - b
    assert np.linalg.norm(r) <= 1e-13 * np.linalg.norm(A, 1) * np.linalg.norm(x)


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (70, 33, 17), (300, 129, 64), (513, 200, 1000)])
def test_zgemm_device(M, N, K):
    import torch
    rng = np.random.default_rng(M + N + K)
    A = rng.normal(size=(M, K)) + 1j * rng.normal(size=(M, K))
    B = rng.normal(size=(K, N)) + 1j * rng.normal(size=(K, N))
    Cm = rng.normal(size=(M, N)) + 1j * rng.normal(size=(M, N))
    # column-major device copies: store the transposes row-major
    dA = torch.tensor(A.T.copy(), device="cuda")
    dB = torch.tensor(B.T.copy(), device="cuda")
    dC = torch.tensor(Cm.T.copy(), device="cuda")
    buffem.zgemm_sub_device(M, N, K, dA.data_ptr(), M, dB.data_ptr(), K, dC.data_ptr(), M)
    buffem.synchronize()
    out = dC.cpu().numpy().T
    ref = Cm - A @ B
    assert np.max(np.abs(out - ref)) <= 1e-13 * max(1.0, np.abs(A).max() * np.abs(B).max() * K)


@pytest.mark.parametrize("case", ["tensor_sphere", "two_spheres"])
def test_full_pft_parity(sphere, oracle_lib, case):
    """GetPFTMatrix, EMT, all 8 columns (PAbs, PScat, force, torque) -- GPU vs
    oracle, for one anisotropic sphere and for two displaced spheres (the
    different-object formulas and two torque centres).  Tolerance 1e-9 of
    the largest entry of each column kind."""
    w = 1.3
    if case == "tensor_sphere":
        t = np.array([[4, 0.5, 0], [0.5, 6, 0], [0, 0, 9]], complex) + 0.1j * np.eye(3)
        Gb, Go = pair(sphere(3), buffem.Material(kind=buffem.BG_MAT_CONST_TENSOR, tensor=t),
                      oracle_lib.material(kind=oracle_lib.MAT_CONST_TENSOR, tensor=t), oracle_lib=oracle_lib)
    else:
        disp = [[0, 0, 0], [0.3, 0, 2.4]]
        meshes = [sphere(2, radius=0.8), sphere(3, radius=1.0)]
        Gb, Go = pair(meshes, [buffem.Material(eps=4 + 0.2j), buffem.Material(eps=9 + 1j)],
                      [oracle_lib.material(eps=4 + 0.2j), oracle_lib.material(eps=9 + 1j)], disp=disp,
                      oracle_lib=oracle_lib)
    M = Go.assemble(complex(w))
    E0, nh = np.array([1, 0.3j, 0], complex), np.array([0.6, 0, 0.8])
    J = sl.lu_solve(sl.lu_factor(M), Go.rhs_planewave(complex(w), E0, nh))
    pb = Gb.GetPFTMatrix(J, w, buffem.PlaneWave(E0, nh), full=True)
    po = Go.pft_emt8(complex(w), J, E0, nh)
    for cols in (slice(0, 2), slice(2, 5), slice(5, 8)):
        scale = np.abs(po[:, cols]).max()
        np.testing.assert_allclose(pb[:, cols], po[:, cols], rtol=0, atol=1e-9 * scale)
    np.testing.assert_allclose(pb[:, :2], Gb.GetPFTMatrix(J, w, buffem.PlaneWave(E0, nh)), rtol=1e-13)
