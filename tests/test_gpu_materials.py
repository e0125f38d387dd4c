"""Frequency-dependent MATERIAL sections on the device: at each frequency the
assembled matrix and the overlap absorbed power equal those of the same
geometry with the constant permittivity eps(Omega) (the device copy of the
materials is refreshed per call)."""
import numpy as np
import pytest

import buffem

DRUDE = """MATERIAL Metal
  wp = 1.2e15; gam = 4.0e13
  Eps(w) = 1 - wp^2 / (w * (w + i*gam))
ENDMATERIAL
"""


@pytest.mark.gpu
def test_dispersive_assembly_matches_constant(sphere, tmp_path):
    mesh = sphere(3)
    p = tmp_path / "d.buffgeo"
    p.write_text(DRUDE + f"OBJECT A\n MESHFILE {mesh}\n MATERIAL Metal\nENDOBJECT\n")
    G = buffem.SWGGeometry(str(p))
    pw = buffem.PlaneWave([1, 0, 0], [0, 0, 1])
    for omega in (0.8, 1.3, 0.8 + 0.01j):
        eps = G.material_eps(0, omega)
        H = buffem.SWGGeometry(meshfiles=mesh, materials=buffem.Material(eps=eps))
        M = G.AssembleVIEMatrix(omega).download()
        Mc = H.AssembleVIEMatrix(omega).download()
        assert np.array_equal(M, Mc), omega
        J = np.linalg.solve(Mc, H.AssembleRHSVector(omega, pw))
        pa = G.GetPFTMatrix(J, omega, pw, method=buffem.BG_PFT_OVERLAP)
        pc = H.GetPFTMatrix(J, omega, pw, method=buffem.BG_PFT_OVERLAP)
        assert np.array_equal(pa, pc), omega


@pytest.mark.gpu
def test_svtensor_assembly_matches_constant_tensor(sphere, tmp_path):
    """An SVTENSOR tensor of frequency: the matrix at each frequency equals
    that of the same mesh with the constant tensor evaluated there."""
    mesh = sphere(3)
    (tmp_path / "t.SVTensor").write_text(DRUDE + "Qxx = MP_Metal\nQyy = 3 + 0.1*i\nQzz = 5\nQxy = 0.2*w/3e14\n")
    p = tmp_path / "t.buffgeo"
    p.write_text(f"OBJECT A\n MESHFILE {mesh}\n SVTENSOR t.SVTensor\nENDOBJECT\n")
    G = buffem.SWGGeometry(str(p))
    for omega in (0.9, 1.4):
        T = G.material_tensor(0, omega)
        H = buffem.SWGGeometry(meshfiles=mesh, materials=buffem.Material(kind=buffem.BG_MAT_CONST_TENSOR, tensor=T))
        assert np.array_equal(G.AssembleVIEMatrix(omega).download(), H.AssembleVIEMatrix(omega).download()), omega
