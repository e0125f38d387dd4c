"""buff-neq flux chain on the GPU (-m gpu) against the oracle's step-by-step
restatement of ComputeDressedRytovMatrix / GetFlux (GetFlux.cc:155-436).

Tolerances: the dressed Rytov matrix to 1e-9 of its largest entry (FP64
throughout; the chain has three products with S^-1, an LU and two N-column
solves, summed in other orders than LAPACK's); the flux columns to 1e-8 of
the largest entry of each column kind.  At full size: Hermitian DR, PAbs =
-PRad for one body, and the radiated power against Krueger's dipole formula.
"""
import numpy as np
import pytest

import buffem
from test_gpu_parity import pair
from test_oracle_pins import _krueger_prad

pytestmark = pytest.mark.gpu


def flux_close(Fg, Fo, rtol=1e-8):
    for cols in (slice(0, 2), slice(2, 5), slice(5, 8)):
        scale = np.abs(Fo[..., cols]).max()
        assert np.abs(Fg[..., cols] - Fo[..., cols]).max() <= rtol * scale, (cols, Fg[..., cols], Fo[..., cols])


def test_neq_one_sphere(sphere, oracle_lib):
    Gb, Go = pair(sphere(3, jitter=0.05, seed=2), buffem.Material(eps=4 + 0.2j),
                  oracle_lib.material(eps=4 + 0.2j), oracle_lib=oracle_lib)
    w = 0.6
    neq = buffem.NEQ(Gb)
    DRg = neq.DressedRytov(w, 0)
    DRo = Go.dressed_rytov(complex(w), 0)
    assert np.abs(DRg - DRo).max() <= 1e-9 * np.abs(DRo).max()
    flux_close(neq.GetFlux(w), Go.neq_flux(complex(w)))
    # a second frequency re-factors W; the first again matches
    neq.GetFlux(1.1)
    assert np.abs(neq.DressedRytov(w, 0) - DRo).max() <= 1e-9 * np.abs(DRo).max()


def test_neq_two_objects(sphere, oracle_lib):
    """Two displaced spheres of different meshes and materials: flux from
    each source to each destination (heat transfer and forces)."""
    disp = [[0, 0, 0], [0.3, 0, 2.4]]
    meshes = [sphere(2, radius=0.8), sphere(3, radius=1.0)]
    Gb, Go = pair(meshes, [buffem.Material(eps=4 + 0.2j), buffem.Material(eps=9 + 1j)],
                  [oracle_lib.material(eps=4 + 0.2j), oracle_lib.material(eps=9 + 1j)], disp=disp,
                  oracle_lib=oracle_lib)
    w = 0.9
    neq = buffem.NEQ(Gb)
    Fg, Fo = neq.GetFlux(w), Go.neq_flux(complex(w))
    flux_close(Fg, Fo)
    for s in range(2):
        DRg, DRo = neq.DressedRytov(w, s), Go.dressed_rytov(complex(w), s)
        assert np.abs(DRg - DRo).max() <= 1e-9 * np.abs(DRo).max()


def test_pft_with_dr_matches_current_form(sphere, oracle_lib):
    """GetPFTMatrix with DR = J J^H equals the scattering part of the
    current-vector form (no incident field), through the device entry point."""
    import ctypes as C
    import torch
    Gb, Go = pair(sphere(3), buffem.Material(eps=4 + 0.2j), oracle_lib.material(eps=4 + 0.2j),
                  oracle_lib=oracle_lib)
    rng = np.random.default_rng(4)
    J = rng.normal(size=Gb.TotalBFs) + 1j * rng.normal(size=Gb.TotalBFs)
    DR = torch.tensor(np.asfortranarray(np.outer(J, J.conj())).T.copy(), dtype=torch.complex128, device="cuda")
    out = np.zeros(8)
    buffem._check(buffem.lib().bg_pft_dr_device(Gb.h, 1.0, 0.0, C.c_void_p(DR.data_ptr()), Gb.TotalBFs,
                                                  buffem._ptr(out)))
    ref = Go.pft_emt8(1.0 + 0j, J, np.zeros(3, complex), np.array([0, 0, 1.0]))[0]
    np.testing.assert_allclose(out, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())


def test_neq_full_size_properties(sphere):
    """A sphere of N = 8262 basis functions: DR Hermitian, PAbs = -PRad, and
    the radiated power with the self pairs weighted 1/2 within 25% of
    Krueger's dipole formula (the l = 1 expansion is accurate at kR = 0.3)."""
    import ctypes as C
    import torch
    eps, w = 4 + 0.2j, 0.3
    G = buffem.SWGGeometry(meshfiles=sphere(9), materials=buffem.Material(eps=eps))
    N = G.TotalBFs
    neq = buffem.NEQ(G)
    F = neq.GetFlux(w)
    assert abs(F[0, 0, 0] + F[0, 0, 1]) <= 1e-13 * abs(F[0, 0, 1])
    DR = neq.DressedRytov(w, 0)
    assert np.abs(DR - DR.conj().T).max() <= 1e-10 * np.abs(DR).max()
    d = torch.tensor(np.diag(np.diag(DR)), dtype=torch.complex128, device="cuda")
    out = np.zeros(8)
    buffem._check(buffem.lib().bg_pft_dr_device(G.h, w, 0.0, C.c_void_p(d.data_ptr()), N, buffem._ptr(out)))
    r = (F[0, 0, 1] - out[1] / 2) / _krueger_prad(eps, w)
    assert 0.75 < r < 1.05, r


@pytest.mark.parametrize("kind", ["tensor", "gauss"])
def test_neq_anisotropic_and_varying_materials(sphere, oracle_lib, kind):
    """The overlap rows V and Rytov evaluate eps(x) at every quadrature point:
    an anisotropic constant tensor and a Gaussian bump eps(x) against the
    oracle (dressed Rytov matrix and flux columns)."""
    from test_gpu_parity import mats
    val = [[4, .5, 0], [.5, 6, 0], [0, 0, 9]] if kind == "tensor" else None
    mb, mo = mats(kind, val, oracle_lib)
    Gb, Go = pair(sphere(3, jitter=0.05, seed=5), mb, mo, oracle_lib=oracle_lib)
    w = 0.7
    neq = buffem.NEQ(Gb)
    DRg, DRo = neq.DressedRytov(w, 0), Go.dressed_rytov(complex(w), 0)
    assert np.abs(DRg - DRo).max() <= 1e-9 * np.abs(DRo).max()
    flux_close(neq.GetFlux(w), Go.neq_flux(complex(w)))
