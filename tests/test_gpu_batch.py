"""Batching form on the GPU (-m gpu): the batched frequency sweep (captured
CUDA graphs replayed per frequency, concurrent slots, online autotuning)
against the same jobs run one by one through the plain path
(AssembleVIEMatrix, LUFactorize, LUSolve, GetPFTMatrix with the overlap
method).  Tolerance: 1e-10 relative on every absorbed power."""
import numpy as np
import pytest

import buffem

pytestmark = pytest.mark.gpu

WAVE = buffem.PlaneWave([1, 0, 0], [0, 0, 1])


def two_spheres(sphere):
    """Two spheres of uneven size with a Gaussian-profile permittivity each,
    3 + 1.5 exp(-|x - c|^2) + 0.1i about its own centre."""
    r1, r2, gap = 0.7, 1.1, 0.4
    z2 = r1 + gap + r2
    mats = [buffem.Material(kind=buffem.BG_MAT_GAUSSIAN, eps=3 + 0.1j, amp=1.5, width=1.0, center=(0, 0, 0)),
            buffem.Material(kind=buffem.BG_MAT_GAUSSIAN, eps=3 + 0.1j, amp=1.5, width=1.0, center=(0, 0, z2))]
    return buffem.SWGGeometry(meshfiles=[sphere(2, radius=r1), sphere(3, radius=r2)], materials=mats,
                              displacements=[[0, 0, 0], [0, 0, z2]])


def sequential(G, omegas):
    out = np.zeros((len(omegas), buffem.BG_BATCH_MAXOBJ))
    for j, w in enumerate(omegas):
        M = G.AssembleVIEMatrix(w)
        M.LUFactorize()
        x = G.AssembleRHSVector(w, WAVE)
        M.LUSolve(x)
        pft = G.GetPFTMatrix(x, w, WAVE, method=buffem.BG_PFT_OVERLAP)
        out[j, :G.NumObjects] = pft[:, 0]
    return out


def test_batch_sweep_matches_one_by_one(sphere):
    geoms = [buffem.SWGGeometry(meshfiles=sphere(4), materials=buffem.Material(eps=4 + 0.2j)), two_spheres(sphere)]
    omegas = np.logspace(-2, 1, 7)
    pabs, st = buffem.BatchSweep(geoms, omegas, WAVE, max_streams=2)
    assert st[1] == len(geoms) * len(omegas) and st[2] == 1
    assert st[3] == 0          # every slot's launch sequence was captured into a graph
    for i, G in enumerate(geoms):
        ref = sequential(G, omegas)
        np.testing.assert_allclose(pabs[i], ref, rtol=1e-10, atol=1e-14 * np.abs(ref).max())
        assert np.all(pabs[i, :, G.NumObjects:] == 0)
    # direct launches (no graphs) give the same numbers
    pabs2, st2 = buffem.BatchSweep(geoms, omegas, WAVE, max_streams=2, graphs=False)
    assert st2[2] == 0
    np.testing.assert_allclose(pabs2, pabs, rtol=1e-12, atol=0)


def test_batch_sweep_reuses_tuning_for_a_size_class(sphere):
    # N = 1350 (size class 2, not used by the other tests here)
    G1 = buffem.SWGGeometry(meshfiles=sphere(5, jitter=0.05, seed=1), materials=buffem.Material(eps=6 + 0.5j))
    G2 = buffem.SWGGeometry(meshfiles=sphere(5, jitter=0.05, seed=2), materials=buffem.Material(eps=6 + 0.5j))
    omegas = np.linspace(0.5, 3.0, 12)
    pabs, st = buffem.BatchSweep([G1, G2], omegas, WAVE, max_streams=4)
    rows1, slots1, t1, tile1 = st[4:8]
    rows2, slots2, t2, tile2 = st[8:12]
    assert rows1 in (16, 32, 64) and slots1 in (1, 2, 4) and t1 > 0 and tile1 in (0, 1, 2)
    # same size class: the first geometry's choice
    assert (rows2, slots2, tile2) == (rows1, slots1, tile1) and t2 == 0
    np.testing.assert_allclose(pabs[1], sequential(G2, omegas), rtol=1e-10)
