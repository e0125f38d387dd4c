"""Refined singular rule on the GPU against the oracle (needs a B200: -m gpu).

The GPU keeps 24 moments per ordered tetrahedron pair sharing 2-4 vertices
(csrc/singular.cu); the reference evaluates the same static integrals with
Taylor-Duffy at relative tolerance 1e-6 (TTaylorDuffy.cc:284-343,
SWGGeometry.cc:46-47).  Tolerances:
  * GPU moments = the oracle's refined moments (or_sing_moments_refined, the
    same scheme summed in another order) to 1e-10 of each moment's scale
    (|M0| of its kernel, times h or h^2 for first and second moments, h the
    diameter of the row tetrahedron); the refined/not-refined flags agree;
  * every sampled pair within 2e-8 of the adaptive accuracy reference
    (or_sing_static_adaptive), far below the reference's 1e-6.
"""
import numpy as np
import pytest

import buffem

pytestmark = pytest.mark.gpu

GPRE = np.array([0.25, 0.25, 0.125]) / np.pi


def gpu_pairs(G):
    pairs, verts, mom = G.singular_moments()
    xyz, _ = G.vertices(0)
    return pairs, xyz[verts[:, :4]], xyz[verts[:, 4:]], mom


def moment_scales(VA, M):
    """(P, 24) scales: |M0| per kernel times 1, h, h^2 (h = diameter of A)."""
    d = VA[:, :, None, :] - VA[:, None, :, :]
    h2 = (d ** 2).sum(-1).reshape(len(VA), -1).max(1)
    h = np.sqrt(h2)
    sc = np.zeros_like(M)
    for pk in range(3):
        m0 = np.abs(M[:, 8 * pk])
        sc[:, 8 * pk] = m0
        sc[:, 8 * pk + 1:8 * pk + 7] = (m0 * h)[:, None]
        sc[:, 8 * pk + 7] = m0 * h2
    return sc


@pytest.mark.parametrize("name", ["sphere533", "sphere677"])
def test_refined_moments_match_oracle(name, ref_mesh, oracle_lib):
    """The reference's own meshes (src/unitTests/Sphere_533.vmsh,
    examples/MieScattering/Sphere_677.vmsh), every singular pair."""
    G = buffem.SWGGeometry(meshfiles=ref_mesh(name), materials=buffem.Material(eps=10.0))
    st = G.singular_stats()
    assert st["refine_on"] == 1 and st["status"] == 0
    pairs, VA, VB, mom = gpu_pairs(G)
    assert len(pairs) == st["pairs"] > 1000
    Mo, sto, ev, _, _ = oracle_lib.sing_moments_refined_batch(pairs[:, 2], VA, VB)
    assert np.all(sto == 0)
    gflag = (pairs[:, 3] & 1) == 1
    assert np.array_equal(gflag, ev > 0)
    assert st["refined"] == int(gflag.sum()) > 0
    assert st["refine_points"] == int(ev.sum())
    err = np.abs(mom - Mo) / moment_scales(VA, Mo)
    assert err.max() < 1e-10, err.max()


def test_refined_rule_accuracy_against_adaptive_reference(ref_mesh, oracle_lib):
    """Sphere_533: the 40 worst-shaped self pairs, every pair sharing 3
    vertices of the 40 worst-shaped tetrahedra, and 60 seeded pairs sharing 2
    vertices, as the six pair values of GetGME_TetTetInt(KERNEL_STATIC) for
    Q, Q' = the last vertices; error relative to each kernel's magnitude."""
    G = buffem.SWGGeometry(meshfiles=ref_mesh("sphere533"), materials=buffem.Material(eps=10.0))
    pairs, VA, VB, mom = gpu_pairs(G)

    def shape(V):
        s = np.linalg.svd(V[1:] - V[0], compute_uv=False)
        return s[-1] / s[0]

    sh = np.array([shape(V) for V in VA])
    c = pairs[:, 2]
    worst_tets = set(pairs[np.argsort(sh)[:200], 0][:40])
    pick = list(np.where(c == 4)[0][np.argsort(sh[c == 4])[:40]])
    pick += [i for i in np.where(c == 3)[0] if pairs[i, 0] in worst_tets]
    rng = np.random.default_rng(5)
    pick += list(rng.choice(np.where(c == 2)[0], 60, replace=False))
    worst = 0.0
    for i in pick:
        Q, QP = VA[i][-1], VB[i][-1]
        ref, _ = oracle_lib.sing_static_adaptive(int(c[i]), VA[i], VB[i], Q, QP, 5, 1e-10)
        h2 = max(np.sum((a - b) ** 2) for a in VA[i] for b in VA[i])
        scale = np.repeat(np.abs(ref[1::2]), 2) * np.tile([h2, 1.0], 3)
        val = oracle_lib.moments_to_values(mom[i], VA[i], VB[i], Q, QP)
        worst = max(worst, float(np.max(np.abs(val - ref) / scale)))
    assert worst < 2e-8, worst


def test_fixed_rule_still_available(sphere, oracle_lib):
    """singular_refine=False keeps the fixed order-n rule (GPU = oracle's
    or_sing_moments at order n to 1e-10)."""
    G = buffem.SWGGeometry(meshfiles=sphere(2, jitter=0.05, seed=3), materials=buffem.Material(eps=4.0),
                           singular_order=8, singular_refine=False)
    st = G.singular_stats()
    assert st["refine_on"] == 0 and st["refined"] == 0 and st["refine_points"] == 0
    pairs, VA, VB, mom = gpu_pairs(G)
    ref = np.array([oracle_lib.sing_moments(int(cc), a, b, 8)[0] for cc, a, b in zip(pairs[:, 2], VA, VB)])
    assert np.max(np.abs(mom - ref) / moment_scales(VA, ref)) < 1e-10


def test_singular_rule_settings_are_checked(sphere):
    G = buffem.SWGGeometry(meshfiles=sphere(1), materials=buffem.Material(eps=4.0))
    with pytest.raises(buffem.BuffError):
        G2 = buffem.SWGGeometry(meshfiles=sphere(1), materials=buffem.Material(eps=4.0), singular_order=16)
    G.singular_stats()   # runs the precompute
    with pytest.raises(buffem.BuffError):
        buffem._check(buffem.lib().bg_geometry_set_singular_refine(G.h, 0, 1e-8, 1e-9))
