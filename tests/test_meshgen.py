import numpy as np

import meshgen


def test_counts_and_orientation():
    for n in (1, 2, 5):
        V, T = meshgen.sphere_arrays(n)
        assert len(V) == (n + 1) ** 3 and len(T) == 6 * n ** 3
        assert np.all(meshgen.signed_volumes(V, T) > 0)
        assert np.allclose(np.max(np.linalg.norm(V, axis=1)), 1.0)


def test_jitter_keeps_orientation():
    V, T = meshgen.sphere_arrays(4, jitter=0.05, seed=3)
    assert np.all(meshgen.signed_volumes(V, T) > 0)
    V2, _ = meshgen.sphere_arrays(4, jitter=0.05, seed=3)
    assert np.array_equal(V, V2)
