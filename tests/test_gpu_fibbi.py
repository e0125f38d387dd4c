"""The reference's FIBBI cache file format on the GPU path (-m gpu):
files written from the device near table parse with an independent reader
(signature, record size, keys recomputed from the mesh), load back into a
fresh copy of the object (every record) and into a displaced copy (exactly
the records whose float keys the displacement leaves unchanged), and a file
written by that independent writer from the oracle's integrals replaces the
device's own near table so that the assembled matrix matches the oracle's to
rounding."""
import struct

import numpy as np
import pytest

import buffem
import meshgen

pytestmark = pytest.mark.gpu

SIG = b"FIBBI_GCACHE\0"
REC = 27 * 4 + 6 * 8


def keys_from_mesh(V, faces, pairs):
    """GetFIBBICacheKey: float differences of QM_a, V1_a, V2_a, V3_a, QP_b,
    QM_b, V1_b, V2_b, V3_b from QP_a (faces: iV1, iV2, iV3, iQP, iQM, ...)."""
    out = []
    for a, b in pairs:
        fa, fb = faces[a], faces[b]
        qpa = V[fa[3]]
        pts = [V[fa[4]], V[fa[0]], V[fa[1]], V[fa[2]], V[fb[3]], V[fb[4]], V[fb[0]], V[fb[1]], V[fb[2]]]
        out.append(np.concatenate([(p - qpa) for p in pts]).astype(np.float32).tobytes())
    return out


def read_cache(path):
    raw = open(path, "rb").read()
    assert raw[:13] == SIG and (len(raw) - 13) % REC == 0
    recs = {}
    for off in range(13, len(raw), REC):
        recs[raw[off:off + 108]] = np.array(struct.unpack("6d", raw[off + 108:off + REC]))
    return recs, (len(raw) - 13) // REC


def write_cache(path, keys, data):
    with open(path, "wb") as f:
        f.write(SIG)
        for k, d in zip(keys, data):
            f.write(k)
            f.write(struct.pack("6d", *d))


def test_store_format_and_displaced_reload(sphere, tmp_path):
    n = 3
    G = buffem.SWGGeometry(meshfiles=sphere(n), materials=buffem.Material(eps=6 + 0.5j))
    pairs, data = G.near_data()
    path = tmp_path / "sphere.cache"
    assert G.StoreFIBBICache(str(path)) == len(pairs)
    recs, nrec = read_cache(path)
    assert nrec == len(pairs) == len(recs)
    V, _ = meshgen.sphere_arrays(n)
    for k, d in zip(keys_from_mesh(V, G.faces(0), pairs), data):
        np.testing.assert_array_equal(recs[k], d)
    # a fresh copy of the object: every record matches
    G1 = buffem.SWGGeometry(meshfiles=sphere(n), materials=buffem.Material(eps=6 + 0.5j))
    assert G1.PreloadFIBBICache(str(path)) == len(pairs)
    np.testing.assert_array_equal(G1.near_data()[1], data)
    # a displaced copy: the keys are float differences, so only the records
    # whose rounded differences are unchanged by the displacement match
    d = np.array([5.0, -2.0, 3.0])
    G2 = buffem.SWGGeometry(meshfiles=sphere(n), materials=buffem.Material(eps=6 + 0.5j), displacements=[d])
    same = [k1 == k2 for k1, k2 in zip(keys_from_mesh(V, G.faces(0), pairs), keys_from_mesh(V + d, G.faces(0), pairs))]
    assert G2.PreloadFIBBICache(str(path)) == sum(same)
    pairs2, data2 = G2.near_data()
    np.testing.assert_array_equal(pairs2, pairs)
    np.testing.assert_array_equal(data2[np.array(same)], data[np.array(same)])


def test_foreign_cache_replaces_near_table(sphere, oracle_lib, tmp_path):
    n = 2
    path_mesh = sphere(n)
    Go = oracle_lib.Geometry(path_mesh, oracle_lib.material(eps=4 + 0.2j), nang=6)
    G = buffem.SWGGeometry(meshfiles=path_mesh, materials=buffem.Material(eps=4 + 0.2j), singular_order=12)
    pairs, own = G.near_data()
    V, _ = meshgen.sphere_arrays(n)
    ref = np.array([Go.fibbi(int(a), int(b)) for a, b in pairs])
    assert np.abs(ref - own).max() > 0          # different singular rules: the tables differ slightly
    path = tmp_path / "oracle.cache"
    write_cache(path, keys_from_mesh(V, G.faces(0), pairs), ref)
    assert G.PreloadFIBBICache(str(path)) == len(pairs)
    _, loaded = G.near_data()
    np.testing.assert_array_equal(loaded, ref)
    M = G.AssembleVIEMatrix(1.0).download()
    Mo = Go.assemble(1.0 + 0j)
    assert np.abs(M - Mo).max() <= 1e-13 * np.abs(Mo).max()
