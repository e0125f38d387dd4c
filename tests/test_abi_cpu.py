"""C-ABI checks that need no GPU: the library loads, exports every entry point
declared in include/buffem_b200.h, builds the host geometry with the
reference's numbering, and reports errors as status codes."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import buffem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "buffem_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bg_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol(buffem_lib):
    L = buffem_lib.lib()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(buffem.EXPORTS)


def test_face_numbering_matches_oracle(buffem_lib, oracle_lib, sphere, ref_mesh):
    for path in (sphere(2), sphere(3, jitter=0.05, seed=2), ref_mesh("sphere48"), ref_mesh("sphere533")):
        G = buffem.SWGGeometry(meshfiles=path, materials=buffem.Material(eps=4.0))
        O = oracle_lib.Geometry(path, oracle_lib.material(eps=4.0))
        assert G.TotalBFs == O.N
        assert np.array_equal(G.faces(0), O.faces(0))


def test_buffgeo_parser(buffem_lib, sphere, tmp_path):
    p = tmp_path / "two.buffgeo"
    mesh = sphere(2)
    p.write_text(f"OBJECT A\n MESHFILE {mesh}\n MATERIAL CONST_EPS_10\nENDOBJECT\n"
                 f"OBJECT B\n MESHFILE {mesh}\n MATERIAL CONST_EPS_4+0.2i\n DISPLACED 0 0 3\nENDOBJECT\n")
    G = buffem.SWGGeometry(str(p))
    assert G.NumObjects == 2 and G.TotalBFs == 2 * 72
    assert G.BFIndexOffset == [0, 72, 144]


def test_error_statuses(buffem_lib, tmp_path):
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(meshfiles=str(tmp_path / "nope.vmsh"), materials=buffem.Material(eps=2.0))
    assert e.value.status == -2
    # three tetrahedra sharing one face: InitFaceList topology error
    bad = tmp_path / "bad.vmsh"
    bad.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n6\n1 0 0 0\n2 1 0 0\n3 0 1 0\n"
                   "4 0 0 1\n5 0 0 -1\n6 1 1 1\n$EndNodes\n$Elements\n3\n1 4 2 0 1 1 2 3 4\n"
                   "2 4 2 0 1 1 3 2 5\n3 4 2 0 1 1 2 3 6\n$EndElements\n")
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(meshfiles=str(bad), materials=buffem.Material(eps=2.0))
    assert e.value.status == -3
    p = tmp_path / "x.buffgeo"
    p.write_text("OBJECT A\n MESHFILE none.vmsh\n MATERIAL Gold\nENDOBJECT\n")
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(str(p))
    assert e.value.status == -2


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure mode")
def test_compute_without_gpu_fails_loudly(buffem_lib, sphere):
    G = buffem.SWGGeometry(meshfiles=sphere(1), materials=buffem.Material(eps=2.0))
    with pytest.raises(buffem.BuffError) as e:
        G.AllocateVIEMatrix()
    assert e.value.status == -4
    assert "no CPU fallback" in str(e.value) or "CUDA" in str(e.value)


def test_batch_sweep_rejects_bad_arguments(buffem_lib):
    import ctypes as C
    import numpy as np
    L = buffem_lib.lib()
    w = np.array([1.0, 0.0])
    E0 = np.zeros(6)
    nh = np.array([0.0, 0.0, 1.0])
    out = np.zeros(4)
    st = L.bg_batch_sweep(None, 1, w.ctypes.data_as(C.c_void_p), 1, E0.ctypes.data_as(C.c_void_p),
                          nh.ctypes.data_as(C.c_void_p), 1, 0, out.ctypes.data_as(C.c_void_p), None)
    assert st == buffem_lib.BG_ERR_ARG


def test_fibbi_load_rejects_foreign_files(buffem_lib, tmp_path, ref_mesh):
    """A file without the reference's FIBBI signature, or with a partial
    record, is refused before any device work."""
    G = buffem_lib.SWGGeometry(meshfiles=ref_mesh("sphere48"), materials=buffem_lib.Material(eps=10.0))
    bad = tmp_path / "bad.cache"
    bad.write_bytes(b"NOT_A_CACHE\0\0" + bytes(156))
    with pytest.raises(buffem_lib.BuffError) as e:
        G.PreloadFIBBICache(str(bad))
    assert e.value.status == buffem_lib.BG_ERR_IO
    short = tmp_path / "short.cache"
    short.write_bytes(b"FIBBI_GCACHE\0" + bytes(155))
    with pytest.raises(buffem_lib.BuffError) as e:
        G.PreloadFIBBICache(str(short))
    assert e.value.status == buffem_lib.BG_ERR_IO


def test_get_fields_rejects_bad_arguments(buffem_lib, ref_mesh):
    """GetFields checks its arguments before any device work: a negative
    point count, missing points or output, a plane wave without nhat; zero
    points is a no-op."""
    import ctypes as C
    import numpy as np
    L = buffem_lib.lib()
    G = buffem_lib.SWGGeometry(meshfiles=ref_mesh("sphere48"), materials=buffem_lib.Material(eps=10.0))
    X = np.zeros((2, 3))
    out = np.zeros(24)
    E0 = np.zeros(6)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert L.bg_get_fields(G.h, 1.0, 0.0, None, None, None, -1, p(X), p(out)) == buffem_lib.BG_ERR_ARG
    assert L.bg_get_fields(G.h, 1.0, 0.0, None, None, None, 2, None, p(out)) == buffem_lib.BG_ERR_ARG
    assert L.bg_get_fields(G.h, 1.0, 0.0, None, None, None, 2, p(X), None) == buffem_lib.BG_ERR_ARG
    assert L.bg_get_fields(G.h, 1.0, 0.0, None, p(E0), None, 2, p(X), p(out)) == buffem_lib.BG_ERR_ARG
    assert L.bg_get_fields(None, 1.0, 0.0, None, None, None, 2, p(X), p(out)) == buffem_lib.BG_ERR_ARG
    assert L.bg_get_fields(G.h, 1.0, 0.0, None, None, None, 0, None, None) == 0
    with pytest.raises(ValueError):
        G.GetFields(None, np.zeros(G.TotalBFs + 1, complex), 1.0, X)


def test_assemble_with_copy_rejects_missing_matrices(buffem_lib, ref_mesh):
    """The assembly with a complex64 copy checks its handles before any device
    work: a missing geometry, matrix or copy is BG_ERR_ARG with a message."""
    L = buffem_lib.lib()
    G = buffem_lib.SWGGeometry(meshfiles=ref_mesh("sphere48"), materials=buffem_lib.Material(eps=10.0))
    assert L.bg_assemble_with_copy(None, 1.0, 0.0, None, None) == buffem_lib.BG_ERR_ARG
    assert L.bg_assemble_with_copy(G.h, 1.0, 0.0, None, None) == buffem_lib.BG_ERR_ARG
    assert b"bg_assemble_with_copy" in L.bg_last_error()


def test_neq_entry_points_reject_bad_arguments(buffem_lib, ref_mesh):
    """buff-neq's entry points check their arguments before any device work."""
    L = buffem_lib.lib()
    G = buffem.SWGGeometry(meshfiles=ref_mesh("sphere48"), materials=buffem.Material(eps=4.0))
    out = C.c_void_p()
    flux = np.zeros(8)
    assert L.bg_neq_create(None, C.byref(out)) == buffem_lib.BG_ERR_ARG
    assert L.bg_neq_create(G.h, None) == buffem_lib.BG_ERR_ARG
    assert L.bg_neq_flux(None, 1.0, 0.0, flux.ctypes.data_as(C.c_void_p)) == buffem_lib.BG_ERR_ARG
    assert L.bg_neq_dressed_rytov(None, 1.0, 0.0, 0, flux.ctypes.data_as(C.c_void_p)) == buffem_lib.BG_ERR_ARG
    dr = np.zeros(2)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert L.bg_pft_dr_device(None, 1.0, 0.0, p(dr), 10, p(flux)) == buffem_lib.BG_ERR_ARG
    assert L.bg_pft_dr_device(G.h, 0.0, 0.0, p(dr), G.TotalBFs, p(flux)) == buffem_lib.BG_ERR_ARG
    assert L.bg_pft_dr_device(G.h, 1.0, 0.0, p(dr), G.TotalBFs - 1, p(flux)) == buffem_lib.BG_ERR_ARG
    L.bg_neq_destroy(None)


NULL_PROBE = r"""
import re, sys
sys.path.insert(0, sys.argv[1])
import buffem
L = buffem.lib()
src = open(sys.argv[2]).read().replace("\n", " ")
for fn, args in sorted(re.findall(r"L\.(bg_[a-z0-9_]+)\.argtypes = \[([^\]]*)\]", src)):
    parts = [a.strip() for a in re.split(r",(?![^\[]*\])", args) if a.strip()]
    vals = [0 if a in ("I", "C.c_int", "C.c_ulonglong") else 1.0 if a == "D" else None for a in parts]
    r = getattr(L, fn)(*vals)
    print(fn, r, flush=True)
"""


def test_every_entry_point_rejects_null_arguments(buffem_lib, tmp_path):
    """Every entry point called with null handles and pointers returns an
    error status (void destroy functions return) instead of crashing, on a
    machine without a GPU (where a call that gets as far as the device
    returns the no-device status); run in a child process so a crash fails
    the test rather than the session."""
    import subprocess
    import sys
    script = tmp_path / "probe.py"
    script.write_text(NULL_PROBE)
    binding = os.path.join(ROOT, "buff-em_b200", "buffem.py")
    r = subprocess.run([sys.executable, str(script), os.path.join(ROOT, "buff-em_b200"), binding],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    results = dict(line.split() for line in r.stdout.strip().splitlines())
    assert len(results) >= 60
    for fn, ret in results.items():
        assert ret == "None" if fn.endswith("_destroy") else int(ret) < 0, (fn, ret)
