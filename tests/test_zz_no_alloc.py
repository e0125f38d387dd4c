"""Allocation-free device solve (bg_lu_solve_device_noalloc), -m gpu.

Callers that cannot allocate GPU memory at solve time -- an application whose
framework already holds the device memory in its own pool, or a time-critical
loop that cannot take an allocation's failure or implicit synchronisation --
use this entry point, whose only scratch is a fixed device array inside the
library.  The test calls it twice in a row through the C-ABI and checks each
result against the allocating bg_lu_solve_device on the same right-hand
sides (same kernels, so to 1e-14 relative), plus the size limits.  Kept in a
file of its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

import buffem

pytestmark = pytest.mark.gpu


def test_noalloc_solve_matches_allocating_solve(sphere):
    import torch
    G = buffem.SWGGeometry(meshfiles=sphere(3), materials=buffem.Material(eps=4 + 0.2j), singular_order=6)
    N = G.TotalBFs
    M = G.AssembleVIEMatrix(1.0)
    A = M.download()          # before the factorization overwrites it
    M.LUFactorize()
    L = buffem.lib()
    rng = np.random.default_rng(11)
    for call in range(2):
        nrhs = 3 if call == 0 else 4
        B = rng.normal(size=(nrhs, N)) + 1j * rng.normal(size=(nrhs, N))  # rows = columns of B (column-major)
        d1 = torch.tensor(B, dtype=torch.complex128, device="cuda")
        d2 = d1.clone()
        buffem._check(L.bg_lu_solve_device(M.h, C.c_void_p(d1.data_ptr()), N, nrhs))
        buffem._check(L.bg_lu_solve_device_noalloc(M.h, C.c_void_p(d2.data_ptr()), N, nrhs))
        buffem.synchronize()
        x1, x2 = d1.cpu().numpy(), d2.cpu().numpy()
        assert np.max(np.abs(x1 - x2)) <= 1e-14 * np.max(np.abs(x1)), call
        # and it solves the system
        r = A @ x2.T - B.T
        assert np.linalg.norm(r) <= 1e-12 * np.linalg.norm(B)


def test_noalloc_solve_rejects_sizes_beyond_its_scratch(sphere):
    import torch
    G = buffem.SWGGeometry(meshfiles=sphere(2), materials=buffem.Material(eps=4.0), singular_order=6)
    M = G.AssembleVIEMatrix(1.0)
    M.LUFactorize()
    N = G.TotalBFs
    d = torch.zeros((5, N), dtype=torch.complex128, device="cuda")
    st = buffem.lib().bg_lu_solve_device_noalloc(M.h, C.c_void_p(d.data_ptr()), N, 5)
    assert st == -1
    assert "at most 4" in buffem.lib().bg_last_error().decode()


def test_noalloc_solve_rejects_more_bytes_than_its_scratch(tmp_path):
    """N = 65,537 with 4 complex128 right-hand sides needs 4 MiB + 64 bytes,
    just above the fixed array: rejected before any device work (the size is
    checked before the factorization state, so the 69 GB matrix is only
    allocated, never assembled or factored)."""
    import torch
    from test_gpu_parity import _chain_mesh
    N = 65537
    need = 16 * N * N
    if torch.cuda.mem_get_info()[0] < need + (4 << 30):
        pytest.skip("not enough free device memory for the N = 65,537 matrix")
    path = str(tmp_path / "chain.vmsh")
    _chain_mesh(path, N)
    G = buffem.SWGGeometry(meshfiles=path, materials=buffem.Material(eps=2.0))
    assert G.TotalBFs == N
    M = G.AllocateVIEMatrix()
    d = torch.zeros((4, N), dtype=torch.complex128, device="cuda")
    st = buffem.lib().bg_lu_solve_device_noalloc(M.h, C.c_void_p(d.data_ptr()), N, 4)
    assert st == -1
    assert "exceeds its fixed" in buffem.lib().bg_last_error().decode()
    del M
