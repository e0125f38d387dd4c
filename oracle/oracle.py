"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, as the checker and as the timed CPU restatement of the
reference path.  The product library never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

MAT_CONST_ISO, MAT_CONST_TENSOR, MAT_JANUS_Z, MAT_GAUSSIAN = 0, 1, 2, 3

# refined singular rule: fixed orders n and n + 2 (n = 10), refinement boxes
# of 6 Gauss points per dimension where the two orders differ by more than
# 1e-8 of a moment's scale, boxes closed when a split changes them by <= 1e-9
REFINE_ORDER, REFINE_NG, REFINE_FLAG, REFINE_TOL = 10, 6, 1e-8, 1e-9


class OMat(C.Structure):
    _fields_ = [("kind", C.c_int), ("eps", C.c_double * 18), ("eps2", C.c_double * 2),
                ("center", C.c_double * 3), ("amp", C.c_double * 2), ("width", C.c_double)]


def material(kind=MAT_CONST_ISO, eps=4 + 0.2j, tensor=None, eps2=None, center=(0, 0, 0),
             amp=0.0, width=1.0) -> OMat:
    m = OMat()
    m.kind = kind
    if tensor is not None:
        t = np.asarray(tensor, dtype=np.complex128).reshape(3, 3)
        for i in range(3):
            for j in range(3):
                m.eps[2 * (3 * i + j)] = t[i, j].real
                m.eps[2 * (3 * i + j) + 1] = t[i, j].imag
    else:
        m.eps[0], m.eps[1] = complex(eps).real, complex(eps).imag
    if eps2 is not None:
        m.eps2[0], m.eps2[1] = complex(eps2).real, complex(eps2).imag
    for i in range(3):
        m.center[i] = center[i]
    m.amp[0], m.amp[1] = complex(amp).real, complex(amp).imag
    m.width = width
    return m


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P, D, I = C.c_void_p, C.c_double, C.c_int
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        L.or_geom_create.restype = P
        L.or_geom_create.argtypes = [I, C.POINTER(C.c_char_p), C.c_void_p, C.POINTER(OMat)]
        L.or_last_error.restype = C.c_char_p
        L.or_geom_set_nang.argtypes = [P, I]
        for f in ("or_geom_nbf", "or_geom_nobj"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = I
        L.or_geom_ntets.argtypes = [P, I]
        L.or_geom_ntets.restype = I
        L.or_geom_nverts.argtypes = [P, I]
        L.or_geom_nverts.restype = I
        L.or_geom_faces.argtypes = [P, I, ip]
        L.or_geom_destroy.argtypes = [P]
        L.or_sing_static.argtypes = [I, dp, dp, dp, dp, I, dp]
        L.or_sing_static_adaptive.argtypes = [I, dp, dp, dp, dp, I, D, I, dp]
        L.or_sing_static_adaptive.restype = C.c_long
        L.or_sing_static_refined.argtypes = [I, dp, dp, dp, dp, I, I, D, D, dp, C.POINTER(I)]
        L.or_sing_static_refined.restype = C.c_long
        L.or_sing_moments.argtypes = [I, dp, dp, I, dp]
        L.or_sing_moments_refined.argtypes = [I, dp, dp, I, I, D, D, dp, C.POINTER(I)]
        L.or_sing_moments_refined.restype = C.c_long
        lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
        L.or_sing_moments_refined_batch.argtypes = [I, ip, dp, dp, I, I, D, D, dp, ip, lp, ip, ip]
        L.or_geom_set_singular_refine.argtypes = [P, I, I, D, D]
        L.or_geom_singular_status.argtypes = [P]
        L.or_geom_singular_status.restype = I
        L.or_fibbi.argtypes = [P, I, I, dp]
        L.or_gme.argtypes = [P, I, I, D, D, dp]
        L.or_overlaps.argtypes = [P, I, D, ip, dp]
        L.or_overlaps.restype = I
        L.or_overlap_closed_form.argtypes = [P, I, ip, dp]
        L.or_overlap_closed_form.restype = I
        L.or_assemble.argtypes = [P, D, D, dp]
        L.or_assemble_rows.argtypes = [P, D, D, dp, I, I]
        L.or_rhs_planewave.argtypes = [P, D, D, dp, dp, dp]
        L.or_pft_emt.argtypes = [P, D, D, dp, dp, dp, dp]
        L.or_pft_emt8.argtypes = [P, D, D, dp, dp, dp, dp]
        L.or_assemble_g.argtypes = [P, D, D, dp]
        L.or_geom_bf_offset.argtypes = [P, I]
        L.or_geom_bf_offset.restype = I
        L.or_neq_overlaps.argtypes = [P, C.c_int, D, C.c_void_p, dp, dp]
        L.or_neq_overlaps.restype = C.c_int
        L.or_pft_emt8_dr.argtypes = [P, D, D, dp, dp]
        L.or_get_fields.argtypes = [P, D, D, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, dp, dp]
        L.or_pft_opft.argtypes = [P, D, D, dp, dp]
        L.or_num_threads.restype = I
        L.or_cache_build.argtypes = [P]
        L.or_cache_build_rows.argtypes = [P, C.c_void_p, C.c_int]
        L.or_cache_size.argtypes = [P]
        L.or_cache_size.restype = I
        L.or_assemble_row_list.argtypes = [P, D, D, ip, I, dp]
        _LIB = L
    return _LIB


class Geometry:
    """Oracle geometry: a list of (mesh file, displacement, material) objects."""

    def __init__(self, meshfiles, materials, displacements=None, nang=8, refine=False):
        L = lib()
        if isinstance(meshfiles, str):
            meshfiles = [meshfiles]
        if isinstance(materials, OMat):
            materials = [materials]
        n = len(meshfiles)
        arr = (C.c_char_p * n)(*[m.encode() for m in meshfiles])
        mats = (OMat * n)(*materials)
        self._disp = None
        dptr = None
        if displacements is not None:
            self._disp = np.ascontiguousarray(displacements, dtype=np.float64).reshape(n, 3)
            dptr = self._disp.ctypes.data
        self.h = L.or_geom_create(n, arr, dptr, mats)
        if not self.h:
            raise RuntimeError(L.or_last_error().decode())
        L.or_geom_set_nang(self.h, nang)
        if refine:
            L.or_geom_set_singular_refine(self.h, 1, REFINE_NG, REFINE_FLAG, REFINE_TOL)
        self.N = L.or_geom_nbf(self.h)
        self.nobj = L.or_geom_nobj(self.h)
        self.off = [L.or_geom_bf_offset(self.h, i) for i in range(self.nobj + 1)]

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_geom_destroy(self.h)
            self.h = None

    def faces(self, no=0):
        L = lib()
        # interior faces of object no
        cnt = self.off[no + 1] - self.off[no]
        out = np.zeros((cnt, 9), dtype=np.int32)
        L.or_geom_faces(self.h, no, out)
        return out

    def assemble(self, omega, rows=None):
        N = self.N
        M = np.zeros((N, N), dtype=np.complex128, order="F")
        buf = M.view(np.float64).reshape(-1) if False else None
        flat = np.zeros(2 * N * N, dtype=np.float64)
        if rows is None:
            lib().or_assemble(self.h, omega.real, omega.imag, flat)
        else:
            lib().or_assemble_rows(self.h, omega.real, omega.imag, flat, rows[0], rows[1])
        return flat.view(np.complex128).reshape(N, N, order="F")

    def cache_build(self, rows=None):
        """Warm near-field cache (all rows, or only the listed rows)."""
        if rows is None:
            lib().or_cache_build(self.h)
        else:
            r = np.ascontiguousarray(rows, dtype=np.int32)
            lib().or_cache_build_rows(self.h, r.ctypes.data_as(C.c_void_p), len(r))
        return lib().or_cache_size(self.h)

    def assemble_rows(self, omega, rows):
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        out = np.zeros(2 * len(rows) * self.N)
        lib().or_assemble_row_list(self.h, omega.real, omega.imag, rows, len(rows), out)
        return out.view(np.complex128).reshape(len(rows), self.N)

    def gme(self, a, b, omega):
        out = np.zeros(2)
        lib().or_gme(self.h, a, b, omega.real, omega.imag, out)
        return complex(out[0], out[1])

    def fibbi(self, a, b):
        out = np.zeros(6)
        lib().or_fibbi(self.h, a, b, out)
        return out

    def overlaps(self, a, omega):
        idx = np.zeros(7, dtype=np.int32)
        v = np.zeros(14)
        n = lib().or_overlaps(self.h, a, omega, idx, v)
        return idx[:n], v[: 2 * n].view(np.complex128)

    def overlap_closed_form(self, a):
        idx = np.zeros(7, dtype=np.int32)
        v = np.zeros(7)
        n = lib().or_overlap_closed_form(self.h, a, idx, v)
        return idx[:n], v[:n]

    def rhs_planewave(self, omega, E0, nhat):
        E = np.asarray(E0, dtype=np.complex128).view(np.float64).copy()
        nh = np.asarray(nhat, dtype=np.float64).copy()
        out = np.zeros(2 * self.N)
        lib().or_rhs_planewave(self.h, omega.real, omega.imag, E, nh, out)
        return out.view(np.complex128)

    def pft_emt(self, omega, J, E0, nhat):
        Jd = np.ascontiguousarray(J, dtype=np.complex128).view(np.float64)
        E = np.asarray(E0, dtype=np.complex128).view(np.float64).copy()
        nh = np.asarray(nhat, dtype=np.float64).copy()
        out = np.zeros(2 * self.nobj)
        lib().or_pft_emt(self.h, omega.real, omega.imag, Jd, E, nh, out)
        return out.reshape(self.nobj, 2)

    def pft_emt8(self, omega, J, E0, nhat):
        """Full EMT PFT: rows = objects, columns PAbs, PScat, Fx, Fy, Fz, Tx, Ty, Tz."""
        Jd = np.ascontiguousarray(J, dtype=np.complex128).view(np.float64)
        E = np.asarray(E0, dtype=np.complex128).view(np.float64).copy()
        nh = np.asarray(nhat, dtype=np.float64).copy()
        out = np.zeros(8 * self.nobj)
        lib().or_pft_emt8(self.h, omega.real, omega.imag, Jd, E, nh, out)
        return out.reshape(self.nobj, 8)

    def assemble_g(self, omega):
        """G block of the whole geometry (AssembleGBlock for every object pair)."""
        flat = np.zeros(2 * self.N * self.N)
        lib().or_assemble_g(self.h, omega.real, omega.imag, flat)
        return flat.view(np.complex128).reshape(self.N, self.N, order="F")

    def neq_overlaps(self, a, omega):
        idx = np.zeros(7, dtype=np.int32)
        V, R = np.zeros(14), np.zeros(7)
        n = lib().or_neq_overlaps(self.h, a, float(np.real(omega)), idx.ctypes.data_as(C.c_void_p), V, R)
        return idx[:n], V[: 2 * n].view(np.complex128), R[:n]

    def neq_blocks(self, omega):
        """Dense S (Gram, GetOverlapElements), V (all objects) and the Rytov
        block of each object (AssembleOverlapBlocks with SetEntry per row)."""
        N = self.N
        S = np.zeros((N, N))
        V = np.zeros((N, N), complex)
        R = [np.zeros((N, N)) for _ in range(self.nobj)]
        for no in range(self.nobj):
            for a in range(self.off[no], self.off[no + 1]):
                idx, vals = self.overlap_closed_form(a)
                S[a, idx] = vals
                idx, v, r = self.neq_overlaps(a, omega)
                V[a, idx] = v
                R[no][a, idx] = r
        return S, V, R

    def dressed_rytov(self, omega, src, blocks=None, Gm=None):
        """ComputeDressedRytovMatrix (GetFlux.cc:155-272), its steps in order:
        W = (1 + S^-1 V S^-1 G)^-1 by LU, then W \\ (W \\ S^-1 R_src S^-1)^H."""
        import scipy.linalg as sl
        S, V, R = blocks if blocks is not None else self.neq_blocks(omega)
        Gm = self.assemble_g(omega) if Gm is None else Gm
        Sinv = np.linalg.inv(S)                     # SInverse->LUFactorize(); LUInvert()
        M2 = Sinv @ Gm                              # (b)
        M1 = V @ M2                                 # (d)
        M3 = Sinv @ M1                              # (e)
        M3 += np.eye(self.N)                        # (f)
        lu = sl.lu_factor(M3)                       # (g)
        M1 = np.asarray(R[src], complex)            # (h)
        M2 = Sinv @ M1                              # (i)
        M1 = M2 @ Sinv                              # (j)
        M2 = sl.lu_solve(lu, M1)                    # (k)
        M1 = M2.conj().T                            # (l)
        return sl.lu_solve(lu, M1)                  # (m)

    def pft_emt8_dr(self, omega, DR):
        D = np.asfortranarray(DR, dtype=np.complex128)
        out = np.zeros(8 * self.nobj)
        lib().or_pft_emt8_dr(self.h, omega.real, omega.imag, D.reshape(-1, order="F").view(np.float64), out)
        return out.reshape(self.nobj, 8)

    def neq_flux(self, omega):
        """GetFlux (GetFlux.cc:291-436) for one geometry and no transforms:
        flux[src, dst, q], q = PAbs, PScat, Fx, Fy, Fz, Tx, Ty, Tz (EMT)."""
        blocks, Gm = self.neq_blocks(omega), self.assemble_g(omega)
        return np.stack([self.pft_emt8_dr(omega, self.dressed_rytov(omega, s, blocks, Gm))
                         for s in range(self.nobj)])

    def get_fields(self, omega, J, X, E0=None, nhat=None):
        """(P, 6) complex: E and H at the points X (P x 3); J and/or the plane wave may be None."""
        X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
        out = np.zeros(12 * len(X))
        Jd = None if J is None else np.ascontiguousarray(J, dtype=np.complex128).view(np.float64)
        E = None if E0 is None else np.asarray(E0, dtype=np.complex128).view(np.float64).copy()
        nh = None if nhat is None else np.asarray(nhat, dtype=np.float64).copy()
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        lib().or_get_fields(self.h, omega.real, omega.imag, ptr(Jd), ptr(E), ptr(nh), len(X), X, out)
        return out.view(np.complex128).reshape(len(X), 6)

    def pft_opft(self, omega, J):
        Jd = np.ascontiguousarray(J, dtype=np.complex128).view(np.float64)
        out = np.zeros(self.nobj)
        lib().or_pft_opft(self.h, omega.real, omega.imag, Jd, out)
        return out


def sing_static(c, VA, VB, Q, QP, nang=8):
    out = np.zeros(6)
    lib().or_sing_static(c, np.ascontiguousarray(VA, dtype=np.float64).reshape(-1),
                         np.ascontiguousarray(VB, dtype=np.float64).reshape(-1),
                         np.ascontiguousarray(Q, dtype=np.float64),
                         np.ascontiguousarray(QP, dtype=np.float64), nang, out)
    return out


def sing_static_adaptive(c, VA, VB, Q, QP, ng=6, tol=1e-10, maxdepth=10):
    """The six values of sing_static by adaptive bisection of the angular
    cubes (an accuracy reference for the fixed rule); returns (values,
    angular points evaluated)."""
    out = np.zeros(6)
    n = lib().or_sing_static_adaptive(c, np.ascontiguousarray(VA, dtype=np.float64).reshape(-1),
                                      np.ascontiguousarray(VB, dtype=np.float64).reshape(-1),
                                      np.ascontiguousarray(Q, dtype=np.float64),
                                      np.ascontiguousarray(QP, dtype=np.float64), ng, tol, maxdepth, out)
    return out, n


def sing_static_refined(c, VA, VB, Q, QP, n=10, ng=6, flag_tol=1e-7, tol=1e-10):
    """Orders n and n + 2, refined where they disagree (the level-by-level
    scheme); returns (values, angular points of the refinement, status)."""
    out = np.zeros(6)
    st = C.c_int()
    ne = lib().or_sing_static_refined(c, np.ascontiguousarray(VA, dtype=np.float64).reshape(-1),
                                      np.ascontiguousarray(VB, dtype=np.float64).reshape(-1),
                                      np.ascontiguousarray(Q, dtype=np.float64),
                                      np.ascontiguousarray(QP, dtype=np.float64), n, ng, flag_tol, tol, out,
                                      C.byref(st))
    return out, ne, st.value


def sing_moments(c, VA, VB, n=10, refined=False, ng=6, flag_tol=1e-7, tol=1e-9):
    """The 24 moments k_tp_singular keeps for a tetrahedron pair (per kernel
    1/4pi r, 1/4pi, r/8pi: int K, int K (x-o), int K (y-o), int K (x-o).(y-o),
    barycentric measure, o = first common vertex), at order n or refined;
    returns (moments, angular points of the refinement, status)."""
    out = np.zeros(24)
    A = np.ascontiguousarray(VA, dtype=np.float64).reshape(-1)
    B = np.ascontiguousarray(VB, dtype=np.float64).reshape(-1)
    if not refined:
        lib().or_sing_moments(c, A, B, n, out)
        return out, 0, 0
    st = C.c_int()
    ne = lib().or_sing_moments_refined(c, A, B, n, ng, flag_tol, tol, out, C.byref(st))
    return out, ne, st.value


def sing_moments_refined_batch(cs, VA, VB, n=REFINE_ORDER, ng=REFINE_NG, flag_tol=REFINE_FLAG, tol=REFINE_TOL):
    """Refined moments of many pairs (cs: common-vertex counts, VA/VB: (P, 4, 3)
    common-first vertices), OpenMP over pairs; returns (moments (P, 24),
    status, angular points of the refinement, peak open boxes, levels)."""
    cs = np.ascontiguousarray(cs, dtype=np.int32)
    P = len(cs)
    A = np.ascontiguousarray(VA, dtype=np.float64).reshape(-1)
    B = np.ascontiguousarray(VB, dtype=np.float64).reshape(-1)
    out = np.zeros(24 * P)
    st, pk, lv = (np.zeros(P, dtype=np.int32) for _ in range(3))
    ev = np.zeros(P, dtype=np.int64)
    lib().or_sing_moments_refined_batch(P, cs, A, B, n, ng, flag_tol, tol, out, st, ev, pk, lv)
    return out.reshape(P, 24), st, ev, pk, lv


def moments_to_values(M, VA, VB, Q, QP):
    """The six sing_static values from the 24 moments."""
    VA, VB = np.asarray(VA, float), np.asarray(VB, float)
    vol = lambda V: abs(np.linalg.det(np.array([V[1] - V[0], V[2] - V[0], V[3] - V[0]]))) / 6
    f = 36 * vol(VA) * vol(VB)
    o = VA[0]
    q, qp = np.asarray(Q) - o, np.asarray(QP) - o
    out = np.zeros(6)
    for pk, g in enumerate((0.25 / np.pi, 0.25 / np.pi, 0.125 / np.pi)):
        m = M[8 * pk:8 * pk + 8] / g
        out[2 * pk] = f * (m[7] - qp @ m[1:4] - q @ m[4:7] + (q @ qp) * m[0])
        out[2 * pk + 1] = f * m[0]
    return out
