"""Python binding of libbuffem_b200.so (the C-ABI of include/buffem_b200.h).

Mirrors the names of libbuff's C++ API so scripts read like the reference's
drivers (buff-scatter.cc:236-347, unit-test-LFField.cc:50-71):

    G = SWGGeometry("E10Sphere.buffgeo")          # SWGGeometry(const char*)
    M = G.AllocateVIEMatrix()                     # VIEMatrix.cc:465-471
    G.AssembleVIEMatrix(omega, M)                 # VIEMatrix.cc:431-460
    M.LUFactorize()                               # HMatrix::LUFactorize
    J = G.AssembleRHSVector(omega, PlaneWave(E0, nhat))   # RHSVector.cc:85-124
    M.LUSolve(J)                                  # HMatrix::LUSolve
    PFT = G.GetPFTMatrix(J, omega, PlaneWave(...))        # GetPFT.cc:133-189

All compute runs in the CUDA library; there is no CPU fallback.  Loading the
library succeeds without a GPU (for symbol checks); compute calls then raise
BuffError with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbuffem_b200.so")
_LIB = None

BG_C128, BG_C64 = 0, 1
BG_BATCH_MAXOBJ, BG_BATCH_NO_GRAPHS = 4, 1
BG_MAT_CONST_ISO, BG_MAT_CONST_TENSOR, BG_MAT_JANUS_Z, BG_MAT_GAUSSIAN = 0, 1, 2, 3
BG_PFT_EMT, BG_PFT_OVERLAP = 0, 1
BG_OK, BG_ERR_ARG, BG_ERR_IO, BG_ERR_TOPOLOGY, BG_ERR_CUDA, BG_ERR_NOMEM, BG_ERR_STATE, BG_ERR_NUMERIC = 0, -1, -2, -3, -4, -5, -6, -7
PFT_PABS, PFT_PSCAT = 0, 1


class BuffError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class bg_material(C.Structure):
    _fields_ = [("kind", C.c_int), ("eps", C.c_double * 18), ("eps2", C.c_double * 2),
                ("center", C.c_double * 3), ("amp", C.c_double * 2), ("width", C.c_double)]


def Material(kind=BG_MAT_CONST_ISO, eps=1.0, tensor=None, eps2=None, center=(0, 0, 0), amp=0.0, width=1.0):
    """Permittivity functor (closed replacement for SVTensor / MatProp)."""
    m = bg_material()
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


EXPORTS = [
    "bg_last_error", "bg_geometry_create", "bg_geometry_create_objects", "bg_geometry_destroy",
    "bg_geometry_num_bfs", "bg_geometry_num_objects", "bg_geometry_bf_offset", "bg_geometry_faces",
    "bg_geometry_vertices", "bg_geometry_object_index", "bg_geometry_object_label", "bg_geometry_material_eps",
    "bg_trans_file_count", "bg_trans_file_tag", "bg_geometry_create_transformed", "bg_geometry_material_tensor",
    "bg_geometry_precompute", "bg_geometry_set_singular_order", "bg_geometry_near_data",
    "bg_geometry_set_singular_refine", "bg_geometry_singular_stats", "bg_geometry_singular_moments",
    "bg_matrix_create", "bg_matrix_destroy", "bg_assemble", "bg_assemble_with_copy", "bg_matrix_download",
    "bg_matrix_upload",
    "bg_matrix_get_rows",
    "bg_matrix_device_ptr", "bg_lu_factor", "bg_lu_pivots", "bg_lu_solve", "bg_lu_solve_device",
    "bg_rhs_planewave", "bg_rhs_planewave_device", "bg_pft", "bg_kernel_launch_count",
    "bg_synchronize", "bg_stream", "bg_profile_begin", "bg_profile_read", "bg_profile_end",
    "bg_zgemm_sub_device", "bg_cgemm_sub_device", "bg_matrix_convert", "bg_lu_solve_refined", "bg_lu_solve_refined_device",
    "bg_lu_solve_device_noalloc", "bg_precond_create_jacobi", "bg_precond_destroy", "bg_precond_nnz",
    "bg_gmres_solve", "bg_gmres_solve_device", "bg_gnn_create", "bg_gnn_destroy", "bg_gnn_num_params",
    "bg_gnn_get_params", "bg_gnn_set_params", "bg_gnn_get_grads", "bg_gnn_train_step",
    "bg_precond_create_learned", "bg_precond_download", "bg_gmres_solve_mixed", "bg_gmres_solve_mixed_device",
    "bg_precond_bound", "bg_gmres_solve_lu_fallback", "bg_gmres_solve_lu_fallback_device", "bg_batch_sweep",
    "bg_pft_full", "bg_gmres_last_info", "bg_fibbi_store", "bg_fibbi_load", "bg_get_fields", "bg_get_fields_device",
    "bg_neq_create", "bg_neq_destroy", "bg_neq_flux", "bg_neq_dressed_rytov", "bg_pft_dr_device",
]


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise BuffError(-4, f"{LIB_PATH} is not built (run `make -C buff-em_b200`)")
        L = C.CDLL(LIB_PATH)
        P, I, D, VP = C.c_void_p, C.c_int, C.c_double, C.c_void_p
        L.bg_last_error.restype = C.c_char_p
        L.bg_geometry_create.argtypes = [C.c_char_p, C.POINTER(P)]
        L.bg_geometry_create_objects.argtypes = [I, C.POINTER(C.c_char_p), VP, C.POINTER(bg_material),
                                                 C.POINTER(P)]
        L.bg_geometry_destroy.argtypes = [P]
        L.bg_geometry_destroy.restype = None
        for f in ("bg_geometry_num_bfs", "bg_geometry_num_objects", "bg_geometry_precompute"):
            getattr(L, f).argtypes = [P]
        L.bg_geometry_bf_offset.argtypes = [P, I]
        L.bg_geometry_faces.argtypes = [P, I, VP]
        L.bg_geometry_vertices.argtypes = [P, I, VP, VP]
        L.bg_geometry_object_index.argtypes = [P, C.c_char_p]
        L.bg_geometry_object_label.argtypes = [P, I, C.c_char_p, I]
        L.bg_geometry_material_eps.argtypes = [P, I, D, D, VP]
        L.bg_geometry_material_tensor.argtypes = [P, I, D, D, VP, VP]
        L.bg_trans_file_count.argtypes = [C.c_char_p]
        L.bg_trans_file_tag.argtypes = [C.c_char_p, I, C.c_char_p, I]
        L.bg_geometry_create_transformed.argtypes = [C.c_char_p, C.c_char_p, I, C.POINTER(P)]
        L.bg_geometry_set_singular_order.argtypes = [P, I]
        L.bg_geometry_set_singular_refine.argtypes = [P, I, D, D]
        L.bg_geometry_singular_stats.argtypes = [P, VP]
        L.bg_geometry_singular_moments.argtypes = [P, C.POINTER(I), VP, VP, VP]
        L.bg_geometry_near_data.argtypes = [P, C.POINTER(I), VP, VP]
        L.bg_matrix_create.argtypes = [P, I, C.POINTER(P)]
        L.bg_matrix_destroy.argtypes = [P]
        L.bg_matrix_destroy.restype = None
        L.bg_assemble.argtypes = [P, D, D, P]
        L.bg_assemble_with_copy.argtypes = [P, D, D, P, P]
        L.bg_matrix_download.argtypes = [P, VP]
        L.bg_matrix_upload.argtypes = [P, VP]
        L.bg_matrix_get_rows.argtypes = [P, I, VP, VP]
        L.bg_matrix_device_ptr.argtypes = [P, C.POINTER(VP), C.POINTER(I)]
        L.bg_lu_factor.argtypes = [P]
        L.bg_lu_pivots.argtypes = [P, VP]
        L.bg_lu_solve.argtypes = [P, VP, I]
        L.bg_lu_solve_device.argtypes = [P, VP, I, I]
        L.bg_lu_solve_device_noalloc.argtypes = [P, VP, I, I]
        L.bg_precond_create_jacobi.argtypes = [P, C.POINTER(P)]
        L.bg_precond_destroy.argtypes = [P]
        L.bg_precond_destroy.restype = None
        L.bg_precond_nnz.argtypes = [P]
        L.bg_gmres_solve.argtypes = [P, P, VP, I, D, I, I, VP]
        L.bg_gmres_solve_device.argtypes = [P, P, VP, I, I, D, I, I, VP]
        L.bg_gmres_solve_mixed.argtypes = [P, P, P, VP, I, D, I, I, D, VP]
        L.bg_gmres_solve_lu_fallback.argtypes = [P, P, P, VP, I, D, I, I, D, VP]
        L.bg_batch_sweep.argtypes = [VP, I, VP, I, VP, VP, I, I, VP, VP]
        L.bg_gmres_solve_lu_fallback_device.argtypes = [P, P, P, VP, I, I, D, I, I, D, VP]
        L.bg_gmres_solve_mixed_device.argtypes = [P, P, P, VP, I, I, D, I, I, D, VP]
        L.bg_gnn_create.argtypes = [C.c_ulonglong, C.POINTER(P)]
        L.bg_gnn_destroy.argtypes = [P]
        L.bg_gnn_destroy.restype = None
        L.bg_gnn_get_params.argtypes = [P, VP]
        L.bg_gnn_set_params.argtypes = [P, VP]
        L.bg_gnn_get_grads.argtypes = [P, VP]
        L.bg_gnn_train_step.argtypes = [P, P, P, D, VP, I, I, VP, VP, D, D, VP]
        L.bg_precond_create_learned.argtypes = [P, P, D, P, C.POINTER(P)]
        L.bg_precond_download.argtypes = [P, VP, VP, VP]
        L.bg_precond_bound.argtypes = [P, VP, VP]
        L.bg_rhs_planewave.argtypes = [P, D, D, VP, VP, VP]
        L.bg_rhs_planewave_device.argtypes = [P, D, D, VP, VP, VP]
        L.bg_pft.argtypes = [P, D, D, VP, VP, VP, I, VP]
        L.bg_pft_full.argtypes = [P, D, D, VP, VP, VP, VP]
        L.bg_gmres_last_info.argtypes = [VP]
        L.bg_get_fields.argtypes = [P, D, D, VP, VP, VP, C.c_int, VP, VP]
        L.bg_neq_create.argtypes = [P, C.POINTER(P)]
        L.bg_neq_destroy.argtypes = [P]
        L.bg_neq_destroy.restype = None
        L.bg_neq_flux.argtypes = [P, D, D, VP]
        L.bg_neq_dressed_rytov.argtypes = [P, D, D, I, VP]
        L.bg_pft_dr_device.argtypes = [P, D, D, VP, I, VP]
        L.bg_get_fields_device.argtypes = [P, D, D, VP, VP, VP, C.c_int, VP, VP]
        L.bg_fibbi_store.argtypes = [P, I, C.c_char_p, C.POINTER(I)]
        L.bg_fibbi_load.argtypes = [P, I, C.c_char_p, C.POINTER(I)]
        L.bg_kernel_launch_count.restype = C.c_longlong
        L.bg_stream.restype = VP
        L.bg_profile_read.argtypes = [I, VP, VP, VP]
        L.bg_zgemm_sub_device.argtypes = [I, I, I, VP, I, VP, I, VP, I]
        L.bg_cgemm_sub_device.argtypes = [I, I, I, VP, I, VP, I, VP, I]
        L.bg_matrix_convert.argtypes = [P, P]
        L.bg_lu_solve_refined.argtypes = [P, P, VP, I, D, I, VP]
        L.bg_lu_solve_refined_device.argtypes = [P, P, VP, I, I, D, I, VP]
        _LIB = L
    return _LIB


def _check(st):
    if st < 0:
        raise BuffError(st, lib().bg_last_error().decode(errors="replace"))
    return st


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class PlaneWave:
    """Plane wave E = E0 exp(i k nhat.x) (SCUFF-EM PlaneWave(E0, nHat))."""

    def __init__(self, E0, nHat):
        self.E0 = np.ascontiguousarray(E0, dtype=np.complex128).reshape(3)
        self.nHat = np.ascontiguousarray(nHat, dtype=np.float64).reshape(3)


class HMatrix:
    """Device-resident VIE matrix (replaces libhmat's HMatrix for this path)."""

    def __init__(self, geom, precision=BG_C128):
        self.G = geom
        h = C.c_void_p()
        _check(lib().bg_matrix_create(geom.h, precision, C.byref(h)))
        self.h = h
        self.NR = self.NC = geom.TotalBFs
        self.precision = precision

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:   # lib is None at interpreter exit
            lib().bg_matrix_destroy(self.h)
            self.h = None

    def LUFactorize(self):
        info = _check(lib().bg_lu_factor(self.h))
        if info > 0:
            raise BuffError(info, f"singular matrix: zero pivot at {info}")
        return self

    def LUSolve(self, B):
        """Solve in place; B is an N-vector or N x nrhs complex array (Fortran order)."""
        arr = B if isinstance(B, np.ndarray) else np.asarray(B)
        if arr.dtype != np.complex128:
            raise TypeError("LUSolve needs complex128")
        nrhs = 1 if arr.ndim == 1 else arr.shape[1]
        buf = np.asfortranarray(arr)
        _check(lib().bg_lu_solve(self.h, _ptr(buf), nrhs))
        if buf is not arr:
            arr[...] = buf
        return arr

    def pivots(self):
        p = np.zeros(self.NR, dtype=np.int32)
        _check(lib().bg_lu_pivots(self.h, _ptr(p)))
        return p

    def download(self):
        dt = np.complex128 if self.precision == BG_C128 else np.complex64
        out = np.zeros((self.NR, self.NC), dtype=dt, order="F")
        _check(lib().bg_matrix_download(self.h, _ptr(out)))
        return out

    def rows(self, rows):
        """Rows of the matrix, (len(rows), N), without downloading the rest."""
        dt = np.complex128 if self.precision == BG_C128 else np.complex64
        r = np.ascontiguousarray(rows, dtype=np.int32)
        out = np.zeros((len(r), self.NC), dtype=dt)
        _check(lib().bg_matrix_get_rows(self.h, len(r), _ptr(r), _ptr(out)))
        return out

    def upload(self, A):
        dt = np.complex128 if self.precision == BG_C128 else np.complex64
        a = np.asfortranarray(A, dtype=dt)
        _check(lib().bg_matrix_upload(self.h, _ptr(a)))

    def convert_from(self, src):
        """Fill this (complex64) matrix from a complex128 one."""
        _check(lib().bg_matrix_convert(src.h, self.h))
        return self

    def LUSolveRefined(self, F, B, tol=1e-12, maxit=30):
        """Solve with complex64 factors F of this complex128 matrix plus FP64
        iterative refinement; returns (X, stats=(sweeps, final, first residual))."""
        arr = np.asfortranarray(B, dtype=np.complex128)
        nrhs = 1 if arr.ndim == 1 else arr.shape[1]
        st = np.zeros(3)
        _check(lib().bg_lu_solve_refined(self.h, F.h, _ptr(arr), nrhs, float(tol), int(maxit), _ptr(st)))
        return arr, st

    def device_ptr(self):
        p = C.c_void_p()
        ld = C.c_int()
        _check(lib().bg_matrix_device_ptr(self.h, C.byref(p), C.byref(ld)))
        return p.value, ld.value


def ReadTransFile(path):
    """Tags of the transformations of a .trans file, in order (pass the index
    as SWGGeometry(..., TransFile=path, Transformation=k))."""
    n = _check(lib().bg_trans_file_count(path.encode()))
    tags = []
    for k in range(n):
        m = _check(lib().bg_trans_file_tag(path.encode(), k, None, 0))
        buf = C.create_string_buffer(m + 1)
        _check(lib().bg_trans_file_tag(path.encode(), k, buf, m + 1))
        tags.append(buf.value.decode())
    return tags


class SWGGeometry:
    """Replaces buff::SWGGeometry (libbuff.h:200-272) for the VIE hot path."""

    def __init__(self, GeoFileName=None, meshfiles=None, materials=None, displacements=None,
                 singular_order=None, TransFile=None, Transformation=0, singular_refine=None,
                 singular_tol=(1e-8, 1e-9)):
        h = C.c_void_p()
        if GeoFileName is not None and TransFile is not None:
            _check(lib().bg_geometry_create_transformed(GeoFileName.encode(), TransFile.encode(), int(Transformation),
                                                        C.byref(h)))
        elif GeoFileName is not None:
            _check(lib().bg_geometry_create(GeoFileName.encode(), C.byref(h)))
        else:
            if isinstance(meshfiles, str):
                meshfiles = [meshfiles]
            if isinstance(materials, bg_material):
                materials = [materials]
            n = len(meshfiles)
            names = (C.c_char_p * n)(*[m.encode() for m in meshfiles])
            mats = (bg_material * n)(*materials)
            self._disp = None
            dptr = None
            if displacements is not None:
                self._disp = np.ascontiguousarray(displacements, dtype=np.float64).reshape(n, 3)
                dptr = _ptr(self._disp)
            _check(lib().bg_geometry_create_objects(n, names, dptr, mats, C.byref(h)))
        self.h = h
        self.TotalBFs = lib().bg_geometry_num_bfs(h)
        self.NumObjects = lib().bg_geometry_num_objects(h)
        self.BFIndexOffset = [lib().bg_geometry_bf_offset(h, i) for i in range(self.NumObjects + 1)]
        # the singular rule (TaylorDuffyTolerance's role): refined by default;
        # singular_refine=False keeps the fixed rule of singular_order alone
        if singular_refine is not None:
            _check(lib().bg_geometry_set_singular_refine(h, 1 if singular_refine else 0, float(singular_tol[0]),
                                                         float(singular_tol[1])))
        if singular_order is not None:
            _check(lib().bg_geometry_set_singular_order(h, int(singular_order)))

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:   # lib is None at interpreter exit
            lib().bg_geometry_destroy(self.h)
            self.h = None

    def singular_stats(self):
        """dict of the singular-pair statistics (bg_geometry_singular_stats)."""
        out = np.zeros(6, dtype=np.int64)
        _check(lib().bg_geometry_singular_stats(self.h, _ptr(out)))
        keys = ("pairs", "refined", "fixed_points", "refine_points", "status", "refine_on")
        return {k: int(v) for k, v in zip(keys, out)}

    def singular_moments(self):
        """(pairs (P, 4): row tet, column tet, common vertices, flags;
        verts (P, 8): vertex indices, common first; moments (P, 24))."""
        n = C.c_int()
        _check(lib().bg_geometry_singular_moments(self.h, C.byref(n), None, None, None))
        P = n.value
        pairs = np.zeros((P, 4), dtype=np.int32)
        verts = np.zeros((P, 8), dtype=np.int32)
        mom = np.zeros((P, 24))
        if P:
            _check(lib().bg_geometry_singular_moments(self.h, C.byref(n), _ptr(pairs), _ptr(verts), _ptr(mom)))
        return pairs, verts, mom

    def faces(self, obj=0):
        n = self.BFIndexOffset[obj + 1] - self.BFIndexOffset[obj]
        out = np.zeros((n, 9), dtype=np.int32)
        _check(lib().bg_geometry_faces(self.h, obj, _ptr(out)))
        return out

    def GetObjectByLabel(self, label):
        """Index of the object labelled `label` (ignoring case), or -1
        (SWGGeometry::GetObjectByLabel, SWGGeometry.cc:405-419)."""
        st = lib().bg_geometry_object_index(self.h, label.encode())
        return st if st >= 0 else -1

    def material_eps(self, obj, omega):
        """eps of object obj at Omega (units of 3e14 rad/s): a MATERIAL
        section's Eps(w) at w = Omega x 3e14 rad/s, or the object's constant."""
        omega = complex(omega)
        e = np.zeros(2)
        _check(lib().bg_geometry_material_eps(self.h, obj, omega.real, omega.imag, _ptr(e)))
        return complex(e[0], e[1])

    def material_tensor(self, obj, omega, x=(0.0, 0.0, 0.0)):
        """3x3 complex permittivity tensor of object obj at Omega and point x
        (SVTensor::Evaluate)."""
        omega = complex(omega)
        X = np.ascontiguousarray(x, dtype=np.float64)
        Q = np.zeros(18)
        _check(lib().bg_geometry_material_tensor(self.h, obj, omega.real, omega.imag, _ptr(X), _ptr(Q)))
        return (Q[0::2] + 1j * Q[1::2]).reshape(3, 3)

    def label(self, obj=0):
        n = _check(lib().bg_geometry_object_label(self.h, obj, None, 0))
        buf = C.create_string_buffer(n + 1)
        _check(lib().bg_geometry_object_label(self.h, obj, buf, n + 1))
        return buf.value.decode()

    def vertices(self, obj=0):
        """(nv, 3) vertex coordinates of object obj after its one-time
        transformation, and its origin (the torque centre)."""
        nv = _check(lib().bg_geometry_vertices(self.h, obj, None, None))
        xyz = np.zeros((nv, 3))
        origin = np.zeros(3)
        _check(lib().bg_geometry_vertices(self.h, obj, _ptr(xyz), _ptr(origin)))
        return xyz, origin

    def precompute(self):
        _check(lib().bg_geometry_precompute(self.h))

    def near_data(self):
        cnt = C.c_int()
        _check(lib().bg_geometry_near_data(self.h, C.byref(cnt), None, None))
        pairs = np.zeros((cnt.value, 2), dtype=np.int32)
        data = np.zeros((cnt.value, 6), dtype=np.float64)
        _check(lib().bg_geometry_near_data(self.h, C.byref(cnt), _ptr(pairs), _ptr(data)))
        return pairs, data

    def StoreFIBBICache(self, path, obj=0):
        """Write object obj's near-field table as a reference FIBBI cache file; returns the record count."""
        n = C.c_int()
        _check(lib().bg_fibbi_store(self.h, int(obj), os.fsencode(path), C.byref(n)))
        return n.value

    def PreloadFIBBICache(self, path, obj=0):
        """Take the near-field integrals of object obj from a reference FIBBI cache file; returns matches."""
        n = C.c_int()
        _check(lib().bg_fibbi_load(self.h, int(obj), os.fsencode(path), C.byref(n)))
        return n.value

    def AllocateVIEMatrix(self, precision=BG_C128):
        return HMatrix(self, precision)

    def AssembleVIEMatrix(self, Omega, M=None):
        if M is None:
            M = self.AllocateVIEMatrix()
        Omega = complex(Omega)
        _check(lib().bg_assemble(self.h, Omega.real, Omega.imag, M.h))
        return M

    def AssembleVIEMatrixWithCopy(self, Omega, M=None, F=None):
        """AssembleVIEMatrix plus its complex64 copy written by the same
        kernels (the matrix the mixed-precision solvers run on); returns
        (M, F)."""
        if M is None:
            M = self.AllocateVIEMatrix()
        if F is None:
            F = self.AllocateVIEMatrix(BG_C64)
        Omega = complex(Omega)
        _check(lib().bg_assemble_with_copy(self.h, Omega.real, Omega.imag, M.h, F.h))
        return M, F

    def AllocateRHSVector(self):
        return np.zeros(self.TotalBFs, dtype=np.complex128)

    def AssembleRHSVector(self, Omega, IF, RHS=None):
        Omega = complex(Omega)
        out = self.AllocateRHSVector() if RHS is None else RHS
        _check(lib().bg_rhs_planewave(self.h, Omega.real, Omega.imag, _ptr(IF.E0), _ptr(IF.nHat), _ptr(out)))
        return out

    def GetFields(self, IF, J, Omega, X):
        """SWGGeometry::GetFields (GetFields.cc:287-382): (P, 6) complex array of
        Ex, Ey, Ez, Hx, Hy, Hz at the points X (P x 3); IF (a PlaneWave) and J
        may each be None, as the reference's IF = 0 and J = 0."""
        Omega = complex(Omega)
        X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
        out = np.zeros((len(X), 6), complex)
        Jc = None if J is None else np.ascontiguousarray(J, dtype=np.complex128)
        if Jc is not None and Jc.shape != (self.TotalBFs,):
            raise ValueError("J must have TotalBFs entries")
        E0 = _ptr(IF.E0) if IF is not None else None
        nh = _ptr(IF.nHat) if IF is not None else None
        _check(lib().bg_get_fields(self.h, Omega.real, Omega.imag, None if Jc is None else _ptr(Jc), E0, nh,
                                   len(X), _ptr(X), _ptr(out)))
        return out

    def GetPFTMatrix(self, J, Omega, IF=None, method=BG_PFT_EMT, full=False):
        """Rows = objects, columns = (PAbs, PScat); with full=True (EMT only)
        all eight columns PAbs, PScat, Fx, Fy, Fz, Tx, Ty, Tz."""
        if full:
            Omega = complex(Omega)
            Jc = np.ascontiguousarray(J, dtype=np.complex128)
            out = np.zeros((self.NumObjects, 8))
            _check(lib().bg_pft_full(self.h, Omega.real, Omega.imag, _ptr(Jc), _ptr(IF.E0), _ptr(IF.nHat),
                                     _ptr(out)))
            return out
        Omega = complex(Omega)
        Jc = np.ascontiguousarray(J, dtype=np.complex128)
        out = np.zeros((self.NumObjects, 2))
        E0 = _ptr(IF.E0) if IF is not None else None
        nh = _ptr(IF.nHat) if IF is not None else None
        _check(lib().bg_pft(self.h, Omega.real, Omega.imag, _ptr(Jc), E0, nh, method, _ptr(out)))
        return out


class NEQ:
    """buff-neq's flux chain for one geometry (GetFlux, GetFlux.cc:291-436)
    at a uniform temperature per object; the geometry as it stands is the
    single transform.  Holds S^-1 and three N x N work matrices on the device."""

    def __init__(self, G):
        h = C.c_void_p()
        _check(lib().bg_neq_create(G.h, C.byref(h)))
        self.h, self.G = h, G

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:   # lib is None at interpreter exit
            lib().bg_neq_destroy(self.h)
            self.h = None

    def GetFlux(self, Omega):
        """flux[s, d, q]: source s, destination d, q = PAbs, PRad, Fx, Fy, Fz,
        Tx, Ty, Tz (EMT, the buff-neq default); multiply by Delta Theta to get
        the spectral density of power or force."""
        Omega = complex(Omega)
        NO = self.G.NumObjects
        out = np.zeros((NO, NO, 8))
        _check(lib().bg_neq_flux(self.h, Omega.real, Omega.imag, _ptr(out)))
        return out

    def DressedRytov(self, Omega, src):
        """DR_src = W S^-1 R_src S^-1 W^H (ComputeDressedRytovMatrix), N x N."""
        Omega = complex(Omega)
        N = self.G.TotalBFs
        out = np.zeros((N, N), complex, order="F")
        _check(lib().bg_neq_dressed_rytov(self.h, Omega.real, Omega.imag, src, _ptr(out)))
        return out


def cgemm_sub_device(M, N, K, A, lda, B, ldb, C, ldc):
    """C -= A B for device complex64 column-major matrices (tcgen05 TF32 GEMM)."""
    _check(lib().bg_cgemm_sub_device(M, N, K, C_void(A), lda, C_void(B), ldb, C_void(C), ldc))


def zgemm_sub_device(M, N, K, A, lda, B, ldb, C, ldc):
    """C -= A @ B on device pointers (complex128, column-major)."""
    _check(lib().bg_zgemm_sub_device(M, N, K, C_void(A), lda, C_void(B), ldb, C_void(C), ldc))


def C_void(p):
    return C.c_void_p(p)


class Preconditioner:
    """Sparse right preconditioner for GMRES (device CSR, complex128)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def jacobi(cls, M):
        h = C.c_void_p()
        _check(lib().bg_precond_create_jacobi(M.h, C.byref(h)))
        return cls(h)

    @classmethod
    def learned(cls, geo, M, omega, net):
        """Sparse approximate inverse predicted by the graph network `net`."""
        h = C.c_void_p()
        _check(lib().bg_precond_create_learned(geo.h, M.h, float(omega), net.h, C.byref(h)))
        return cls(h)

    def nnz(self):
        return lib().bg_precond_nnz(self.h)

    def bound(self):
        """Learned: (rho(K1), smax), the near-field spectral estimate and the
        Neumann-coefficient bound it set."""
        out = np.zeros(2)
        _check(lib().bg_precond_bound(self.h, _ptr(out[:1]), _ptr(out[1:])))
        return float(out[0]), float(out[1])

    def csr(self, N):
        """(rowptr, col, val) copied to the host."""
        nnz = self.nnz()
        rowptr = np.zeros(N + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz, np.complex128)
        _check(lib().bg_precond_download(self.h, _ptr(rowptr), _ptr(col), _ptr(val)))
        return rowptr, col, val

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:   # lib is None at interpreter exit
            lib().bg_precond_destroy(self.h)
            self.h = None


DEFAULT_GNN_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "gnn_near_spai.f32")


class GNN:
    """Graph network predicting near-field sparse approximate inverses."""

    def __init__(self, seed=0):
        h = C.c_void_p()
        _check(lib().bg_gnn_create(int(seed), C.byref(h)))
        self.h = h

    @classmethod
    def load(cls, path=None):
        """Network with trained weights (raw little-endian float32 file)."""
        path = path or DEFAULT_GNN_WEIGHTS
        w = np.fromfile(path, dtype="<f4")
        if w.size != cls.num_params():
            raise BuffError(-1, f"{path}: {w.size} weights, the network has {cls.num_params()}")
        net = cls(0)
        net.set_params(w)
        return net

    @staticmethod
    def num_params():
        return lib().bg_gnn_num_params()

    def params(self):
        out = np.zeros(self.num_params(), np.float32)
        _check(lib().bg_gnn_get_params(self.h, _ptr(out)))
        return out

    def set_params(self, p):
        arr = np.ascontiguousarray(p, dtype=np.float32)
        assert arr.size == self.num_params()
        _check(lib().bg_gnn_set_params(self.h, _ptr(arr)))

    def grads(self):
        out = np.zeros(self.num_params(), np.float32)
        _check(lib().bg_gnn_get_grads(self.h, _ptr(out)))
        return out

    def train_step(self, geo, M, omega, Z, b=None, x=None, lam=0.0, lr=1e-3, probe_power=0):
        """One Adam step (lr=0: gradients only); returns the objective before the update.
        probe_power > 0 first maps the probes that many times through z <- z - M D^-1 z."""
        Zf = np.asfortranarray(Z, dtype=np.complex128)
        p = 1 if Zf.ndim == 1 else Zf.shape[1]
        bb = None if b is None else np.ascontiguousarray(b, dtype=np.complex128)
        xx = None if x is None else np.ascontiguousarray(x, dtype=np.complex128)
        loss = np.zeros(1)
        _check(lib().bg_gnn_train_step(self.h, geo.h, M.h, float(omega), _ptr(Zf), p, int(probe_power),
                                       _ptr(bb) if bb is not None else None,
                                       _ptr(xx) if xx is not None else None, float(lam), float(lr), _ptr(loss)))
        return float(loss[0])

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:   # lib is None at interpreter exit
            lib().bg_gnn_destroy(self.h)
            self.h = None


def GMRESSolve(M, B, P=None, tol=1e-10, restart=50, maxit=2000):
    """Solve M X = B (M assembled, not factored) with restarted GMRES; returns (X, stats)."""
    arr = np.asfortranarray(B, dtype=np.complex128).copy(order="F")
    nrhs = 1 if arr.ndim == 1 else arr.shape[1]
    st = np.zeros(3)
    _check(lib().bg_gmres_solve(M.h, P.h if P is not None else None, _ptr(arr), nrhs, float(tol), int(restart),
                                int(maxit), _ptr(st)))
    return arr, st


def GMRESSolveMixed(M, F, B, P=None, tol=1e-10, restart=50, maxit=2000, inner_tol=1e-5):
    """Solve M X = B with GMRES on the complex64 copy F of M plus FP64
    iterative refinement against M; returns (X, stats)."""
    arr = np.asfortranarray(B, dtype=np.complex128).copy(order="F")
    nrhs = 1 if arr.ndim == 1 else arr.shape[1]
    st = np.zeros(3)
    _check(lib().bg_gmres_solve_mixed(M.h, F.h, P.h if P is not None else None, _ptr(arr), nrhs, float(tol),
                                      int(restart), int(maxit), float(inner_tol), _ptr(st)))
    return arr, st


def GMRESLastInfo():
    """The calling thread's last mixed-precision solve: dict of steps,
    relres, sweeps, switched_to_jacobi, stopped_early, longest_cycle."""
    out = np.zeros(6)
    _check(lib().bg_gmres_last_info(_ptr(out)))
    return {"steps": int(out[0]), "relres": float(out[1]), "sweeps": int(out[2]),
            "switched_to_jacobi": bool(out[3]), "stopped_early": bool(out[4]), "longest_cycle": int(out[5])}


def SolveLearned(M, F, B, P=None, tol=1e-10, restart=80, maxit=1000, inner_tol=1e-5):
    """Mixed-precision GMRES with preconditioner P and the LU fallback (F
    holds LU factors afterwards if the fallback ran); returns (X, stats) with
    stats = (Krylov steps, final relative residual, sweeps, fallback used)."""
    arr = np.asfortranarray(B, dtype=np.complex128).copy(order="F")
    nrhs = 1 if arr.ndim == 1 else arr.shape[1]
    st = np.zeros(4)
    _check(lib().bg_gmres_solve_lu_fallback(M.h, F.h, P.h if P is not None else None, _ptr(arr), nrhs, float(tol),
                                            int(restart), int(maxit), float(inner_tol), _ptr(st)))
    return arr, st


def BatchSweep(geoms, omegas, IF, max_streams=4, graphs=True):
    """Batched frequency sweep: for every geometry and omega, assemble, LU,
    solve the plane wave IF and return the absorbed power of each object
    (overlap method).  Returns (pabs[ngeom, nomega, BG_BATCH_MAXOBJ], stats)."""
    geoms = list(geoms)
    w = np.ascontiguousarray(np.asarray(omegas, dtype=np.complex128))
    hs = (C.c_void_p * len(geoms))(*[g.h for g in geoms])
    out = np.zeros((len(geoms), len(w), BG_BATCH_MAXOBJ))
    st = np.zeros(4 + 4 * len(geoms))
    _check(lib().bg_batch_sweep(C.cast(hs, C.c_void_p), len(geoms), _ptr(w), len(w), _ptr(IF.E0), _ptr(IF.nHat),
                                int(max_streams), 0 if graphs else BG_BATCH_NO_GRAPHS, _ptr(out), _ptr(st)))
    return out, st


def launch_count():
    return lib().bg_kernel_launch_count()


def synchronize():
    _check(lib().bg_synchronize())


PROF_CLASSES = ("lu_gemm", "lu_panel", "lu_laswp", "trsm_leaf", "assemble_far", "assemble_near_gram",
                "gmres_matvec", "gnn_precond", "gmres_orthogonalise", "gmres_precond_apply", "lu_solve_trsv",
                "refine_residual")


def profile_begin():
    _check(lib().bg_profile_begin())


def profile_read():
    n = len(PROF_CLASSES)
    cnt = np.zeros(n, dtype=np.int64)
    ms = np.zeros(n)
    fl = np.zeros(n)
    _check(lib().bg_profile_read(n, _ptr(cnt), _ptr(ms), _ptr(fl)))
    return {k: dict(launches=int(cnt[i]), ms=float(ms[i]), flops=float(fl[i])) for i, k in enumerate(PROF_CLASSES)}


def profile_end():
    _check(lib().bg_profile_end())
