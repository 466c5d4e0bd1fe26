"""Python host bindings for the B200 variational-MPS sweep library.

The product is the C-ABI shared library ``lib/libnutcracker_b200.so``
(declared in ``include/nutcracker_b200.h``).  This module binds it with
ctypes and mirrors the reference's ``Nutcracker::Core`` wrappers
(``includes/nutcracker/core.hpp:34-302``): same function names and argument
meaning, numpy arrays with the reference's Fortran shapes in and out.

There is no CPU fallback: importing this module raises if the library is
missing, and every call raises ``NutcrackerError`` when the library reports a
failure.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libnutcracker_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError("nutcracker_b200: CUDA library not built (%s); run "
                      "`python nutcracker-1_b200/nutcracker_b200/build.py`" % LIB_PATH)

lib = ct.CDLL(LIB_PATH)

C128 = np.complex128
_u32p = ct.POINTER(ct.c_uint32)
_vp = ct.c_void_p


class NutcrackerError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("[%d] %s" % (code, msg))
        self.code = code


lib.nc_last_status.restype = ct.c_int
lib.nc_last_error.restype = ct.c_char_p
lib.nc_launch_count.restype = ct.c_uint64
lib.nc_version.restype = ct.c_char_p


def _check():
    st = lib.nc_last_status()
    if st != 0:
        raise NutcrackerError(st, lib.nc_last_error().decode())


def _u(x):
    return ct.byref(ct.c_uint32(int(x)))


def _c(a):
    """Column-major complex128 buffer pointer (keeps `a` alive via caller)."""
    return a.ctypes.data_as(_vp)


def _F(a):
    return np.asfortranarray(np.asarray(a, dtype=C128))


def _idx(a):
    return np.asfortranarray(np.asarray(a, dtype=np.uint32))


def launch_count():
    return int(lib.nc_launch_count())


def version():
    return lib.nc_version().decode()


class Core:
    """ctypes mirror of Nutcracker::Core (core.hpp:34-302) over the GPU library."""

    @staticmethod
    def compute_expectation(bl, br, cl, cr, d, L, S, nnz, idx, W, R):
        L, S, W, R, idx = _F(L), _F(S), _F(W), _F(R), _idx(idx)
        out = np.zeros(1, C128)
        lib.compute_expectation_(_u(bl), _u(br), _u(cl), _u(cr), _u(d), _c(L), _c(S), _u(nnz),
                                 idx.ctypes.data_as(_u32p), _c(W), _c(R), _c(out))
        _check()
        return complex(out[0])

    @staticmethod
    def compute_optimization_matrix(bl, br, cl, cr, d, L, nnz, idx, W, R):
        L, W, R, idx = _F(L), _F(W), _F(R), _idx(idx)
        n = bl * br * d
        H = np.zeros((n, n), C128, order="F")
        lib.compute_optimization_matrix_(_u(bl), _u(br), _u(cl), _u(cr), _u(d), _c(L), _u(nnz),
                                         idx.ctypes.data_as(_u32p), _c(W), _c(R), _c(H))
        _check()
        return H

    @staticmethod
    def construct_left_exp_boundary(b, c, sb, ob):
        sb, ob = _F(sb), _F(ob)
        out = np.zeros((b, b, c), C128, order="F")
        lib.construct_left_exp_boundary_(_u(b), _u(c), _c(sb), _c(ob), _c(out))
        _check()
        return out

    @staticmethod
    def construct_right_exp_boundary(b, c, sb, ob):
        sb, ob = _F(sb), _F(ob)
        out = np.zeros((b, b, c), C128, order="F")
        lib.construct_right_exp_boundary_(_u(b), _u(c), _c(sb), _c(ob), _c(out))
        _check()
        return out

    @staticmethod
    def contract_expectation_boundaries(b, c, L, R):
        L, R = _F(L), _F(R)
        out = np.zeros(1, C128)
        lib.contract_expectation_boundaries_(_u(b), _u(c), _c(L), _c(R), _c(out))
        _check()
        return complex(out[0])

    @staticmethod
    def contract_sos_left(bl, br, cl, cr, d, L, nnz, idx, W, S):
        L, W, S, idx = _F(L), _F(W), _F(S), _idx(idx)
        out = np.zeros((br, br, cr), C128, order="F")
        lib.contract_sos_left_(_u(bl), _u(br), _u(cl), _u(cr), _u(d), _c(L), _u(nnz),
                               idx.ctypes.data_as(_u32p), _c(W), _c(S), _c(out))
        _check()
        return out

    @staticmethod
    def contract_sos_right(bl, br, cl, cr, d, R, nnz, idx, W, S):
        R, W, S, idx = _F(R), _F(W), _F(S), _idx(idx)
        out = np.zeros((bl, bl, cl), C128, order="F")
        lib.contract_sos_right_(_u(bl), _u(br), _u(cl), _u(cr), _u(d), _c(R), _u(nnz),
                                idx.ctypes.data_as(_u32p), _c(W), _c(S), _c(out))
        _check()
        return out

    @staticmethod
    def contract_vs_left(blo, bro, bln, brn, d, Lov, P, S):
        Lov, P, S = _F(Lov), _F(P), _F(S)
        out = np.zeros((brn, bro), C128, order="F")
        lib.contract_vs_left_(_u(blo), _u(bro), _u(bln), _u(brn), _u(d), _c(Lov), _c(P), _c(S), _c(out))
        _check()
        return out

    @staticmethod
    def contract_vs_right(blo, bro, bln, brn, d, Rov, P, S):
        Rov, P, S = _F(Rov), _F(P), _F(S)
        out = np.zeros((blo, bln), C128, order="F")
        lib.contract_vs_right_(_u(blo), _u(bro), _u(bln), _u(brn), _u(d), _c(Rov), _c(P), _c(S), _c(out))
        _check()
        return out

    @staticmethod
    def form_overlap_vector(blo, bro, bln, brn, d, Lov, Rov, P):
        Lov, Rov, P = _F(Lov), _F(Rov), _F(P)
        out = np.zeros((brn, bln, d), C128, order="F")
        lib.form_overlap_vector_(_u(blo), _u(bro), _u(bln), _u(brn), _u(d), _c(Lov), _c(Rov), _c(P), _c(out))
        _check()
        return out

    @staticmethod
    def form_overlap_site_tensor(br, bl, d, S):
        S = _F(S)
        out = np.zeros((bl, d, br), C128, order="F")
        lib.form_overlap_site_tensor_(_u(br), _u(bl), _u(d), _c(S), _c(out))
        _check()
        return out


def _int32(u):
    u = int(u) & 0xFFFFFFFF
    return u - (1 << 32) if u >= (1 << 31) else u


class _CoreSolver:
    @staticmethod
    def optimize(bl, br, cl, cr, d, L, nnz, idx, W, R, nproj, nrefl, orth_dim, reflectors, coefficients,
                 swaps, which, tol, iterations, guess):
        """core.cpp:694-733.  Returns (info, iterations, eigenvalue, result, normal)."""
        L, W, R, guess, idx = _F(L), _F(W), _F(R), _F(guess), _idx(idx)
        if nproj:
            reflectors, coefficients = _F(reflectors), _F(coefficients)
            swaps = _idx(swaps)
            rp, cp, sp = _c(reflectors), _c(coefficients), swaps.ctypes.data_as(_u32p)
        else:
            rp = cp = sp = None
        result = np.zeros((br, bl, d), C128, order="F")
        ev = np.zeros(1, C128)
        normal = ct.c_double(0)
        it = ct.c_uint32(int(iterations))
        w = ct.create_string_buffer(which.encode() if isinstance(which, str) else which, 2)
        lib.optimize_.restype = ct.c_uint32
        info = lib.optimize_(_u(bl), _u(br), _u(cl), _u(cr), _u(d), _c(L), _u(nnz), idx.ctypes.data_as(_u32p),
                             _c(W), _c(R), _u(nproj), _u(nrefl), _u(orth_dim), rp, cp, sp, w,
                             ct.byref(ct.c_double(tol)), ct.byref(it), _c(guess), _c(result), _c(ev),
                             ct.byref(normal))
        _check()
        return _int32(info), int(it.value), complex(ev[0]), result, float(normal.value)

    @staticmethod
    def convert_vectors_to_reflectors(n, m, vectors):
        """core.cpp:370-391.  Returns (reflectors, rank, coefficients, swaps)."""
        v = np.array(_F(vectors), order="F", copy=True)
        k = min(n, m)
        coeff = np.zeros(max(k, 1), C128)
        swaps = np.zeros(max(k, 1), np.uint32)
        rank = ct.c_uint32(0)
        lib.convert_vectors_to_reflectors_(_u(n), _u(m), _c(v), ct.byref(rank), _c(coeff),
                                           swaps.ctypes.data_as(_u32p))
        _check()
        return v, int(rank.value), coeff[:k], swaps[:k]

    @staticmethod
    def filter_components_outside_orthog(n, nproj, nrefl, orth_dim, reflectors, coefficients, swaps, x):
        reflectors, coefficients, x, swaps = _F(reflectors), _F(coefficients), _F(x), _idx(swaps)
        out = np.zeros(n, C128)
        lib.filter_components_outside_orthog_(_u(n), _u(nproj), _u(nrefl), _u(orth_dim), _c(reflectors),
                                              _c(coefficients), swaps.ctypes.data_as(_u32p), _c(x), _c(out))
        _check()
        return out

    @staticmethod
    def compute_overlap_with_projectors(nproj, nrefl, reflectors, coefficients, swaps, n, x):
        reflectors, coefficients, x, swaps = _F(reflectors), _F(coefficients), _F(x), _idx(swaps)
        out = np.zeros(1, C128)
        lib.compute_overlap_with_projectors_(_u(nproj), _u(nrefl), _c(reflectors), _c(coefficients),
                                             swaps.ctypes.data_as(_u32p), _u(n), _c(x), _c(out))
        _check()
        return complex(out[0])

    @staticmethod
    def random_projector_matrix(length, nproj):
        """core.cpp:766-781 / projectors.cpp:145-171.  Returns (rank, reflectors, coefficients, swaps)."""
        k = min(length, nproj)
        refl = np.zeros((length, nproj), C128, order="F")
        coeff = np.zeros(max(k, 1), C128)
        swaps = np.zeros(max(k, 1), np.uint32)
        rank = ct.c_uint32(0)
        lib.random_projector_matrix_(_u(length), _u(nproj), ct.byref(rank), _c(refl), _c(coeff),
                                     swaps.ctypes.data_as(_u32p))
        _check()
        return int(rank.value), refl, coeff[:k], swaps[:k]


    # -- gauge moves (core.cpp:570-765) -----------------------------------
    @staticmethod
    def norm_denorm_going_left(bl, bm, br, dl, dr, A, B):
        """Returns (info, denormalized A (bm,bl,dl), normalized B (br,bm,dr))."""
        A, B = _F(A), _F(B)
        oA = np.zeros((bm, bl, dl), C128, order="F")
        oB = np.zeros((br, bm, dr), C128, order="F")
        info = lib.norm_denorm_going_left_(_u(bl), _u(bm), _u(br), _u(dl), _u(dr), _c(A), _c(B), _c(oA), _c(oB))
        _check()
        return info, oA, oB

    @staticmethod
    def norm_denorm_going_right(bl, bm, br, dl, dr, A, B):
        """Returns (info, normalized A (bm,bl,dl), denormalized B (br,bm,dr))."""
        A, B = _F(A), _F(B)
        oA = np.zeros((bm, bl, dl), C128, order="F")
        oB = np.zeros((br, bm, dr), C128, order="F")
        info = lib.norm_denorm_going_right_(_u(bl), _u(bm), _u(br), _u(dl), _u(dr), _c(A), _c(B), _c(oA), _c(oB))
        _check()
        return info, oA, oB

    @staticmethod
    def norm_for_left(br, bl, d, S):
        S = _F(S)
        out = np.zeros((br, bl, d), C128, order="F")
        info = lib.norm_for_left_(_u(br), _u(bl), _u(d), _c(S), _c(out))
        _check()
        return info, out

    @staticmethod
    def norm_for_right(br, bl, d, S):
        S = _F(S)
        out = np.zeros((br, bl, d), C128, order="F")
        info = lib.norm_for_right_(_u(br), _u(bl), _u(d), _c(S), _c(out))
        _check()
        return info, out

    @staticmethod
    def increase_bandwidth_between(bl, bm, br, dl, dr, new_bm, A, B):
        A, B = _F(A), _F(B)
        oA = np.zeros((new_bm, bl, dl), C128, order="F")
        oB = np.zeros((br, new_bm, dr), C128, order="F")
        info = lib.increase_bandwidth_between_(_u(bl), _u(bm), _u(br), _u(dl), _u(dr), _u(new_bm), _c(A), _c(B),
                                               _c(oA), _c(oB))
        _check()
        return info, oA, oB

    @staticmethod
    def rand_norm_state_site_tensor(br, bl, d):
        out = np.zeros((br, bl, d), C128, order="F")
        lib.rand_norm_state_site_tensor_(_u(br), _u(bl), _u(d), _c(out))
        _check()
        return out

    @staticmethod
    def rand_unnorm_state_site_tensor(br, bl, d):
        out = np.zeros((br, bl, d), C128, order="F")
        lib.rand_unnorm_state_site_tensor_(_u(br), _u(bl), _u(d), _c(out))
        _check()
        return out

    @staticmethod
    def form_norm_overlap_tensors(bl, bm, br, dl, dr, S1, S2):
        S1, S2 = _F(S1), _F(S2)
        lno = np.zeros((bl, dl, bm), C128, order="F")
        uno = np.zeros((bl, dl, bm), C128, order="F")
        dS2 = np.zeros((br, bm, dr), C128, order="F")
        rno = np.zeros((bm, dr, br), C128, order="F")
        lib.form_norm_overlap_tensors_(_u(bl), _u(bm), _u(br), _u(dl), _u(dr), _c(S1), _c(S2), _c(lno), _c(uno),
                                       _c(dS2), _c(rno))
        _check()
        return lno, uno, dS2, rno


for _name in ("optimize", "convert_vectors_to_reflectors", "filter_components_outside_orthog",
              "compute_overlap_with_projectors", "random_projector_matrix", "norm_denorm_going_left",
              "norm_denorm_going_right", "norm_for_left", "norm_for_right", "increase_bandwidth_between",
              "rand_norm_state_site_tensor", "rand_unnorm_state_site_tensor", "form_norm_overlap_tensors"):
    setattr(Core, _name, getattr(_CoreSolver, _name))

lib.norm_denorm_going_left_.restype = ct.c_int32
lib.norm_denorm_going_right_.restype = ct.c_int32
lib.norm_for_left_.restype = ct.c_int32
lib.norm_for_right_.restype = ct.c_int32
lib.increase_bandwidth_between_.restype = ct.c_int32


def set_krylov_dimension(m):
    if lib.nc_set_krylov_dimension(int(m)) != 0:
        _check()
