"""ctypes binding of the C API with the reference's names (include/nutcracker.h;
sources/c-interface/*.cpp): matrices, vectors, operator and state terms and
builders (the automaton compiler), protobuf serialization, the simple solvers
and state overlaps / expectation values.

Functions raise ``NutcrackerError`` with the library's message when the C
call reports an error through ``Nutcracker_getError``.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import NutcrackerError, lib

_vp = ct.c_void_p
_c = ct.c_double * 2


def _cz(z):
    z = complex(z)
    return _c(z.real, z.imag)


def _err():
    m = lib.Nutcracker_getError()
    if m is not None:
        lib.Nutcracker_clearError()
        raise NutcrackerError(-1, m.decode())


def _call(fn, *args):
    lib.Nutcracker_clearError()
    r = fn(*args)
    _err()
    return r


def _decl(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args


for _n in ("Nutcracker_clearError",):
    _decl(_n, None, [])
_decl("Nutcracker_getError", ct.c_char_p, [])
_decl("Nutcracker_setError", None, [ct.c_char_p])
for _n in ("Matrix", "Vector"):
    _decl("Nutcracker_%s_free" % _n, None, [_vp])
    _decl("Nutcracker_%s_add" % _n, _vp, [_vp, _vp])
    _decl("Nutcracker_%s_multiply" % _n, _vp, [ct.POINTER(_c), _vp])
    _decl("Nutcracker_%s_getSize" % _n, ct.c_uint32, [_vp])
for _p in "IXYZ":
    _decl("Nutcracker_Matrix_getPauli" + _p, _vp, [])
_decl("Nutcracker_Matrix_new", _vp, [ct.c_uint32, _vp])
_decl("Nutcracker_Matrix_newDiagonal", _vp, [ct.c_uint32, _vp])
_decl("Nutcracker_Matrix_getElementAtCoordinate", None, [_vp, ct.c_uint32, ct.c_uint32, ct.POINTER(_c)])
_decl("Nutcracker_Vector_new", _vp, [ct.c_uint32, _vp])
_decl("Nutcracker_Vector_newBasis", _vp, [ct.c_uint32, ct.c_uint32])
_decl("Nutcracker_Vector_getElementAtIndex", None, [_vp, ct.c_uint32, ct.POINTER(_c)])
for _k in ("Operator", "State"):
    _decl("Nutcracker_%sBuilder_new" % _k, _vp, [ct.c_uint32, ct.POINTER(ct.c_uint32)])
    _decl("Nutcracker_%sBuilder_newSimple" % _k, _vp, [ct.c_uint32, ct.c_uint32])
    _decl("Nutcracker_%sBuilder_free" % _k, None, [_vp])
    _decl("Nutcracker_%sBuilder_numberOfSites" % _k, ct.c_uint32, [_vp])
    _decl("Nutcracker_%sBuilder_dimensionOfSite" % _k, ct.c_uint32, [_vp, ct.c_uint32])
    _decl("Nutcracker_%sBuilder_addProductTerm" % _k, None, [_vp, ct.POINTER(_vp)])
    _decl("Nutcracker_%sBuilder_addTerm" % _k, None, [_vp, _vp])
    _decl("Nutcracker_%sBuilder_compile" % _k, _vp, [_vp])
    _decl("Nutcracker_%sTerm_free" % _k, None, [_vp])
    _decl("Nutcracker_%sTerm_add" % _k, _vp, [_vp, _vp])
    _decl("Nutcracker_%sTerm_multiply" % _k, _vp, [ct.POINTER(_c), _vp])
    _decl("Nutcracker_%s_free" % _k, None, [_vp])
    _decl("Nutcracker_%s_serialize" % _k, _vp, [_vp])
    _decl("Nutcracker_%s_deserialize" % _k, _vp, [ct.c_uint32, ct.c_char_p])
_decl("Nutcracker_OperatorBuilder_compileCustomized", _vp, [_vp, ct.c_bool, ct.c_bool])
_decl("Nutcracker_StateBuilder_compileCustomized", _vp, [_vp, ct.c_bool])
_decl("Nutcracker_OperatorTerm_create_LocalExternalField", _vp, [ct.c_uint32, _vp])
_decl("Nutcracker_OperatorTerm_create_GlobalExternalField", _vp, [_vp])
_decl("Nutcracker_OperatorTerm_create_LocalNeighborCouplingField", _vp, [ct.c_uint32, _vp, _vp])
_decl("Nutcracker_OperatorTerm_create_GlobalNeighborCouplingField", _vp, [_vp, _vp])
_decl("Nutcracker_OperatorTerm_create_TransverseIsingField", _vp, [_vp, _vp, _vp])
_decl("Nutcracker_StateTerm_create_ProductWithOneSiteDifferent", _vp, [ct.c_uint32, _vp, _vp])
_decl("Nutcracker_StateTerm_create_W", _vp, [_vp, _vp, ct.c_bool])
_decl("Nutcracker_Operator_simpleSolveForLeastEigenvalues", None, [_vp, ct.c_uint32, ct.POINTER(ct.c_float)])
_decl("Nutcracker_Operator_simpleSolveForLeastEigenvaluesWithEigenvectors", None,
      [_vp, ct.c_uint32, ct.POINTER(ct.c_float), ct.POINTER(_vp)])
_decl("Nutcracker_State_computeOverlap", None, [_vp, _vp, ct.POINTER(_c)])
_decl("Nutcracker_State_computeExpectation", None, [_vp, _vp, ct.POINTER(_c)])
_decl("Nutcracker_Serialization_free", None, [_vp])
_decl("Nutcracker_Serialization_getSize", ct.c_uint32, [_vp])
_decl("Nutcracker_Serialization_write", None, [_vp, ct.c_char_p])
_decl("Nutcracker_Version_getComponent", ct.c_uint32, [ct.c_uint32])
_decl("Nutcracker_Version_getSize", ct.c_uint32, [])
_decl("Nutcracker_Version_getString", ct.c_char_p, [])


class _Handle:
    _free = None

    def __init__(self, h):
        if not h:
            _err()
            raise NutcrackerError(-1, "null handle")
        self.h = ct.c_void_p(h)

    def close(self):
        if getattr(self, "h", None) is not None and self._free:
            getattr(lib, self._free)(self.h)
        self.h = None

    def __del__(self):
        self.close()


def _serialized(h):
    size = lib.Nutcracker_Serialization_getSize(h)
    buf = ct.create_string_buffer(size)
    lib.Nutcracker_Serialization_write(h, buf)
    lib.Nutcracker_Serialization_free(h)
    return buf.raw[:size]


class Matrix(_Handle):
    _free = "Nutcracker_Matrix_free"

    @classmethod
    def new(cls, m):
        m = np.ascontiguousarray(np.asarray(m, dtype=complex))   # row-major, as the C API takes it
        return cls(_call(lib.Nutcracker_Matrix_new, m.shape[0], m.ctypes.data))

    @classmethod
    def diagonal(cls, d):
        d = np.ascontiguousarray(np.asarray(d, dtype=complex))
        return cls(_call(lib.Nutcracker_Matrix_newDiagonal, d.size, d.ctypes.data))

    @staticmethod
    def pauli(p):
        m = Matrix(getattr(lib, "Nutcracker_Matrix_getPauli" + p)())
        m._free = None   # owned by the library
        return m

    def __add__(self, o):
        return Matrix(_call(lib.Nutcracker_Matrix_add, self.h, o.h))

    def __rmul__(self, c):
        z = _cz(c)
        return Matrix(_call(lib.Nutcracker_Matrix_multiply, ct.byref(z), self.h))

    def size(self):
        return lib.Nutcracker_Matrix_getSize(self.h)

    def element(self, i, j):
        z = _c()
        _call(lib.Nutcracker_Matrix_getElementAtCoordinate, self.h, i, j, ct.byref(z))
        return complex(z[0], z[1])

    def array(self):
        n = self.size()
        return np.array([[self.element(i, j) for j in range(n)] for i in range(n)])


class Vector(_Handle):
    _free = "Nutcracker_Vector_free"

    @classmethod
    def new(cls, v):
        v = np.ascontiguousarray(np.asarray(v, dtype=complex))
        return cls(_call(lib.Nutcracker_Vector_new, v.size, v.ctypes.data))

    @classmethod
    def basis(cls, d, k):
        return cls(_call(lib.Nutcracker_Vector_newBasis, d, k))

    def __add__(self, o):
        return Vector(_call(lib.Nutcracker_Vector_add, self.h, o.h))

    def __rmul__(self, c):
        z = _cz(c)
        return Vector(_call(lib.Nutcracker_Vector_multiply, ct.byref(z), self.h))

    def array(self):
        out = []
        for i in range(lib.Nutcracker_Vector_getSize(self.h)):
            z = _c()
            _call(lib.Nutcracker_Vector_getElementAtIndex, self.h, i, ct.byref(z))
            out.append(complex(z[0], z[1]))
        return np.array(out)


class _Term(_Handle):
    _kind = ""

    def __add__(self, o):
        return type(self)(_call(getattr(lib, "Nutcracker_%sTerm_add" % self._kind), self.h, o.h))

    def __rmul__(self, c):
        z = _cz(c)
        return type(self)(_call(getattr(lib, "Nutcracker_%sTerm_multiply" % self._kind), ct.byref(z), self.h))


class OperatorTerm(_Term):
    _free = "Nutcracker_OperatorTerm_free"
    _kind = "Operator"

    @classmethod
    def local_external_field(cls, site, m):
        return cls(_call(lib.Nutcracker_OperatorTerm_create_LocalExternalField, site, m.h))

    @classmethod
    def global_external_field(cls, m):
        return cls(_call(lib.Nutcracker_OperatorTerm_create_GlobalExternalField, m.h))

    @classmethod
    def local_neighbor_coupling_field(cls, site, left, right):
        return cls(_call(lib.Nutcracker_OperatorTerm_create_LocalNeighborCouplingField, site, left.h, right.h))

    @classmethod
    def global_neighbor_coupling_field(cls, left, right):
        return cls(_call(lib.Nutcracker_OperatorTerm_create_GlobalNeighborCouplingField, left.h, right.h))

    @classmethod
    def transverse_ising_field(cls, external, left, right):
        return cls(_call(lib.Nutcracker_OperatorTerm_create_TransverseIsingField, external.h, left.h, right.h))


class StateTerm(_Term):
    _free = "Nutcracker_StateTerm_free"
    _kind = "State"

    @classmethod
    def product_with_one_site_different(cls, site, common, special):
        return cls(_call(lib.Nutcracker_StateTerm_create_ProductWithOneSiteDifferent, site, common.h, special.h))

    @classmethod
    def w(cls, common, special, normalized=True):
        return cls(_call(lib.Nutcracker_StateTerm_create_W, common.h, special.h, bool(normalized)))


class Operator(_Handle):
    _free = "Nutcracker_Operator_free"

    def serialize(self):
        return _serialized(_call(lib.Nutcracker_Operator_serialize, self.h))

    @classmethod
    def deserialize(cls, data):
        return cls(_call(lib.Nutcracker_Operator_deserialize, len(data), data))

    def simple_solve(self, levels, with_eigenvectors=False):
        e = (ct.c_float * levels)()
        if not with_eigenvectors:
            _call(lib.Nutcracker_Operator_simpleSolveForLeastEigenvalues, self.h, levels, e)
            return list(e)
        v = (_vp * levels)()
        _call(lib.Nutcracker_Operator_simpleSolveForLeastEigenvaluesWithEigenvectors, self.h, levels, e, v)
        return list(e), [State(v[k]) for k in range(levels)]


class State(_Handle):
    _free = "Nutcracker_State_free"

    def serialize(self):
        return _serialized(_call(lib.Nutcracker_State_serialize, self.h))

    @classmethod
    def deserialize(cls, data):
        return cls(_call(lib.Nutcracker_State_deserialize, len(data), data))

    def overlap(self, other):
        z = _c()
        _call(lib.Nutcracker_State_computeOverlap, self.h, other.h, ct.byref(z))
        return complex(z[0], z[1])

    def expectation(self, op):
        z = _c()
        _call(lib.Nutcracker_State_computeExpectation, self.h, op.h, ct.byref(z))
        return complex(z[0], z[1])


class _Builder(_Handle):
    _kind = ""
    _result = None
    _component = None

    def __init__(self, dims):
        arr = (ct.c_uint32 * len(dims))(*dims)
        super().__init__(_call(getattr(lib, "Nutcracker_%sBuilder_new" % self._kind), len(dims), arr))
        self._free = "Nutcracker_%sBuilder_free" % self._kind

    def number_of_sites(self):
        return getattr(lib, "Nutcracker_%sBuilder_numberOfSites" % self._kind)(self.h)

    def dimension_of_site(self, i):
        return _call(getattr(lib, "Nutcracker_%sBuilder_dimensionOfSite" % self._kind), self.h, i)

    def add_product_term(self, components):
        # the C call reads one component per site, so the count is checked here
        n = self.number_of_sites()
        if len(components) != n:
            raise NutcrackerError(-1, "The number of sites in the argument (%d) does not match the number of sites "
                                      "in the system (%d).  [%d != %d]" % (len(components), n, len(components), n))
        arr = (_vp * len(components))(*[c.h.value for c in components])
        _call(getattr(lib, "Nutcracker_%sBuilder_addProductTerm" % self._kind), self.h, arr)
        return self

    def add_term(self, term):
        _call(getattr(lib, "Nutcracker_%sBuilder_addTerm" % self._kind), self.h, term.h)
        return self


class OperatorBuilder(_Builder):
    _kind = "Operator"

    def compile(self, optimize=True, add_start_and_end_loops=True):
        return Operator(_call(lib.Nutcracker_OperatorBuilder_compileCustomized, self.h, optimize,
                              add_start_and_end_loops))


class StateBuilder(_Builder):
    _kind = "State"

    def compile(self, optimize=True):
        return State(_call(lib.Nutcracker_StateBuilder_compileCustomized, self.h, optimize))


def version():
    return (lib.Nutcracker_Version_getString().decode(),
            [lib.Nutcracker_Version_getComponent(i) for i in range(lib.Nutcracker_Version_getSize())])
