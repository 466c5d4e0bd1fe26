"""The reference's YAML operator format through the library's reader and writer
(``nc_yaml_*``, include/nutcracker_b200.h; yaml.cpp:169-306, README:27-187).

``read_operator(text)`` returns the chain's sites as ``OperatorSite`` objects
(the format of ``nutcracker_b200.operators``), ready for ``Chain`` and
``Server.submit``; errors raise ``NutcrackerError`` with the reference's
messages.  ``write_operator(sites)`` emits the same format.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import NutcrackerError, _check, lib
from .chain import _operator_structs, nc_operator_site
from .operators import OperatorSite

lib.nc_yaml_read_operator.restype = ct.c_void_p
lib.nc_yaml_read_operator.argtypes = [ct.c_char_p, ct.c_size_t, ct.c_char_p]
lib.nc_parsed_operator_number_of_sites.restype = ct.c_uint32
lib.nc_parsed_operator_number_of_sites.argtypes = [ct.c_void_p]
lib.nc_parsed_operator_sites.restype = ct.POINTER(nc_operator_site)
lib.nc_parsed_operator_sites.argtypes = [ct.c_void_p]
lib.nc_parsed_operator_free.argtypes = [ct.c_void_p]
lib.nc_yaml_write_operator.restype = ct.c_size_t
lib.nc_yaml_write_operator.argtypes = [ct.c_uint32, ct.POINTER(nc_operator_site), ct.c_char_p, ct.c_size_t]


def read_operator(text, location=None):
    """Sites of the operator in YAML ``text`` (str or bytes); ``location`` is a
    slash-separated path of keys to the operator inside the document."""
    data = text.encode() if isinstance(text, str) else bytes(text)
    h = lib.nc_yaml_read_operator(data, len(data), location.encode() if location else None)
    if not h:
        _check()
        raise NutcrackerError(-1, "nc_yaml_read_operator failed")
    try:
        n = lib.nc_parsed_operator_number_of_sites(h)
        arr = lib.nc_parsed_operator_sites(h)
        sites = []
        for i in range(n):
            s = arr[i]
            d, nnz = s.physical_dimension, s.number_of_matrices
            idx = np.ctypeslib.as_array(s.indices, shape=(2 * nnz,)).reshape((2, nnz), order="F").copy(order="F") \
                if nnz else np.zeros((2, 0), dtype=np.uint32, order="F")
            if nnz:
                raw = np.ctypeslib.as_array(ct.cast(s.matrices, ct.POINTER(ct.c_double)), shape=(2 * d * d * nnz,))
                W = (raw[0::2] + 1j * raw[1::2]).reshape((d, d, nnz), order="F").copy(order="F")
            else:
                W = np.zeros((d, d, 0), dtype=complex, order="F")
            sites.append(OperatorSite(d, s.left_dimension, s.right_dimension, idx.astype(np.uint32), W))
        return sites
    finally:
        lib.nc_parsed_operator_free(h)


def write_operator(sites):
    """The operator in the reference's YAML format (identical sites listed once)."""
    arr, keep = _operator_structs(sites)
    n = lib.nc_yaml_write_operator(len(sites), arr, None, 0)
    buf = ct.create_string_buffer(n + 1)
    lib.nc_yaml_write_operator(len(sites), arr, buf, n + 1)
    return buf.value.decode()
