"""Build tensors from the reference's known-answer fixtures.

The C++ constructors fill data in Fortran order and infer the remaining
dimension from the data length (tensors.hpp:789-1854); these helpers do the
same so that the fixtures read exactly like the reference tests.
"""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KATS = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))


def cplx(vals):
    out = []
    for v in vals:
        out.append(complex(v[0], v[1]) if isinstance(v, list) else complex(v))
    return np.array(out, dtype=np.complex128)


def exp_boundary(vals, c):
    a = cplx(vals)
    b = int(round((a.size / c) ** 0.5))
    return np.asfortranarray(a.reshape((b, b, c), order="F"))


def state_site(vals, bl, br):
    a = cplx(vals)
    d = a.size // (bl * br)
    return np.asfortranarray(a.reshape((br, bl, d), order="F"))


def overlap_site(vals, bl, br):
    a = cplx(vals)
    d = a.size // (bl * br)
    return np.asfortranarray(a.reshape((bl, d, br), order="F"))


def operator_site(indices, matrices, cl, cr):
    idx = np.array([int(round(v)) for v in indices], dtype=np.uint32)
    nnz = idx.size // 2
    W = cplx(matrices)
    d = int(round((W.size / nnz) ** 0.5))
    return (np.asfortranarray(idx.reshape((2, nnz), order="F")),
            np.asfortranarray(W.reshape((d, d, nnz), order="F")), d)
