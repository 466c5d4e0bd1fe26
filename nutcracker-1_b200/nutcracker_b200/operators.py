"""MPO constructors (sources/common/operators.cpp) for the device chain.

Each site is an ``OperatorSite`` with the reference's storage
(tensors.hpp:1641-1854): ``idx`` (2, nnz) uint32 1-based (from, to) pairs and
``W`` (d, d, nnz) column-major, filled from row-major link matrices exactly as
``constructOperatorSite`` does (operators.cpp:83-112), so W(o1, o2) =
M[o2][o1] and the applied operator is M.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

I2 = np.eye(2, dtype=complex)
PAULI_X = np.array([[0, 1], [1, 0]], dtype=complex)
PAULI_Y = np.array([[0, -1j], [1j, 0]], dtype=complex)
PAULI_Z = np.array([[1, 0], [0, -1]], dtype=complex)


@dataclass
class OperatorSite:
    d: int
    cl: int
    cr: int
    idx: np.ndarray
    W: np.ndarray

    @property
    def nnz(self):
        return self.W.shape[2]


def construct_operator_site(d, cl, cr, links):
    """operators.cpp:83-112.  links: (from, to, M) with M row-major d x d."""
    nnz = len(links)
    idx = np.zeros((2, nnz), dtype=np.uint32, order="F")
    W = np.zeros((d, d, nnz), dtype=complex, order="F")
    for n, (f, t, M) in enumerate(links):
        idx[0, n], idx[1, n] = f, t
        M = np.asarray(M, dtype=complex)
        if M.shape != (d, d):
            raise ValueError("link matrix has the wrong shape")
        W[:, :, n] = M.T
    return OperatorSite(d, cl, cr, idx, W)


def _chain(first, middle, last, n):
    return [first] + [middle(i) for i in range(1, n - 1)] + [last]


def transverse_ising_model(n, coupling):
    """constructTransverseIsingModelOperator (operators.cpp:114-165):
    H = sum Z_i + coupling sum X_i X_{i+1}."""
    if n < 2:
        raise ValueError("need at least two sites")
    X2 = coupling * PAULI_X
    first = construct_operator_site(2, 1, 3, [(1, 1, I2), (1, 2, PAULI_X), (1, 3, PAULI_Z)])
    mid = construct_operator_site(2, 3, 3, [(1, 1, I2), (1, 2, PAULI_X), (2, 3, X2), (1, 3, PAULI_Z), (3, 3, I2)])
    last = construct_operator_site(2, 3, 1, [(1, 1, PAULI_Z), (2, 1, X2), (3, 1, I2)])
    return _chain(first, lambda i: mid, last, n)


def ferromagnetic_transverse_ising(n, lam):
    """H = -sum Z_i Z_{i+1} - lam sum X_i (automaton 1->1 I, 1->2 Z, 2->3 -Z,
    1->3 -lam X, 3->3 I; the last site maps state 3 to 1)."""
    if n < 2:
        raise ValueError("need at least two sites")
    first = construct_operator_site(2, 1, 3, [(1, 1, I2), (1, 2, PAULI_Z), (1, 3, -lam * PAULI_X)])
    mid = construct_operator_site(2, 3, 3, [(1, 1, I2), (1, 2, PAULI_Z), (2, 3, -PAULI_Z), (1, 3, -lam * PAULI_X),
                                            (3, 3, I2)])
    last = construct_operator_site(2, 3, 1, [(2, 1, -PAULI_Z), (1, 1, -lam * PAULI_X), (3, 1, I2)])
    return _chain(first, lambda i: mid, last, n)


def _two_body_chain(n, d, sx, sy, sz, onsite=None, couplings=None):
    Id = np.eye(d, dtype=complex)

    def js(i):
        if couplings is None:
            return sx, sy, sz
        J, D = couplings[i]
        return J * sx, J * sy, J * D * sz

    def first():
        a, b, c = js(0)
        L = [(1, 1, Id), (1, 2, a), (1, 3, b), (1, 4, c)]
        if onsite is not None:
            L.append((1, 5, onsite))
        return construct_operator_site(d, 1, 5, L)

    def mid(i):
        a, b, c = js(i)
        L = [(1, 1, Id), (1, 2, a), (1, 3, b), (1, 4, c), (2, 5, sx), (3, 5, sy), (4, 5, sz), (5, 5, Id)]
        if onsite is not None:
            L.append((1, 5, onsite))
        return construct_operator_site(d, 5, 5, L)

    L = [(2, 1, sx), (3, 1, sy), (4, 1, sz), (5, 1, Id)]
    if onsite is not None:
        L.append((1, 1, onsite))
    last = construct_operator_site(d, 5, 1, L)
    return _chain(first(), mid, last, n)


def heisenberg(n):
    """H = sum (X_i X_{i+1} + Y_i Y_{i+1} + Z_i Z_{i+1}), MPO bond dimension 5."""
    return _two_body_chain(n, 2, PAULI_X, PAULI_Y, PAULI_Z)


def spin1_matrices():
    s = 1.0 / np.sqrt(2.0)
    sx = np.array([[0, s, 0], [s, 0, s], [0, s, 0]], dtype=complex)
    sy = np.array([[0, -1j * s, 0], [1j * s, 0, -1j * s], [0, 1j * s, 0]], dtype=complex)
    sz = np.diag([1.0, 0.0, -1.0]).astype(complex)
    return sx, sy, sz


def heisenberg_spin1(n, D=0.5):
    """H = sum S_i . S_{i+1} + D sum (S^z_i)^2 for spin 1 (d=3)."""
    sx, sy, sz = spin1_matrices()
    return _two_body_chain(n, 3, sx, sy, sz, onsite=D * (sz @ sz))


def xxz_random(n, rng):
    """H = sum_i J_i (X X + Y Y + Delta_i Z Z), J_i ~ U[0.5,1.5], Delta_i ~ U[0,2]."""
    coup = [(rng.uniform(0.5, 1.5), rng.uniform(0.0, 2.0)) for _ in range(n)]
    return _two_body_chain(n, 2, PAULI_X, PAULI_Y, PAULI_Z, couplings=coup)


def external_field(n, field):
    """constructExternalFieldOperator (operators.cpp:25-81): sum_i field_i."""
    field = np.asarray(field, dtype=complex)
    d = field.shape[0]
    Id = np.eye(d, dtype=complex)
    if n == 1:
        return [construct_operator_site(d, 1, 1, [(1, 1, field)])]
    first = construct_operator_site(d, 1, 2, [(1, 1, Id), (1, 2, field)])
    mid = construct_operator_site(d, 2, 2, [(1, 1, Id), (1, 2, field), (2, 2, Id)])
    last = construct_operator_site(d, 2, 1, [(1, 1, field), (2, 1, Id)])
    return _chain(first, lambda i: mid, last, n)
