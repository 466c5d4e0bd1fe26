"""MPO builders for the reference operator and the synthetic workloads.

TEST INFRASTRUCTURE and input generation.  Each builder returns a list of
``driver.OperatorSite`` in the reference's layout (``operators.cpp:83-112``):
links are (from, to, M) with M the row-major d x d matrix applied to the
physical index, stored column-major so that W(o1,o2) = M[o2][o1].

* ``transverse_ising_reference``: the reference's own TFIM
  H = sum Z_i + lambda sum X_i X_{i+1} (operators.cpp:114-165).
* ``transverse_ising_ferro``: H = -sum Z_i Z_{i+1} - lambda sum X_i with the
  3-state automaton 1->1 I, 1->2 Z, 2->3 -Z, 1->3 -lambda X, 3->3 I.
* ``heisenberg``: H = sum (X X + Y Y + Z Z) (D=5 automaton).
* ``heisenberg_spin1``: H = sum S.S + D sum (S^z)^2, d=3 (D=5 automaton).
* ``xxz_random``: H = sum_i J_i (X X + Y Y + Delta_i Z Z) per bond i.
"""
from __future__ import annotations

import numpy as np

from .driver import make_operator_site

I2 = np.eye(2, dtype=complex)
X = np.array([[0, 1], [1, 0]], dtype=complex)
Y = np.array([[0, -1j], [1j, 0]], dtype=complex)
Z = np.array([[1, 0], [0, -1]], dtype=complex)


def _chain(first, middle, last, n):
    return [first] + [middle(i) for i in range(1, n - 1)] + [last]


def transverse_ising_reference(n, lam):
    """operators.cpp:114-165."""
    assert n > 1
    X2 = lam * X
    first = make_operator_site(2, 1, 3, [(1, 1, I2), (1, 2, X), (1, 3, Z)])
    mid = make_operator_site(2, 3, 3, [(1, 1, I2), (1, 2, X), (2, 3, X2), (1, 3, Z), (3, 3, I2)])
    last = make_operator_site(2, 3, 1, [(1, 1, Z), (2, 1, X2), (3, 1, I2)])
    return _chain(first, lambda i: mid, last, n)


def transverse_ising_ferro(n, lam):
    """H = -sum Z_i Z_{i+1} - lam sum X_i; first site keeps from=1 rows, the
    last site maps automaton state 3 to 1."""
    assert n > 1
    first = make_operator_site(2, 1, 3, [(1, 1, I2), (1, 2, Z), (1, 3, -lam * X)])
    mid = make_operator_site(2, 3, 3, [(1, 1, I2), (1, 2, Z), (2, 3, -Z), (1, 3, -lam * X), (3, 3, I2)])
    last = make_operator_site(2, 3, 1, [(2, 1, -Z), (1, 1, -lam * X), (3, 1, I2)])
    return _chain(first, lambda i: mid, last, n)


def _heis_like(n, d, sx, sy, sz, onsite=None, couplings=None):
    """D=5 automaton 1->1 I, 1->{2,3,4} J{Sx,Sy,Delta Sz}, {2,3,4}->5 {Sx,Sy,Sz},
    5->5 I, optional 1->5 on-site term."""
    Id = np.eye(d, dtype=complex)

    def jterms(i):
        if couplings is None:
            return sx, sy, sz
        J, Dz = couplings[i]
        return J * sx, J * sy, J * Dz * sz

    def links_first():
        a, b, c = jterms(0)
        L = [(1, 1, Id), (1, 2, a), (1, 3, b), (1, 4, c)]
        if onsite is not None:
            L.append((1, 5, onsite))
        return make_operator_site(d, 1, 5, L)

    def links_mid(i):
        a, b, c = jterms(i)
        L = [(1, 1, Id), (1, 2, a), (1, 3, b), (1, 4, c), (2, 5, sx), (3, 5, sy), (4, 5, sz), (5, 5, Id)]
        if onsite is not None:
            L.append((1, 5, onsite))
        return make_operator_site(d, 5, 5, L)

    L = [(2, 1, sx), (3, 1, sy), (4, 1, sz), (5, 1, Id)]
    if onsite is not None:
        L.append((1, 1, onsite))
    last = make_operator_site(d, 5, 1, L)
    return _chain(links_first(), links_mid, last, n)


def heisenberg(n):
    """H = sum_i (X_i X_{i+1} + Y_i Y_{i+1} + Z_i Z_{i+1})."""
    return _heis_like(n, 2, X, Y, Z)


def spin1_matrices():
    s = 1.0 / np.sqrt(2.0)
    sx = np.array([[0, s, 0], [s, 0, s], [0, s, 0]], dtype=complex)
    sy = np.array([[0, -1j * s, 0], [1j * s, 0, -1j * s], [0, 1j * s, 0]], dtype=complex)
    sz = np.diag([1.0, 0.0, -1.0]).astype(complex)
    return sx, sy, sz


def heisenberg_spin1(n, D=0.5):
    """H = sum S_i . S_{i+1} + D sum (S^z_i)^2 (spin 1)."""
    sx, sy, sz = spin1_matrices()
    return _heis_like(n, 3, sx, sy, sz, onsite=D * (sz @ sz))


def xxz_random(n, rng):
    """H = sum_i J_i (X X + Y Y + Delta_i Z Z), J_i ~ U[0.5,1.5], Delta_i ~ U[0,2]."""
    coup = [(rng.uniform(0.5, 1.5), rng.uniform(0.0, 2.0)) for _ in range(n)]
    return _heis_like(n, 2, X, Y, Z, couplings=coup)


# ---------------------------------------------------------------------------
# YAML in the reference's input format (README:27-187, yaml.cpp:169-271)
# ---------------------------------------------------------------------------

def _yaml_complex(z):
    z = complex(z)
    if z.imag == 0:
        return repr(float(z.real))
    return "[%r, %r]" % (float(z.real), float(z.imag))


def to_yaml(ops):
    """Emit the operator as reference-format YAML (paths/sequence form)."""
    uniq = []
    seq = []
    for o in ops:
        for k, u in enumerate(uniq):
            if u is o:
                seq.append(k + 1)
                break
        else:
            uniq.append(o)
            seq.append(len(uniq))
    out = ["sites:"]
    for o in uniq:
        out.append("  - physical dimension: %d" % o.d)
        out.append("    left dimension: %d" % o.cl)
        out.append("    right dimension: %d" % o.cr)
        out.append("    matrices:")
        for n in range(o.nnz):
            M = o.W[:, :, n].T
            out.append("      - from: %d" % o.idx[0, n])
            out.append("        to: %d" % o.idx[1, n])
            out.append("        data: [%s]" % ", ".join(_yaml_complex(z) for z in M.ravel()))
    out.append("sequence: [%s]" % ", ".join(str(s) for s in seq))
    return "\n".join(out) + "\n"
