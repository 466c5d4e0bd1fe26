"""C API (include/nutcracker.h): matrices, vectors, the operator compiler and
protobuf serialization, no GPU.

Compiled operators are decoded from their protobuf serialization with an
independent wire-format reader below (nutcracker.proto: OperatorBuffer), turned
into dense Hamiltonians by the oracle's MPO contraction and compared with the
same Hamiltonian assembled directly from Kronecker products.  The compiler's
bond dimensions and error messages follow compiler.hpp:444-1141.
"""
import struct

import numpy as np
import pytest

from oracle import ed

X = np.array([[0, 1], [1, 0]], dtype=complex)
Y = np.array([[0, -1j], [1j, 0]])
Z = np.diag([1.0, -1.0]).astype(complex)
I2 = np.eye(2, dtype=complex)


@pytest.fixture(scope="module")
def C():
    from nutcracker_b200 import capi
    return capi


# ---- independent protobuf reader (proto2 wire format) ----------------------
def _varint(b, p):
    v = s = 0
    while True:
        c = b[p]
        p += 1
        v |= (c & 0x7F) << s
        s += 7
        if not c & 0x80:
            return v, p


def _fields(b):
    p, out = 0, []
    while p < len(b):
        tag, p = _varint(b, p)
        f, w = tag >> 3, tag & 7
        if w == 0:
            v, p = _varint(b, p)
        elif w == 2:
            n, p = _varint(b, p)
            v, p = b[p:p + n], p + n
        elif w == 1:
            v, p = b[p:p + 8], p + 8
        else:
            raise AssertionError("unexpected wire type %d" % w)
        out.append((f, w, v))
    return out


def _packed_varints(b):
    p, out = 0, []
    while p < len(b):
        v, p = _varint(b, p)
        out.append(v)
    return out


class _Site:
    def __init__(self, d, cl, cr, idx, W):
        self.d, self.cl, self.cr, self.idx, self.W = d, cl, cr, idx, W

    @property
    def nnz(self):
        return self.W.shape[2]


def decode_operator(data):
    unique, seq = [], []
    for f, w, v in _fields(data):
        if f == 1:
            m = {ff: vv for ff, ww, vv in _fields(v)}
            nnz, d, cl, cr = m[1], m[2], m[3], m[4]
            vals = struct.unpack("<%dd" % (2 * nnz * d * d), m.get(5, b""))
            W = (np.array(vals[0::2]) + 1j * np.array(vals[1::2])).reshape((d, d, nnz), order="F")
            idx = np.array(_packed_varints(m.get(6, b"")), dtype=np.uint32).reshape((2, nnz), order="F")
            unique.append(_Site(d, cl, cr, idx, W))
        elif f == 2:
            seq += _packed_varints(v)
    return [unique[k] for k in seq], len(unique), seq


def kron_sum(n, terms):
    """sum over terms of products; a term is {site: matrix}."""
    H = 0
    for t in terms:
        P = np.eye(1)
        for s in range(n):
            P = np.kron(P, t.get(s, I2))
        H = H + P
    return H


def dense(C, op):
    sites, _, _ = decode_operator(op.serialize())
    return ed.mpo_to_matrix(sites), sites


def test_matrices_and_vectors(C):
    m = C.Matrix.new([[1, 2j], [3, 4]])
    assert np.array_equal(m.array(), [[1, 2j], [3, 4]])
    assert np.array_equal((m + C.Matrix.pauli("Y")).array(), np.array([[1, 2j], [3, 4]]) + Y)
    assert np.array_equal((2j * m).array(), 2j * np.array([[1, 2j], [3, 4]]))
    assert np.array_equal(C.Matrix.diagonal([1, 2, 3]).array(), np.diag([1, 2, 3]))
    for p, M in zip("IXYZ", [I2, X, Y, Z]):
        assert np.array_equal(C.Matrix.pauli(p).array(), M)
    v = C.Vector.new([1, 1j, 2])
    assert np.array_equal((v + 3 * C.Vector.basis(3, 2)).array(), [1, 1j, 5])
    from nutcracker_b200 import NutcrackerError
    with pytest.raises(NutcrackerError, match="out of range"):
        m.element(2, 0)
    with pytest.raises(NutcrackerError, match="different dimensions"):
        m + C.Matrix.diagonal([1, 2, 3])
    with pytest.raises(NutcrackerError):
        C.Vector.basis(2, 2)
    assert C.version() == ("1.0.0", [1, 0, 0])


@pytest.mark.parametrize("n", [1, 2, 5])
def test_transverse_ising_field(C, n):
    b = C.OperatorBuilder([2] * n)
    b.add_term(C.OperatorTerm.transverse_ising_field(C.Matrix.pauli("Z"), 0.3 * C.Matrix.pauli("X"),
                                                     C.Matrix.pauli("X")))
    H, sites = dense(C, b.compile())
    want = kron_sum(n, [{s: Z} for s in range(n)] + [{s: 0.3 * X, s + 1: X} for s in range(n - 1)])
    assert np.allclose(H, want, atol=1e-14)
    if n > 2:   # the automaton start / coupling / end: bond dimension 3 inside
        assert [s.cr for s in sites] == [3] * (n - 1) + [1]


def test_product_and_local_terms_and_scalars(C):
    n = 4
    b = C.OperatorBuilder([2] * n)
    b.add_product_term([C.Matrix.pauli(p) for p in "XYZX"])
    b.add_term(C.OperatorTerm.local_external_field(2, C.Matrix.pauli("Y")))
    b.add_term(C.OperatorTerm.local_neighbor_coupling_field(1, C.Matrix.pauli("Z"), C.Matrix.pauli("Z")))
    t = C.OperatorTerm.global_external_field(C.Matrix.pauli("X")) + \
        C.OperatorTerm.global_neighbor_coupling_field(C.Matrix.pauli("Y"), C.Matrix.pauli("Y"))
    b.add_term((0.5 - 0.25j) * t)   # scales both summands
    H, _ = dense(C, b.compile())
    c = 0.5 - 0.25j
    want = kron_sum(n, [{0: X, 1: Y, 2: Z, 3: X}, {2: Y}, {1: Z, 2: Z}] +
                    [{s: c * X} for s in range(n)] + [{s: c * Y, s + 1: Y} for s in range(n - 1)])
    assert np.allclose(H, want, atol=1e-14)


def test_mixed_dimensions(C):
    S1z = np.diag([1.0, 0, -1.0]).astype(complex)
    b = C.OperatorBuilder([2, 3, 2])
    b.add_product_term([C.Matrix.pauli("Z"), C.Matrix.new(S1z), C.Matrix.pauli("X")])
    b.add_term(C.OperatorTerm.local_external_field(1, C.Matrix.diagonal([1, 2, 3])))
    H, sites = dense(C, b.compile())
    assert [s.d for s in sites] == [2, 3, 2]
    want = np.kron(np.kron(Z, S1z), X) + np.kron(np.kron(I2, np.diag([1, 2, 3])), I2)
    assert np.allclose(H, want, atol=1e-14)
    assert b.dimension_of_site(1) == 3 and b.number_of_sites() == 3


def test_optimisation_shares_sites_and_serialization_round_trips(C):
    n = 8
    b = C.OperatorBuilder([2] * n)
    b.add_term(C.OperatorTerm.transverse_ising_field(C.Matrix.pauli("Z"), C.Matrix.pauli("X"), C.Matrix.pauli("X")))
    op = b.compile()
    data = op.serialize()
    sites, n_unique, seq = decode_operator(data)
    assert n_unique == 3 and seq == [0] + [1] * (n - 2) + [2]   # first, repeated middle, last; 0-based
    again = C.Operator.deserialize(data)
    assert again.serialize() == data


def test_unoptimised_compile_reports_signal_conflict(C):
    from nutcracker_b200 import NutcrackerError
    b = C.OperatorBuilder([2] * 4)
    b.add_term(C.OperatorTerm.transverse_ising_field(C.Matrix.pauli("Z"), C.Matrix.pauli("X"), C.Matrix.pauli("X")))
    with pytest.raises(NutcrackerError, match=r"The left signals at site 0, \[1,2,3\], do not match the right "
                                              r"signals of its left neighbor, \[1\]\."):
        b.compile(optimize=False)
    # the start and end loops reach every site, so unoptimised compilation
    # only works without them; a product term then compiles as it is
    b = C.OperatorBuilder([2] * 3)
    b.add_product_term([C.Matrix.pauli("Z")] * 3)
    with pytest.raises(NutcrackerError, match=r"site 0, \[1,2\]"):
        b.compile(optimize=False)
    H, _ = dense(C, b.compile(optimize=False, add_start_and_end_loops=False))
    assert np.allclose(H, np.kron(np.kron(Z, Z), Z))


@pytest.mark.parametrize("call,message", [
    (lambda C: C.OperatorBuilder([2] * 3).add_product_term([C.Matrix.pauli("Z")] * 2),
     "The number of sites in the argument (2) does not match the number of sites in the system (3).  [2 != 3]"),
    (lambda C: C.OperatorBuilder([2] * 3).add_term(C.OperatorTerm.local_external_field(3, C.Matrix.pauli("Z"))),
     "Site number 3 is too large because there are only 3 sites."),
    (lambda C: C.OperatorBuilder([2, 3]).add_term(C.OperatorTerm.local_external_field(1, C.Matrix.pauli("Z"))),
     "Attempted to add matrix which has dimension 2 to site number 1 which has dimension 3. (2 != 3)"),
])
def test_builder_errors(C, call, message):
    from nutcracker_b200 import NutcrackerError
    with pytest.raises(NutcrackerError) as e:
        call(C)
    assert message in str(e.value)


def test_deserialize_errors(C):
    from nutcracker_b200 import NutcrackerError
    b = C.OperatorBuilder([2] * 3)
    b.add_term(C.OperatorTerm.global_external_field(C.Matrix.pauli("Z")))
    data = b.compile().serialize()
    fields = _fields(data)
    sites = b"".join(bytes([0x0A]) + _len(v) + v for f, w, v in fields if f == 1)
    bad_seq = sites + bytes([0x12]) + _len(bytes([0, 5, 2])) + bytes([0, 5, 2])
    with pytest.raises(NutcrackerError, match="non-existent operator site number 5"):
        C.Operator.deserialize(bad_seq)
    with pytest.raises(NutcrackerError, match="No operator sites were specified."):
        C.Operator.deserialize(sites)
    with pytest.raises(NutcrackerError, match="truncated"):
        C.Operator.deserialize(data[:-3])


def _len(b):
    out, n = b"", len(b)
    while n >= 0x80:
        out += bytes([(n & 0x7F) | 0x80])
        n >>= 7
    return out + bytes([n])


def _enc(n):
    out = b""
    while n >= 0x80:
        out += bytes([(n & 0x7F) | 0x80])
        n >>= 7
    return out + bytes([n])


def _state_buffer(sites, norms=True):
    """StateBuffer (nutcracker.proto) from (d, bl, br, complex array) sites."""
    out = b""
    for k, (d, bl, br, A) in enumerate(sites):
        m = b""
        if norms:
            m += b"\x08" + _enc(0 if k == 0 else 2)
        m += b"\x10" + _enc(d) + b"\x18" + _enc(bl) + b"\x20" + _enc(br)
        raw = np.asarray(A, dtype=complex).ravel(order="F").view(np.float64).tobytes()
        m += b"\x2a" + _enc(len(raw)) + raw
        out += b"\x0a" + _enc(len(m)) + m
    return out


def test_state_buffer_round_trip_and_errors(C):
    from nutcracker_b200 import NutcrackerError
    rng = np.random.default_rng(4)
    sites = [(2, 1, 3, rng.normal(size=(3, 1, 2)) + 1j * rng.normal(size=(3, 1, 2))),
             (2, 3, 1, rng.normal(size=(1, 3, 2)))]
    data = _state_buffer(sites)
    assert C.State.deserialize(data).serialize() == data
    # fields of an unknown number are skipped, a missing normalisation is accepted
    st = C.State.deserialize(b"\x9a\x01\x02hi" + _state_buffer(sites, norms=False))
    assert st.serialize() == data
    with pytest.raises(NutcrackerError, match="does not match its dimensions"):
        C.State.deserialize(_state_buffer([(2, 1, 3, np.zeros((3, 1, 1)))]))
    with pytest.raises(NutcrackerError, match="state site dimensions do not match"):
        C.State.deserialize(_state_buffer([sites[0], (2, 2, 1, np.zeros((1, 2, 2)))]))
    with pytest.raises(NutcrackerError, match="at least one site"):
        C.State.deserialize(b"")


@pytest.mark.parametrize("seed", range(6))
def test_random_term_sets_compile_to_their_hamiltonian(C, seed):
    """Random sums of product, scaled local-field and neighbour-coupling terms on
    sites of mixed dimension: the compiled operator equals the sum of the terms'
    Kronecker products."""
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(2, 5))
    dims = [int(x) for x in rng.integers(2, 4, size=n)]

    def rmat(d):
        return rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))

    def kron_terms(terms):
        H = 0
        for t in terms:
            P = np.eye(1)
            for s in range(n):
                P = np.kron(P, t.get(s, np.eye(dims[s])))
            H = H + P
        return H

    b = C.OperatorBuilder(dims)
    terms = []
    for _ in range(int(rng.integers(1, 6))):
        kind = int(rng.integers(0, 3))
        if kind == 0:
            comps = [rmat(d) for d in dims]
            b.add_product_term([C.Matrix.new(m) for m in comps])
            terms.append(dict(enumerate(comps)))
        elif kind == 1:
            s = int(rng.integers(0, n))
            m = rmat(dims[s])
            c = complex(rng.normal(), rng.normal())
            b.add_term(c * C.OperatorTerm.local_external_field(s, C.Matrix.new(m)))
            terms.append({s: c * m})
        else:
            s = int(rng.integers(0, n - 1))
            ml, mr = rmat(dims[s]), rmat(dims[s + 1])
            b.add_term(C.OperatorTerm.local_neighbor_coupling_field(s, C.Matrix.new(ml), C.Matrix.new(mr)))
            terms.append({s: ml, s + 1: mr})
    H, sites = dense(C, b.compile())
    want = kron_terms(terms)
    assert np.allclose(H, want, atol=1e-12 * max(1.0, np.abs(want).max()))
    assert [s.d for s in sites] == dims


def test_heisenberg_from_bond_terms_compiles_to_bond_dimension_five(C):
    """Sum over bonds of XX + YY + ZZ, added bond by bond: merging equivalent
    signals leaves the minimal automaton (start, X, Y, Z, end)."""
    n = 6
    b = C.OperatorBuilder([2] * n)
    for s in range(n - 1):
        for p in "XYZ":
            b.add_term(C.OperatorTerm.local_neighbor_coupling_field(s, C.Matrix.pauli(p), C.Matrix.pauli(p)))
    H, sites = dense(C, b.compile())
    want = kron_sum(n, [{s: P, s + 1: P} for s in range(n - 1) for P in (X, Y, Z)])
    assert np.allclose(H, want, atol=1e-13)
    assert [s.cr for s in sites] == [4] + [5] * (n - 3) + [4, 1]
