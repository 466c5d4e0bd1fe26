"""C API on the GPU: the simple solvers and states (operator.cpp, state.cpp,
state_builder.cpp).  The transverse-Ising operator Sum Z + 0.1 Sum X X built
through the compiler at N=10 must give the energies the reference's tests pin
(tests/chain.cpp:300-305, 418-430) to float precision, its eigenvector states
must be orthonormal and reproduce their energies as expectation values, and
compiled states must match dense vectors assembled in numpy.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF = [-10.022510957077, -8.213705725703, -8.188197237172, -8.148553771957]


@pytest.fixture(scope="module")
def C():
    from nutcracker_b200 import capi
    return capi


def tfim(C, n=10, lam=0.1):
    b = C.OperatorBuilder([2] * n)
    b.add_term(C.OperatorTerm.transverse_ising_field(C.Matrix.pauli("Z"), lam * C.Matrix.pauli("X"),
                                                     C.Matrix.pauli("X")))
    return b.compile()


def test_simple_solve_matches_reference_energies(C):
    e = tfim(C).simple_solve(4)
    assert np.allclose(e, REF, rtol=1e-6)


def test_eigenvectors_are_orthonormal_and_give_their_energies(C):
    op = tfim(C)
    e, states = op.simple_solve(3, with_eigenvectors=True)
    assert np.allclose(e, REF[:3], rtol=1e-6)
    for i, si in enumerate(states):
        assert abs(si.overlap(si) - 1) < 1e-10
        assert abs(si.expectation(op) - REF[i]) < 1e-7 * abs(REF[i])
        for sj in states[:i]:
            assert abs(si.overlap(sj)) < 1e-6
    # a state survives serialization
    back = C.State.deserialize(states[1].serialize())
    assert abs(back.overlap(states[1]) - 1) < 1e-12


def _dense(vectors_per_site):
    v = np.ones(1)
    for a in vectors_per_site:
        v = np.kron(v, a)
    return v


def test_compiled_states_match_dense_vectors(C):
    n = 5
    up, down = C.Vector.basis(2, 0), C.Vector.basis(2, 1)
    plus = C.Vector.new([1, 1])
    # product state |+ + + + +>, then a W state and a one-site-different state
    prod = C.StateBuilder([2] * n).add_product_term([plus] * n).compile()
    w = C.StateBuilder([2] * n).add_term(C.StateTerm.w(up, down)).compile()
    one = C.StateBuilder([2] * n).add_term(C.StateTerm.product_with_one_site_different(2, up, down)).compile()
    e0, e1 = np.array([1, 0]), np.array([0, 1])
    d_prod = _dense([np.array([1, 1])] * n)
    d_w = sum(_dense([e1 if k == j else e0 for k in range(n)]) for j in range(n))
    d_one = _dense([e1 if k == 2 else e0 for k in range(n)])
    dens = [d_prod / np.linalg.norm(d_prod), d_w / np.linalg.norm(d_w), d_one]
    states = [prod, w, one]
    for i in range(3):
        for j in range(3):
            want = np.vdot(dens[i], dens[j])
            assert abs(states[i].overlap(states[j]) - want) < 1e-12, (i, j)
    # expectation of Sum Z: compiled operator against the dense vectors
    b = C.OperatorBuilder([2] * n)
    b.add_term(C.OperatorTerm.global_external_field(C.Matrix.pauli("Z")))
    op = b.compile()
    Zs = np.diag(np.array([sum(1 - 2 * ((idx >> (n - 1 - k)) & 1) for k in range(n)) for idx in range(2 ** n)]))
    for s, d in zip(states, dens):
        assert abs(s.expectation(op) - np.vdot(d, Zs @ d)) < 1e-12
