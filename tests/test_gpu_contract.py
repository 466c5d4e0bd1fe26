"""GPU parity: sparse-MPO contractions through the C-ABI vs the CPU oracle.

Tolerance: FP64 (complex128) throughout; relative Frobenius error <= 1e-12
(the reductions run over at most a few thousand terms).  Known-answer cases
are integer-valued and must match exactly.
"""
import numpy as np
import pytest

from gpu_util import rand_c, random_mpo_site, rel_err
from kat_inputs import KATS, cplx, exp_boundary, operator_site, overlap_site, state_site
from oracle import core, mpo

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def nb():
    import nutcracker_b200
    return nutcracker_b200


def test_kat_contract_expectation_boundaries(nb):
    k = KATS["contract_expectation_boundaries"]
    L = exp_boundary(k["left"], k["c"])
    R = exp_boundary(k["right"], k["c"])
    assert nb.Core.contract_expectation_boundaries(L.shape[0], k["c"], L, R) == complex(*k["expected"])


@pytest.mark.parametrize("side", ["left", "right"])
def test_kat_contract_sos(nb, side):
    k = KATS["contract_sos_" + side]
    c0 = k["c_left"] if side == "left" else k["c_right"]
    E = exp_boundary(k["boundary"], c0)
    S = state_site(k["state"], k["state_left"], k["state_right"])
    idx, W, d = operator_site(k["indices"], k["matrices"], k["op_left"], k["op_right"])
    br, bl, _ = S.shape
    f = nb.Core.contract_sos_left if side == "left" else nb.Core.contract_sos_right
    got = f(bl, br, k["op_left"], k["op_right"], d, E, idx.shape[1], idx, W, S)
    np.testing.assert_array_equal(got.ravel(order="F"), cplx(k["expected"]))


def test_kat_contract_vs(nb):
    k = KATS["contract_vs_left"]
    P = overlap_site(k["overlap_site"], k["overlap_left"], k["overlap_right"])
    S = state_site(k["state"], k["state_left"], k["state_right"])
    Lov = np.asfortranarray(cplx(k["boundary"]).reshape((S.shape[1], P.shape[0]), order="F"))
    got = nb.Core.contract_vs_left(P.shape[0], P.shape[2], S.shape[1], S.shape[0], P.shape[1], Lov, P, S)
    np.testing.assert_array_equal(got.ravel(order="F"), cplx(k["expected"]))
    k = KATS["contract_vs_right"]
    P = overlap_site(k["overlap_site"], k["overlap_left"], k["overlap_right"])
    S = state_site(k["state"], k["state_left"], k["state_right"])
    Rov = np.asfortranarray(cplx(k["boundary"]).reshape((P.shape[2], S.shape[0]), order="F"))
    got = nb.Core.contract_vs_right(P.shape[0], P.shape[2], S.shape[1], S.shape[0], P.shape[1], Rov, P, S)
    np.testing.assert_array_equal(got.ravel(order="F"), cplx(k["expected"]))


SHAPES = [  # (bl, br, cl, cr, d, nnz)
    (1, 1, 1, 1, 1, 1), (1, 2, 1, 3, 2, 3), (2, 4, 3, 3, 2, 5), (3, 7, 2, 5, 3, 7),
    (17, 16, 5, 5, 2, 8), (33, 65, 4, 2, 4, 9), (64, 64, 5, 5, 2, 8), (130, 97, 3, 6, 3, 11),
]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_random_contractions_match_oracle(nb, shape):
    bl, br, cl, cr, d, nnz = shape
    rng = np.random.default_rng(hash(shape) % 2 ** 32)
    L = rand_c(rng, (bl, bl, cl)); R = rand_c(rng, (br, br, cr)); S = rand_c(rng, (br, bl, d))
    idx, W = random_mpo_site(rng, cl, cr, d, nnz)
    want = core.contract_sos_left(bl, br, cl, cr, d, L, idx, W, S)
    assert rel_err(nb.Core.contract_sos_left(bl, br, cl, cr, d, L, nnz, idx, W, S), want) < TOL
    want = core.contract_sos_right(bl, br, cl, cr, d, R, idx, W, S)
    assert rel_err(nb.Core.contract_sos_right(bl, br, cl, cr, d, R, nnz, idx, W, S), want) < TOL
    want = core.compute_expectation(bl, br, cl, cr, d, L, S, idx, W, R)
    got = nb.Core.compute_expectation(bl, br, cl, cr, d, L, S, nnz, idx, W, R)
    assert abs(got - want) <= TOL * max(abs(want), 1.0) * 10
    if bl * br * d <= 400:
        want = core.compute_optimization_matrix(bl, br, cl, cr, d, L, idx, W, R)
        assert rel_err(nb.Core.compute_optimization_matrix(bl, br, cl, cr, d, L, nnz, idx, W, R), want) < TOL


@pytest.mark.parametrize("dims", [(1, 1, 1, 1, 1), (3, 2, 4, 5, 2), (16, 17, 9, 33, 3), (70, 40, 64, 64, 2)])
def test_random_overlap_contractions_match_oracle(nb, dims):
    blo, bro, bln, brn, d = dims
    rng = np.random.default_rng(sum(dims))
    P = rand_c(rng, (blo, d, bro)); S = rand_c(rng, (brn, bln, d))
    Lov = rand_c(rng, (bln, blo)); Rov = rand_c(rng, (bro, brn))
    assert rel_err(nb.Core.contract_vs_left(blo, bro, bln, brn, d, Lov, P, S),
                   core.contract_vs_left(blo, bro, bln, brn, d, Lov, P, S)) < TOL
    assert rel_err(nb.Core.contract_vs_right(blo, bro, bln, brn, d, Rov, P, S),
                   core.contract_vs_right(blo, bro, bln, brn, d, Rov, P, S)) < TOL
    assert rel_err(nb.Core.form_overlap_vector(blo, bro, bln, brn, d, Lov, Rov, P),
                   core.form_overlap_vector(blo, bro, bln, brn, d, Lov, Rov, P)) < TOL
    assert rel_err(nb.Core.form_overlap_site_tensor(brn, bln, d, S),
                   core.form_overlap_site_tensor(brn, bln, d, S)) == 0.0


def test_exp_boundary_construction(nb):
    rng = np.random.default_rng(1)
    sb = rand_c(rng, (5,)); ob = rand_c(rng, (3,))
    np.testing.assert_allclose(nb.Core.construct_left_exp_boundary(5, 3, sb, ob),
                               core.construct_left_exp_boundary(5, 3, sb, ob), rtol=1e-15, atol=1e-15)
    np.testing.assert_allclose(nb.Core.construct_right_exp_boundary(5, 3, sb, ob),
                               core.construct_right_exp_boundary(5, 3, sb, ob), rtol=1e-15, atol=1e-15)


def test_heisenberg_interior_chi256(nb):
    """Full-width interior site of the Heisenberg MPO (d=2, D=5, nnz=8) at chi=256."""
    op = mpo.heisenberg(4)[1]
    chi = 256
    rng = np.random.default_rng(256)
    L = rand_c(rng, (chi, chi, 5)); R = rand_c(rng, (chi, chi, 5)); S = rand_c(rng, (chi, chi, 2))
    want = core.contract_sos_left(chi, chi, 5, 5, 2, L, op.idx, op.W, S)
    assert rel_err(nb.Core.contract_sos_left(chi, chi, 5, 5, 2, L, op.nnz, op.idx, op.W, S), want) < TOL
    want = core.contract_sos_right(chi, chi, 5, 5, 2, R, op.idx, op.W, S)
    assert rel_err(nb.Core.contract_sos_right(chi, chi, 5, 5, 2, R, op.nnz, op.idx, op.W, S), want) < TOL


def test_bad_operator_index_reports_error(nb):
    one = np.ones((1, 1, 1), complex, order="F")
    idx = np.array([[2], [1]], np.uint32)  # from=2 > cl=1
    W = np.ones((1, 1, 1), complex, order="F")
    with pytest.raises(nb.NutcrackerError):
        nb.Core.contract_sos_left(1, 1, 1, 1, 1, one, 1, idx, W, one)


def test_contract_matrix_left_and_extend_state_vector_fragment():
    """core.f95:1163-1234 restated in numpy: L' = M L M^H and the state-vector
    fragment extension of flat.cpp."""
    import ctypes as ct

    import nutcracker_b200 as nb
    from gpu_util import rand_c, rel_err

    u = lambda x: ct.byref(ct.c_uint32(x))
    p = lambda a: a.ctypes.data_as(ct.c_void_p)
    rng = np.random.default_rng(17)
    bl, br = 7, 5
    L, M = rand_c(rng, (bl, bl)), rand_c(rng, (br, bl))
    out = np.zeros((br, br), dtype=complex, order="F")
    nb.lib.contract_matrix_left_(u(bl), u(br), p(L), p(M), p(out))
    assert nb.lib.nc_last_status() == 0
    assert rel_err(out, M @ L @ M.conj().T) < 1e-13
    bm, br, dl, dr = 6, 4, 3, 2
    old, S = rand_c(rng, (bm, dl)), rand_c(rng, (br, bm, dr))
    new = np.zeros((br, dr, dl), dtype=complex, order="F")
    nb.lib.extend_state_vector_fragment_(u(bm), u(br), u(dl), u(dr), p(old), p(S), p(new))
    assert nb.lib.nc_last_status() == 0
    assert rel_err(new, np.einsum("rms,ma->rsa", S, old)) < 1e-13
    # the infinite-chain routine is exported but reports that it is unsupported
    z = np.zeros(8, dtype=complex)
    nb.lib.increase_bandwidth_with_environment_(u(1), u(1), u(2), u(2), p(z), p(z), p(z), p(z), p(z), p(z))
    assert nb.lib.nc_last_status() != 0
