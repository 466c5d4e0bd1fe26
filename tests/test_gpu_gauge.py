"""GPU parity: gauge moves, bandwidth growth, random sites, projector sites.

The Level-0 gauge entry points return the reference's exact polar factor
(core.f95:2708-2960: U V^H of the SVD, the neighbour absorbing U S U^H), so
their outputs are compared element-wise with the oracle's zgesdd-based
moves (1e-10 relative: the polar factor of these random sites is
conditioned to ~1e3).  The device chain's Householder-QR gauge (selected
with nc_set_level0_gauge(0)) is compared through the gauge-invariant
quantities the reference's own tests use (tests/states.cpp,
tests/chain.cpp:143-169): the contracted two-site tensor, orthonormality of
the normalised site, and the state itself.  Tolerance 1e-12 relative.
"""
import ctypes as ct
import numpy as np
import pytest

from gpu_util import rand_c, rel_err
from oracle import core

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import nutcracker_b200
    return nutcracker_b200


def pair(A, B):
    """Two-site tensor sum_m A(m,l,s) B(r,m,t) -> (l,s,r,t)."""
    return np.einsum("mls,rmt->lsrt", A, B)


def left_normal_err(S):
    br, bl, d = S.shape
    M = np.reshape(S, (br, bl * d), order="F")
    return np.abs(M @ M.conj().T - np.eye(br)).max()


def right_normal_err(S):
    br, bl, d = S.shape
    M = np.reshape(np.transpose(S, (1, 0, 2)), (bl, br * d), order="F")
    return np.abs(M @ M.conj().T - np.eye(bl)).max()


DIMS = [(1, 2, 2, 2, 2), (2, 4, 8, 2, 2), (3, 5, 4, 2, 3), (16, 32, 16, 2, 2), (40, 60, 33, 2, 2),
        (100, 200, 100, 2, 2), (256, 300, 256, 2, 2), (120, 250, 250, 3, 3)]


@pytest.mark.parametrize("dims", DIMS, ids=lambda d: "x".join(map(str, d)))
def test_norm_denorm_going_right(nb, dims):
    bl, bm, br, dl, dr = dims
    if bl * dl < bm:
        pytest.skip("not normalisable")
    rng = np.random.default_rng(sum(dims))
    A = rand_c(rng, (bm, bl, dl)); B = rand_c(rng, (br, bm, dr))
    info, nA, dB = nb.Core.norm_denorm_going_right(bl, bm, br, dl, dr, A, B)
    assert info == 0
    assert left_normal_err(nA) < 1e-12
    assert rel_err(pair(nA, dB), pair(A, B)) < 1e-12
    # the reference's polar move, element by element
    _, rA, rB = core.norm_denorm_going_right(bl, bm, br, dl, dr, A, B)
    assert rel_err(pair(nA, dB), pair(rA, rB)) < 1e-12
    assert rel_err(nA, rA) < 1e-10
    assert rel_err(dB, rB) < 1e-10


@pytest.mark.parametrize("dims", DIMS, ids=lambda d: "x".join(map(str, d)))
def test_norm_denorm_going_left(nb, dims):
    bl, bm, br, dl, dr = dims
    if br * dr < bm:
        pytest.skip("not normalisable")
    rng = np.random.default_rng(7 + sum(dims))
    A = rand_c(rng, (bm, bl, dl)); B = rand_c(rng, (br, bm, dr))
    info, dA, nB = nb.Core.norm_denorm_going_left(bl, bm, br, dl, dr, A, B)
    assert info == 0
    assert right_normal_err(nB) < 1e-12
    assert rel_err(pair(dA, nB), pair(A, B)) < 1e-12
    _, rA, rB = core.norm_denorm_going_left(bl, bm, br, dl, dr, A, B)
    assert rel_err(dA, rA) < 1e-10
    assert rel_err(nB, rB) < 1e-10


@pytest.mark.parametrize("dims", [(8, 12, 3), (40, 30, 2), (64, 128, 2), (300, 200, 3)],
                         ids=lambda d: "x".join(map(str, d)))
def test_norm_for_left_right_polar(nb, dims):
    """core.f95:2880-2960: the polar factor alone, element by element."""
    br, bl, d = dims
    rng = np.random.default_rng(br + 3 * bl)
    S = rand_c(rng, (br, bl, d))
    if bl * d >= br:
        info, got = nb.Core.norm_for_left(br, bl, d, S)
        assert info == 0
        assert rel_err(got, core.norm_for_left(br, bl, d, S)[1]) < 1e-10
    if br * d >= bl:
        info, got = nb.Core.norm_for_right(br, bl, d, S)
        assert info == 0
        assert rel_err(got, core.norm_for_right(br, bl, d, S)[1]) < 1e-10


def test_qr_gauge_option(nb):
    """nc_set_level0_gauge(0): the device chain's QR gauge, same state."""
    bl, bm, br, dl, dr = 64, 100, 64, 2, 2
    rng = np.random.default_rng(5)
    A = rand_c(rng, (bm, bl, dl)); B = rand_c(rng, (br, bm, dr))
    assert nb.lib.nc_set_level0_gauge(ct.c_int(0)) == 0
    try:
        info, nA, dB = nb.Core.norm_denorm_going_right(bl, bm, br, dl, dr, A, B)
    finally:
        assert nb.lib.nc_set_level0_gauge(ct.c_int(1)) == 0
    assert info == 0
    _, rA, rB = core.norm_denorm_going_right(bl, bm, br, dl, dr, A, B)
    assert left_normal_err(nA) < 1e-12
    assert rel_err(pair(nA, dB), pair(rA, rB)) < 1e-12
    assert rel_err(nA, rA) > 1e-3   # a different gauge


def test_rank_deficient_gauge(nb):
    """A site of rank 3 < bm still yields an exactly left-normalised factor."""
    rng = np.random.default_rng(5)
    bl, bm, br, d = 20, 16, 16, 2
    U = rand_c(rng, (bm, 3)); V = rand_c(rng, (3, bl * d))
    A = np.asfortranarray(np.reshape(U @ V, (bm, bl, d), order="F"))
    B = rand_c(rng, (br, bm, d))
    info, nA, dB = nb.Core.norm_denorm_going_right(bl, bm, br, d, d, A, B)
    assert info == 0 and left_normal_err(nA) < 1e-12
    assert rel_err(pair(nA, dB), pair(A, B)) < 1e-12


def test_norm_for_left_right(nb):
    rng = np.random.default_rng(9)
    S = rand_c(rng, (12, 10, 2))
    info, L = nb.Core.norm_for_left(12, 10, 2, S)
    assert info == 0 and left_normal_err(L) < 1e-12
    # same row space as the reference's polar factor
    _, Lr = core.norm_for_left(12, 10, 2, S)
    P = lambda X: np.reshape(X, (12, 20), order="F").conj().T @ np.reshape(X, (12, 20), order="F")
    assert rel_err(P(L), P(Lr)) < 1e-12
    S = rand_c(rng, (10, 12, 2))
    info, R = nb.Core.norm_for_right(10, 12, 2, S)
    assert info == 0 and right_normal_err(R) < 1e-12


@pytest.mark.parametrize("dims", [(2, 2, 4, 2, 2, 4), (4, 6, 8, 2, 2, 8), (16, 20, 32, 2, 2, 32), (9, 9, 9, 3, 3, 20)])
def test_increase_bandwidth_between(nb, dims):
    bl, bm, br, dl, dr, nbm = dims
    rng = np.random.default_rng(sum(dims))
    A = rand_c(rng, (bm, bl, dl)); B = rand_c(rng, (br, bm, dr))
    info, oA, oB = nb.Core.increase_bandwidth_between(bl, bm, br, dl, dr, nbm, A, B)
    assert info == 0 and oA.shape == (nbm, bl, dl) and oB.shape == (br, nbm, dr)
    assert right_normal_err(oB) < 1e-12
    assert rel_err(pair(oA, oB), pair(A, B)) < 1e-12


def test_random_sites(nb):
    S = nb.Core.rand_norm_state_site_tensor(8, 16, 2)
    assert right_normal_err(S) < 1e-12
    T = nb.Core.rand_unnorm_state_site_tensor(8, 16, 2)
    assert abs(np.linalg.norm(T) - 1) < 1e-14
    U = nb.Core.rand_unnorm_state_site_tensor(8, 16, 2)
    assert rel_err(T, U) > 0.1  # fresh draws


def test_form_norm_overlap_tensors(nb):
    rng = np.random.default_rng(12)
    bl, bm, br, dl, dr = 4, 8, 6, 2, 2
    S1 = rand_c(rng, (bm, bl, dl))
    _, S2 = core.norm_for_right(br, bm, dr, rand_c(rng, (br, bm, dr)))
    lno, uno, dS2, rno = nb.Core.form_norm_overlap_tensors(bl, bm, br, dl, dr, S1, S2)
    rl, ru, rd, rr = core.form_norm_overlap_tensors(bl, bm, br, dl, dr, S1, S2)
    assert rel_err(uno, ru) == 0 and rel_err(rno, rr) == 0
    # the left-normalised overlap site and the denormalised site 2 carry the same pair
    back = lambda O: np.conj(np.transpose(O, (2, 0, 1)))  # overlap (bl,d,br) -> state (br,bl,d)
    assert rel_err(pair(back(lno), dS2), pair(back(rl), rd)) < 1e-12
    # with the exact polar factor, element by element
    assert rel_err(lno, rl) < 1e-10 and rel_err(dS2, rd) < 1e-10


@pytest.mark.parametrize("direction", [1, -1])
def test_gauge_move_dev_matches_host_entry(nb, direction):
    """nc_gauge_move_dev (device pointers, the chain's QR gauge) gives the host
    entry points' results in their QR mode (nc_set_level0_gauge(0)) bit for
    bit, and leaves its inputs unchanged."""
    import ctypes as ct

    import torch

    bl, bm, br, dl, dr = 256, 300, 256, 2, 2
    rng = np.random.default_rng(5 + direction)
    A = rand_c(rng, (bm, bl, dl)); B = rand_c(rng, (br, bm, dr))
    assert nb.lib.nc_set_level0_gauge(ct.c_int(0)) == 0
    try:
        if direction > 0:
            _, wantA, wantB = nb.Core.norm_denorm_going_right(bl, bm, br, dl, dr, A, B)
        else:
            _, wantA, wantB = nb.Core.norm_denorm_going_left(bl, bm, br, dl, dr, A, B)
    finally:
        assert nb.lib.nc_set_level0_gauge(ct.c_int(1)) == 0
    dA = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    dB = torch.from_numpy(B.ravel(order="F").copy()).cuda()
    oA, oB = torch.empty_like(dA), torch.empty_like(dB)
    torch.cuda.synchronize()
    st = nb.lib.nc_gauge_move_dev(direction, bl, bm, br, dl, dr, *[ct.c_void_p(t.data_ptr()) for t in (dA, dB, oA, oB)])
    assert st == 0, nb.lib.nc_last_error()
    assert nb.lib.nc_synchronize() == 0
    gotA = oA.cpu().numpy().reshape(A.shape, order="F")
    gotB = oB.cpu().numpy().reshape(B.shape, order="F")
    assert np.array_equal(gotA, wantA) and np.array_equal(gotB, wantB)
    assert np.array_equal(dA.cpu().numpy(), A.ravel(order="F"))
    assert np.array_equal(dB.cpu().numpy(), B.ravel(order="F"))
