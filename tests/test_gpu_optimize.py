"""GPU parity: the site eigen-solve and projector algebra through the C-ABI.

Mirrors the reference's optimizer tests (tests/optimizer.cpp:22-138 and the
property tests of tests/python/test.py:878-1160): random Hermitian
environments and Hermitian MPO blocks, with and without projectors, checked
against the oracle (scipy ARPACK / LAPACK) and dense eigh of H_eff.

Tolerances: eigenvalues 1e-10 relative; eigenvectors compared up to phase,
1 - |<gpu|ref>| <= 1e-8 when the spectral gap is at least 1e-3 of the scale.
"""
import numpy as np
import pytest

from gpu_util import rand_c, rel_err
from kat_inputs import KATS
from oracle import core, driver, mpo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import nutcracker_b200
    return nutcracker_b200


def herm_env(rng, b, c):
    A = rand_c(rng, (b, b, c))
    return np.asfortranarray(0.5 * (A + np.conj(np.transpose(A, (1, 0, 2)))))


def herm_mpo(rng, cl, cr, d, nnz):
    idx = np.asfortranarray(np.stack([rng.integers(1, cl + 1, nnz), rng.integers(1, cr + 1, nnz)]).astype(np.uint32))
    B = rand_c(rng, (d, d, nnz))
    W = np.asfortranarray(0.5 * (B + np.conj(np.transpose(B, (1, 0, 2)))))
    return idx, W


def dense_ref(bl, br, cl, cr, d, L, idx, W, R, which, proj=None):
    H = core.compute_optimization_matrix(bl, br, cl, cr, d, L, idx, W, R)
    n = H.shape[0]
    if proj is not None:
        nproj, nrefl, orth, refl, tau, swaps = proj
        B = np.stack([core.unproject_from_orthogonal_space(n, nproj, nrefl, orth, refl, tau, swaps, e)
                      for e in np.eye(orth)], axis=1)
        Hp = B.conj().T @ H @ B
    else:
        B = np.eye(n)
        Hp = H
    w, V = np.linalg.eigh(0.5 * (Hp + Hp.conj().T))
    if which == "SR":
        k = 0
    elif which == "LR":
        k = len(w) - 1
    else:
        k = len(w) - 1 if abs(w[-1]) > abs(w[0]) else 0
    gap = min([abs(w[k] - x) for j, x in enumerate(w) if j != k] or [np.inf])
    return w[k], B @ V[:, k], gap, np.max(np.abs(w))


@pytest.mark.parametrize("case", KATS["optimizer_modes"]["cases"], ids=lambda c: c["mode"] + str(c["value"]))
def test_optimizer_modes_kat(nb, case):
    """tests/optimizer.cpp:71-138 through optimize_."""
    rng = np.random.default_rng(0)
    op = driver.make_operator_site(4, 1, 1, [(1, 1, np.diag(case["diagonal"]))])
    one = np.ones((1, 1, 1), complex, order="F")
    which = driver.MODES[case["mode"]][0]
    for _ in range(3):
        S = core.rand_unnorm_state_site_tensor(1, 1, 4, rng)
        info, iters, ev, res, normal = nb.Core.optimize(1, 1, 1, 1, 4, one, 1, op.idx, op.W, one, 0, 0, 4,
                                                        None, None, None, which, 0.0, 10000, S)
        assert info == 0 and iters == 0
        assert abs(ev.real - case["value"]) <= 1e-12 * abs(case["value"])
        v = res.ravel(order="F")
        assert np.all(np.abs(v[:3]) <= 1e-15) and abs(abs(v[3]) - 1) < 1e-12


@pytest.mark.parametrize("d", [1, 2, 3, 4])
def test_one_site_external_field(nb, d):
    """tests/optimizer.cpp:22-69: diag(1,...,1,-1) gives -1 on the last basis vector."""
    rng = np.random.default_rng(d)
    diag = np.ones(d); diag[-1] = -1
    op = driver.make_operator_site(d, 1, 1, [(1, 1, np.diag(diag))])
    one = np.ones((1, 1, 1), complex, order="F")
    S = core.rand_unnorm_state_site_tensor(1, 1, d, rng)
    info, iters, ev, res, normal = nb.Core.optimize(1, 1, 1, 1, d, one, 1, op.idx, op.W, one, 0, 0, d,
                                                    None, None, None, "SR", 0.0, 10000, S)
    assert info == 0 and iters == 0 and abs(ev.real + 1) < 1e-12
    v = res.ravel(order="F")
    assert np.all(np.abs(v[:-1]) <= 1e-15) and abs(abs(v[-1]) - 1) < 1e-12


SHAPES = [(1, 2, 1, 2, 2, 3), (2, 2, 2, 3, 2, 5), (3, 4, 2, 2, 3, 4), (4, 4, 3, 3, 2, 6),
          (5, 7, 4, 3, 2, 8), (8, 6, 5, 5, 3, 10), (10, 10, 5, 5, 4, 12), (9, 10, 10, 10, 2, 20)]


@pytest.mark.parametrize("which", ["SR", "LR", "LM"])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_optimize_random_hermitian(nb, shape, which):
    bl, br, cl, cr, d, nnz = shape
    rng = np.random.default_rng(abs(hash((shape, which))) % 2 ** 32)
    L = herm_env(rng, bl, cl); R = herm_env(rng, br, cr)
    idx, W = herm_mpo(rng, cl, cr, d, nnz)
    n = bl * br * d
    guess = rand_c(rng, (br, bl, d))
    info, iters, ev, res, normal = nb.Core.optimize(bl, br, cl, cr, d, L, nnz, idx, W, R, 0, 0, n,
                                                    None, None, None, which, 1e-12, 10000, guess)
    assert info == 0
    w, v, gap, scale = dense_ref(bl, br, cl, cr, d, L, idx, W, R, which)
    assert abs(ev.real - w) <= 1e-10 * max(abs(w), 1e-3 * scale)
    assert abs(normal - 1) < 1e-12
    if gap > 1e-3 * scale:
        ov = abs(np.vdot(v, res.ravel(order="F")))
        assert 1 - ov <= 1e-8


@pytest.mark.parametrize("nproj", [1, 2, 3])
@pytest.mark.parametrize("shape", [(3, 4, 2, 2, 2, 4), (6, 5, 3, 4, 2, 7), (8, 8, 5, 5, 2, 10)],
                         ids=lambda s: "x".join(map(str, s)))
def test_optimize_with_projectors(nb, shape, nproj):
    bl, br, cl, cr, d, nnz = shape
    rng = np.random.default_rng(nproj * 1000 + sum(shape))
    L = herm_env(rng, bl, cl); R = herm_env(rng, br, cr)
    idx, W = herm_mpo(rng, cl, cr, d, nnz)
    n = bl * br * d
    vecs = rand_c(rng, (n, nproj))
    refl, rank, tau, swaps = core.convert_vectors_to_reflectors(n, nproj, vecs)
    orth = n - rank
    y = rand_c(rng, (orth,))
    guess = core.unproject_from_orthogonal_space(n, nproj, min(n, nproj), orth, refl, tau, swaps, y)
    guess = np.asfortranarray(np.reshape(guess, (br, bl, d), order="F"))
    info, iters, ev, res, normal = nb.Core.optimize(bl, br, cl, cr, d, L, nnz, idx, W, R, nproj, min(n, nproj),
                                                    orth, refl, tau, swaps, "SR", 1e-12, 10000, guess)
    assert info == 0
    proj = (nproj, min(n, nproj), orth, refl, tau, swaps)
    w, v, gap, scale = dense_ref(bl, br, cl, cr, d, L, idx, W, R, "SR", proj)
    assert abs(ev.real - w) <= 1e-10 * max(abs(w), 1e-3 * scale)
    ov = core.compute_overlap_with_projectors(nproj, min(n, nproj), refl, tau, swaps, n, res)
    assert ov < 1e-12
    # oracle ARPACK path agrees too
    oinfo, _, oev, ores, _ = core.optimize(bl, br, cl, cr, d, L, idx, W, R, nproj, min(n, nproj), orth,
                                           refl, tau, swaps, "SR", 1e-12, 10000, guess)
    assert oinfo == 0 and abs(oev.real - ev.real) <= 1e-10 * max(abs(w), 1e-3 * scale)


def test_optimize_guess_in_projector_space(nb):
    """info 11 when the guess overlaps the projectors (core.f95:1976-1983)."""
    rng = np.random.default_rng(11)
    bl, br, cl, cr, d, nnz = 3, 3, 2, 2, 2, 3
    L = herm_env(rng, bl, cl); R = herm_env(rng, br, cr)
    idx, W = herm_mpo(rng, cl, cr, d, nnz)
    n = bl * br * d
    vecs = rand_c(rng, (n, 1))
    refl, rank, tau, swaps = core.convert_vectors_to_reflectors(n, 1, vecs)
    guess = np.asfortranarray(np.reshape(np.conj(vecs[:, 0]), (br, bl, d), order="F"))
    info = nb.Core.optimize(bl, br, cl, cr, d, L, nnz, idx, W, R, 1, 1, n - rank, refl, tau, swaps, "SR",
                            1e-12, 10000, guess)[0]
    assert info == 11
    info = nb.Core.optimize(bl, br, cl, cr, d, L, nnz, idx, W, R, 1, 1, n + 1, refl, tau, swaps, "SR",
                            1e-12, 10000, guess)[0]
    assert info == 5


def test_heisenberg_chi64_matches_arpack(nb):
    op = mpo.heisenberg(4)[1]
    chi = 64
    rng = np.random.default_rng(64)
    L = herm_env(rng, chi, 5); R = herm_env(rng, chi, 5)
    guess = rand_c(rng, (chi, chi, 2))
    n = chi * chi * 2
    info, iters, ev, res, normal = nb.Core.optimize(chi, chi, 5, 5, 2, L, op.nnz, op.idx, op.W, R, 0, 0, n,
                                                    None, None, None, "SR", 1e-12, 10000, guess)
    oinfo, _, oev, ores, _ = core.optimize(chi, chi, 5, 5, 2, L, op.idx, op.W, R, 0, 0, n, None, None, None,
                                           "SR", 1e-12, 10000, guess)
    assert info == 0 and oinfo == 0
    assert abs(ev.real - oev.real) <= 1e-10 * abs(oev)
    assert 1 - abs(np.vdot(ores, res)) <= 1e-8


@pytest.mark.parametrize("n,m", [(7, 1), (20, 3), (50, 4), (5, 5), (3, 4)])
def test_convert_vectors_to_reflectors(nb, n, m):
    rng = np.random.default_rng(n * 10 + m)
    vecs = rand_c(rng, (n, m))
    r0, rank0, t0, s0 = core.convert_vectors_to_reflectors(n, m, vecs)
    r1, rank1, t1, s1 = nb.Core.convert_vectors_to_reflectors(n, m, vecs)
    assert rank0 == rank1 and np.array_equal(s0, s1)
    assert rel_err(r1, r0) < 1e-12 and rel_err(t1, t0) < 1e-12
    x = rand_c(rng, (n,))
    k = min(n, m)
    orth = n - rank0
    if orth > 0:
        f0 = core.filter_components_outside_orthog(n, m, k, orth, r0, t0, s0, x)
        f1 = nb.Core.filter_components_outside_orthog(n, m, k, orth, r0, t0, s0, x)
        assert rel_err(f1, f0) < 1e-12
    o0 = core.compute_overlap_with_projectors(m, k, r0, t0, s0, n, x)
    o1 = nb.Core.compute_overlap_with_projectors(m, k, r0, t0, s0, n, x)
    assert abs(o1.real - o0) <= 1e-12 * max(1, o0) and o1.imag == 0


def test_convert_vectors_rank_deficient(nb):
    rng = np.random.default_rng(3)
    a = rand_c(rng, (12, 1))
    vecs = np.asfortranarray(np.concatenate([a, 2 * a, rand_c(rng, (12, 1))], axis=1))
    r0, rank0, t0, s0 = core.convert_vectors_to_reflectors(12, 3, vecs)
    r1, rank1, t1, s1 = nb.Core.convert_vectors_to_reflectors(12, 3, vecs)
    assert rank0 == rank1 == 2 and np.array_equal(s0, s1)
    x = rand_c(rng, (12,))
    f0 = core.filter_components_outside_orthog(12, 3, 3, 12 - rank0, r0, t0, s0, x)
    f1 = nb.Core.filter_components_outside_orthog(12, 3, 3, 12 - rank0, r1, t1, s1, x)
    assert rel_err(f1, f0) < 1e-10


def test_random_projector_matrix(nb):
    rank, refl, tau, swaps = nb.Core.random_projector_matrix(30, 3)
    assert rank == 3 and list(swaps) == [1, 2, 3]
    x = rand_c(np.random.default_rng(0), (30,))
    f = nb.Core.filter_components_outside_orthog(30, 3, 3, 27, refl, tau, swaps, x)
    assert nb.Core.compute_overlap_with_projectors(3, 3, refl, tau, swaps, 30, f).real < 1e-12
