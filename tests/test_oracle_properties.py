"""Properties of the CPU oracle's routines against independent dense
formulations (CPU only).

The reference tests each Fortran routine against an einsum-style contractor
and against its defining properties (tests/python/test.py: the contraction
stages, contract_sos_left/right, contract_vs_left/right,
form_overlap_vector, compute_expectation, the gauge moves, the projector
algebra, the random and bandwidth-growth tensors).  The same properties are
checked here for the oracle's restatements (oracle/core.py), with the dense
objects built independently: the Hamiltonian as a sum of Kronecker products
over the MPO's automaton paths (oracle/ed.py) and the state as a dense vector
contracted site by site.  These pin the oracle beyond the reference's
known-answer vectors (test_oracle_kats.py): a chain of environment updates
must give <psi|H|psi>, a chain of overlap updates <P|psi>, a gauge move must
leave the state unchanged.
"""
import numpy as np
import pytest

from oracle import core, ed, mpo

TOL = 1e-11


def _rc(rng, *shape):
    return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


def _random_mps(rng, dims, phys):
    return [_rc(rng, dims[i + 1], dims[i], phys[i]) for i in range(len(phys))]


OPERATORS = {
    "heisenberg_N5": lambda rng: mpo.heisenberg(5),
    "transverse_ising_N6": lambda rng: mpo.transverse_ising_ferro(6, 0.7),
    "spin1_N4": lambda rng: mpo.heisenberg_spin1(4, 0.5),
    "xxz_random_N5": lambda rng: mpo.xxz_random(5, rng),
}


def _bonds(phys, chi):
    n = len(phys)
    left = [1]
    for d in phys[:-1]:
        left.append(min(chi, left[-1] * d))
    right = [1]
    for d in reversed(phys[1:]):
        right.append(min(chi, right[-1] * d))
    right = list(reversed(right))
    return [min(a, b) for a, b in zip(left + [1], [1] + right)][:n + 1]


def _left_envs(ops, sites):
    """L_0 .. L_N: L_k is the left environment of site k."""
    envs = [np.ones((1, 1, 1), dtype=complex, order="F")]
    for o, S in zip(ops, sites):
        br, bl, d = S.shape
        envs.append(core.contract_sos_left(bl, br, o.cl, o.cr, d, envs[-1], o.idx, o.W, S))
    return envs


def _right_envs(ops, sites):
    """R_0 .. R_N: R_k is the right environment of site k-1 (R_N trivial)."""
    envs = [np.ones((1, 1, 1), dtype=complex, order="F")]
    for o, S in zip(reversed(ops), reversed(sites)):
        br, bl, d = S.shape
        envs.append(core.contract_sos_right(bl, br, o.cl, o.cr, d, envs[-1], o.idx, o.W, S))
    return list(reversed(envs))


def _close(a, b, tol=TOL):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(1.0, float(np.max(np.abs(b))))
    assert np.max(np.abs(a - b)) <= tol * scale, (a, b)


@pytest.mark.parametrize("name", sorted(OPERATORS))
def test_environment_chains_give_the_dense_energy(name):
    """core.f95:623-848, 1045-1161: the environment updates from either end,
    the expectation at every site and at every bond all equal <psi|H|psi> of
    the dense Hamiltonian and dense state."""
    rng = np.random.default_rng(11)
    ops = OPERATORS[name](rng)
    phys = [o.d for o in ops]
    sites = _random_mps(rng, _bonds(phys, 3), phys)
    v = ed.mps_to_dense(sites)
    want = np.vdot(v, ed.mpo_to_matrix(ops) @ v)
    L, R = _left_envs(ops, sites), _right_envs(ops, sites)
    _close(L[-1].ravel()[0], want)
    _close(R[0].ravel()[0], want)
    for k, (o, S) in enumerate(zip(ops, sites)):
        br, bl, d = S.shape
        _close(core.compute_expectation(bl, br, o.cl, o.cr, d, L[k], S, o.idx, o.W, R[k + 1]), want)
        b, c = L[k].shape[0], L[k].shape[2]
        _close(core.contract_expectation_boundaries(b, c, L[k], R[k]), want)


@pytest.mark.parametrize("name", sorted(OPERATORS))
def test_effective_hamiltonian_at_every_site(name):
    """core.f95:532-621, 1090-1140, 2529-2556: at every site, <S|H_eff S> is
    the energy, the product equals the dense optimisation matrix times S, and
    that matrix is Hermitian for a Hermitian MPO."""
    rng = np.random.default_rng(12)
    ops = OPERATORS[name](rng)
    phys = [o.d for o in ops]
    sites = _random_mps(rng, _bonds(phys, 3), phys)
    v = ed.mps_to_dense(sites)
    want = np.vdot(v, ed.mpo_to_matrix(ops) @ v)
    L, R = _left_envs(ops, sites), _right_envs(ops, sites)
    for k, (o, S) in enumerate(zip(ops, sites)):
        br, bl, d = S.shape
        y = core.apply_heff(bl, br, o.cl, o.cr, d, L[k], o.idx, o.W, R[k + 1], S)
        _close(np.vdot(S.ravel(order="F"), np.asarray(y).ravel(order="F")), want)
        M = core.compute_optimization_matrix(bl, br, o.cl, o.cr, d, L[k], o.idx, o.W, R[k + 1])
        _close(M @ S.ravel(order="F"), np.asarray(y).ravel(order="F"))
        _close(M, M.conj().T)


def test_overlap_chains_give_the_dense_inner_product():
    """core.f95:850-1005, 3299-3313: overlap environments from either end and
    the overlap vector at every site all give <P|psi>."""
    rng = np.random.default_rng(13)
    phys = [2, 3, 2, 2, 3]
    dims = _bonds(phys, 4)
    sites, proj = _random_mps(rng, dims, phys), _random_mps(rng, dims, phys)
    want = np.vdot(ed.mps_to_dense(proj), ed.mps_to_dense(sites))
    ov = [core.form_overlap_site_tensor(P.shape[0], P.shape[1], P.shape[2], P) for P in proj]   # (bl, d, br)
    left = [np.ones((1, 1), dtype=complex, order="F")]
    for O, S in zip(ov, sites):
        br, bl, d = S.shape
        left.append(core.contract_vs_left(O.shape[0], O.shape[2], bl, br, d, left[-1], O, S))
    right = [np.ones((1, 1), dtype=complex, order="F")]
    for O, S in zip(reversed(ov), reversed(sites)):
        br, bl, d = S.shape
        right.append(core.contract_vs_right(O.shape[0], O.shape[2], bl, br, d, right[-1], O, S))
    right = list(reversed(right))
    _close(left[-1].ravel()[0], want)
    _close(right[0].ravel()[0], want)
    for k, (O, S) in enumerate(zip(ov, sites)):
        br, bl, d = S.shape
        vec = core.form_overlap_vector(O.shape[0], O.shape[2], bl, br, d, left[k], right[k + 1], O)
        # the overlap vector enters unconjugated: <P|psi> = sum ov * S
        _close(np.sum(np.asarray(vec) * S), want)


@pytest.mark.parametrize("bl,bm,br,dl,dr", [(2, 4, 3, 2, 2), (3, 5, 2, 3, 3), (1, 2, 4, 2, 2)])
def test_gauge_moves_keep_the_state_and_normalise(bl, bm, br, dl, dr):
    """core.f95:2708-2960: both moves leave the two-site tensor unchanged and
    make the moved-from site an isometry; norm_for_left/right give the
    closest isometry (the polar factor)."""
    rng = np.random.default_rng(14)
    A, B = _rc(rng, bm, bl, dl), _rc(rng, br, bm, dr)

    def theta(a, b):   # (l, s1, s2, r)
        return np.einsum("mls,rmt->lstr", a, b)

    info, nA, dB = core.norm_denorm_going_right(bl, bm, br, dl, dr, A, B)
    assert info == 0
    _close(theta(nA, dB), theta(A, B))
    a = nA.reshape(bm, bl * dl, order="F")
    _close(a @ a.conj().T, np.eye(bm))
    info, dA, nB = core.norm_denorm_going_left(bl, bm, br, dl, dr, A, B)
    assert info == 0
    _close(theta(dA, nB), theta(A, B))
    b = np.transpose(nB, (1, 0, 2)).reshape(bm, br * dr, order="F")
    _close(b @ b.conj().T, np.eye(bm))
    # polar factors: U V^H of the site's matrix, row-orthonormal
    S = _rc(rng, 3, 4, 2)
    info, nL = core.norm_for_left(3, 4, 2, S)
    U, _, Vh = np.linalg.svd(S.reshape(3, 8, order="F"), full_matrices=False)
    _close(nL.reshape(3, 8, order="F"), U @ Vh)
    S = _rc(rng, 4, 3, 2)
    info, nR = core.norm_for_right(4, 3, 2, S)
    m = np.transpose(nR, (1, 0, 2)).reshape(3, 8, order="F")
    _close(m @ m.conj().T, np.eye(3))


def test_gauge_move_inside_a_chain_keeps_the_dense_state():
    rng = np.random.default_rng(15)
    phys = [2, 2, 2, 2, 2]
    sites = _random_mps(rng, [1, 2, 4, 4, 2, 1], phys)
    want = ed.mps_to_dense(sites)
    moved = list(sites)
    for k in range(len(sites) - 1):
        br, bl, d = moved[k].shape
        brr = moved[k + 1].shape[0]
        _, moved[k], moved[k + 1] = core.norm_denorm_going_right(bl, br, brr, d, phys[k + 1], moved[k], moved[k + 1])
    _close(ed.mps_to_dense(moved), want)
    for k in range(len(sites) - 1, 0, -1):
        br, bl, d = moved[k].shape
        bll = moved[k - 1].shape[1]
        _, moved[k - 1], moved[k] = core.norm_denorm_going_left(bll, bl, br, phys[k - 1], d, moved[k - 1], moved[k])
    _close(ed.mps_to_dense(moved), want)


def test_random_sites_and_bandwidth_growth():
    """core.f95:2611-2671, 2962-3144: random sites are right-normalised or of
    unit norm; the growth isometry has orthonormal columns; growing a bond
    keeps the state and leaves the right site right-normalised."""
    rng = np.random.default_rng(16)
    S = core.rand_norm_state_site_tensor(4, 3, 2, rng)       # (br, bl, d)
    m = np.transpose(S, (1, 0, 2)).reshape(3, 8, order="F")
    _close(m @ m.conj().T, np.eye(3))
    S = core.rand_unnorm_state_site_tensor(4, 3, 2, rng)
    _close(np.vdot(S, S).real, 1.0)
    M = core.create_bandwidth_increase_matrix(3, 7, rng)      # (new_b, old_b)
    _close(M.conj().T @ M, np.eye(3))
    # a left-normalised A (bm, bl, dl) and a B (br, bm, dr); grow bm = 2 -> 4
    bl, bm, br, dl, dr, new_bm = 2, 2, 3, 2, 2, 4
    _, A, B = core.norm_denorm_going_right(bl, bm, br, dl, dr, _rc(rng, bm, bl, dl), _rc(rng, br, bm, dr))
    info, eA, eB = core.increase_bandwidth_between(bl, bm, br, dl, dr, new_bm, A, B, rng)
    assert info == 0 and eA.shape == (new_bm, bl, dl) and eB.shape == (br, new_bm, dr)
    _close(np.einsum("mls,rmt->lstr", eA, eB), np.einsum("mls,rmt->lstr", A, B))
    b = np.transpose(eB, (1, 0, 2)).reshape(new_bm, br * dr, order="F")
    _close(b @ b.conj().T, np.eye(new_bm))


@pytest.mark.parametrize("n,k,duplicate", [(12, 3, False), (10, 4, True), (9, 1, False)])
def test_projector_algebra(n, k, duplicate):
    """core.f95:464-530, 1266-1909: the overlap vectors o_i act unconjugated
    (o_i . x).  Projecting into the orthogonal space and back is an isometry
    onto {x : o_i . x = 0}; the filter is that projection; for independent
    vectors the overlap norm is |(o_i . x)_i|; a linearly dependent vector
    lowers the rank."""
    rng = np.random.default_rng(17 + n)
    O = _rc(rng, n, k)
    if duplicate:
        O[:, -1] = 2.0 * O[:, 0] - 0.5j * O[:, 1]
    refl, rank, tau, swaps = core.convert_vectors_to_reflectors(n, k, O)
    assert rank == (k - 1 if duplicate else k)
    orth = n - rank
    x = _rc(rng, n).ravel()
    y = core.project_into_orthogonal_space(n, k, rank, orth, refl, tau, swaps, x)
    assert y.shape == (orth,)
    back = core.unproject_from_orthogonal_space(n, k, rank, orth, refl, tau, swaps, y)
    _close(O.T @ back, np.zeros(k))                           # in the orthogonal space
    _close(np.linalg.norm(back), np.linalg.norm(y))           # isometry
    _close(core.project_into_orthogonal_space(n, k, rank, orth, refl, tau, swaps, back), y)
    f = core.filter_components_outside_orthog(n, k, rank, orth, refl, tau, swaps, x)
    _close(f, back)
    _close(core.filter_components_outside_orthog(n, k, rank, orth, refl, tau, swaps, f), f)   # idempotent
    # x - f lies in the span of conj(o_i): the removed part is orthogonal to f
    _close(np.vdot(f, x - f), 0.0)
    if rank == k:
        _close(core.compute_overlap_with_projectors(k, rank, refl, tau, swaps, n, x), np.linalg.norm(O.T @ x))
        _close(core.compute_overlap_with_projectors(k, rank, refl, tau, swaps, n, f), 0.0)
    else:
        # The reference's formula (core.f95:1321-1329) dots the stored columns
        # of the dependent vectors over all n rows, reflector data below the
        # diagonal included, so with dependent vectors it does not give the
        # overlap norm: it is not zero even for a vector in the orthogonal
        # space.  The oracle and the device both restate it as written.
        assert core.compute_overlap_with_projectors(k, rank, refl, tau, swaps, n, f) > 1e-3
    # the projected matrix is the compression of H onto the orthogonal space
    H = _rc(rng, n, n)
    H = H + H.conj().T
    Hp = core.project_matrix_into_orthog_space(n, k, rank, orth, refl, tau, swaps, H)
    basis = np.stack([core.unproject_from_orthogonal_space(n, k, rank, orth, refl, tau, swaps, e)
                      for e in np.eye(orth, dtype=complex)], axis=1)
    _close(Hp, basis.conj().T @ H @ basis)


def test_swaps_are_inverse():
    rng = np.random.default_rng(18)
    swaps = np.array([3, 2, 5, 5, 5], dtype=np.uint32)
    v = rng.standard_normal(5) + 0j
    w = v.copy()
    core.swap_inplace(swaps, w)
    core.unswap_inplace(swaps, w)
    np.testing.assert_array_equal(w, v)
