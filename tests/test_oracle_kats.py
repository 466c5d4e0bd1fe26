"""Pin the CPU oracle against the reference's own known answers.

Every expected value below comes from the reference's test sources, extracted
by ``tests/golden/make_golden.py`` into ``tests/golden/reference_kats.json``.
"""
import numpy as np
import pytest

from kat_inputs import KATS, cplx, exp_boundary, operator_site, overlap_site, state_site
from oracle import core, driver, ed, mpo


def test_contract_expectation_boundaries_kat():
    k = KATS["contract_expectation_boundaries"]
    L = exp_boundary(k["left"], k["c"])
    R = exp_boundary(k["right"], k["c"])
    got = core.contract_expectation_boundaries(L.shape[0], k["c"], L, R)
    assert got == complex(*k["expected"])


def test_contract_sos_left_kat():
    k = KATS["contract_sos_left"]
    L = exp_boundary(k["boundary"], k["c_left"])
    S = state_site(k["state"], k["state_left"], k["state_right"])
    idx, W, d = operator_site(k["indices"], k["matrices"], k["op_left"], k["op_right"])
    br, bl, _ = S.shape
    got = core.contract_sos_left(bl, br, k["op_left"], k["op_right"], d, L, idx, W, S)
    np.testing.assert_array_equal(got.ravel(order="F"), cplx(k["expected"]))


def test_contract_sos_right_kat():
    k = KATS["contract_sos_right"]
    R = exp_boundary(k["boundary"], k["c_right"])
    S = state_site(k["state"], k["state_left"], k["state_right"])
    idx, W, d = operator_site(k["indices"], k["matrices"], k["op_left"], k["op_right"])
    br, bl, _ = S.shape
    got = core.contract_sos_right(bl, br, k["op_left"], k["op_right"], d, R, idx, W, S)
    np.testing.assert_array_equal(got.ravel(order="F"), cplx(k["expected"]))


def test_contract_vs_left_kat():
    k = KATS["contract_vs_left"]
    P = overlap_site(k["overlap_site"], k["overlap_left"], k["overlap_right"])
    S = state_site(k["state"], k["state_left"], k["state_right"])
    Lov = np.asfortranarray(cplx(k["boundary"]).reshape((S.shape[1], P.shape[0]), order="F"))
    got = driver.contract_vs_left(Lov, P, S)
    np.testing.assert_array_equal(got.ravel(order="F"), cplx(k["expected"]))
    k2 = KATS["contract_vs_left_d2"]
    P = overlap_site(k2["overlap_site"], 1, 1)
    S = state_site(k2["state"], 1, 1)
    got = driver.contract_vs_left(np.ones((1, 1), complex), P, S)
    assert got[0, 0] == complex(*k2["expected"])


def test_contract_vs_right_kat():
    k = KATS["contract_vs_right"]
    P = overlap_site(k["overlap_site"], k["overlap_left"], k["overlap_right"])
    S = state_site(k["state"], k["state_left"], k["state_right"])
    Rov = np.asfortranarray(cplx(k["boundary"]).reshape((P.shape[2], S.shape[0]), order="F"))
    got = driver.contract_vs_right(Rov, P, S)
    np.testing.assert_array_equal(got.ravel(order="F"), cplx(k["expected"]))


def test_expectation_small_kats():
    one = np.ones((1, 1, 1), complex, order="F")
    idx = np.array([[1], [1]], np.uint32)
    W = np.array([1j], complex).reshape((1, 1, 1))
    S = np.ones((1, 1, 1), complex, order="F")
    assert core.compute_expectation(1, 1, 1, 1, 1, one, S, idx, W, one) == 1j
    Wz = np.asfortranarray(np.array([1, 0, 0, -1], complex).reshape((2, 2, 1), order="F"))
    for name, args in KATS["expectation_d2"]["cases"]:
        a, b, c = [complex(eval(t.replace("complex<double>", "complex"))) for t in
                   args.replace("complex<double>(0,1)", "1j").split(",")]
        S = np.asfortranarray(np.array([a, b]).reshape((1, 1, 2), order="F"))
        assert core.compute_expectation(1, 1, 1, 1, 2, one, S, idx, Wz, one) == c


def _random_case(rng, bl, br, cl, cr, d, nnz):
    L = core.F(rng.normal(size=(bl, bl, cl)) + 1j * rng.normal(size=(bl, bl, cl)))
    R = core.F(rng.normal(size=(br, br, cr)) + 1j * rng.normal(size=(br, br, cr)))
    S = core.F(rng.normal(size=(br, bl, d)) + 1j * rng.normal(size=(br, bl, d)))
    idx = np.asfortranarray(np.stack([rng.integers(1, cl + 1, nnz), rng.integers(1, cr + 1, nnz)]).astype(np.uint32))
    W = core.F(rng.normal(size=(d, d, nnz)) + 1j * rng.normal(size=(d, d, nnz)))
    return L, R, S, idx, W


def test_expectation_consistency():
    """tests/boundaries.cpp:468-548: site expectation == via left update == via right update."""
    rng = np.random.default_rng(5)
    for _ in range(10):
        cl, cr, bl, br, d, nnz = (int(x) for x in rng.integers(1, 6, 6))
        L, R, S, idx, W = _random_case(rng, bl, br, cl, cr, d, nnz)
        e = core.compute_expectation(bl, br, cl, cr, d, L, S, idx, W, R)
        Ln = core.contract_sos_left(bl, br, cl, cr, d, L, idx, W, S)
        Rn = core.contract_sos_right(bl, br, cl, cr, d, R, idx, W, S)
        e1 = core.contract_expectation_boundaries(br, cr, Ln, R)
        e2 = core.contract_expectation_boundaries(bl, cl, L, Rn)
        assert abs(e - e1) <= 1e-10 * abs(e) and abs(e - e2) <= 1e-10 * abs(e)


def test_optimization_matrix_matches_matvec():
    rng = np.random.default_rng(7)
    for _ in range(5):
        cl, cr, bl, br, d, nnz = (int(x) for x in rng.integers(1, 5, 6))
        L, R, S, idx, W = _random_case(rng, bl, br, cl, cr, d, nnz)
        H = core.compute_optimization_matrix(bl, br, cl, cr, d, L, idx, W, R)
        y = core.apply_heff(bl, br, cl, cr, d, L, idx, W, R, S)
        np.testing.assert_allclose(H @ S.ravel(order="F"), y.ravel(order="F"), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("case", KATS["optimizer_modes"]["cases"], ids=lambda c: c["mode"] + str(c["value"]))
def test_optimizer_modes_kat(case):
    """tests/optimizer.cpp:71-138."""
    rng = np.random.default_rng(0)
    op = driver.make_operator_site(4, 1, 1, [(1, 1, np.diag(case["diagonal"]))])
    one = np.ones((1, 1, 1), complex, order="F")
    S = core.rand_unnorm_state_site_tensor(1, 1, 4, rng)
    iters, ev, new = driver.optimize_state_site(one, S, op, one, driver.ProjectorMatrix(), 0, 0, 10000,
                                                case["mode"])
    assert abs(ev - case["value"]) <= 1e-5 * abs(case["value"]) and iters == 0
    assert np.all(np.abs(new.ravel()[:3]) <= 1e-15) and abs(abs(new.ravel()[3]) - 1) < 1e-5


@pytest.mark.parametrize("case", KATS["sweep_until_converged"]["cases"], ids=lambda c: c["name"])
def test_sweep_until_converged_kat(case):
    """tests/chain.cpp:286-307 (1e-7 relative)."""
    ops = mpo.transverse_ising_reference(case["sites"], case["lambda"])
    ch = driver.Chain(ops, driver.ChainOptions(initial_bandwidth_dimension=case["chi"]), seed=3)
    ch.sweep_until_converged()
    e = case["energy"]
    assert abs(ch.get_energy() - e) <= 1e-7 * abs(e)


@pytest.mark.parametrize("case", KATS["optimize_chain"]["cases"], ids=lambda c: c["name"])
def test_optimize_chain_kat(case):
    """tests/chain.cpp:390-432 (1e-10 relative, least-value mode)."""
    ops = mpo.transverse_ising_reference(case["sites"], case["lambda"])
    ch = driver.Chain(ops, driver.ChainOptions(), seed=4)
    ch.optimize_chain()
    assert abs(-ch.get_energy() - case["abs_energy"]) <= 1e-10 * case["abs_energy"]


def test_stress_levels_kat_one_case():
    """tests/stress.cpp:80-187, N=6 lambda=0.1 least value, 4 levels (1e-7)."""
    case = [c for c in KATS["stress_levels"]["cases"] if c["mode"] == "least_value" and c["sites"] == 6][0]
    ops = mpo.transverse_ising_reference(case["sites"], case["lambda"])
    opts = driver.ChainOptions(initial_bandwidth_dimension=2, site_convergence_threshold=1e-10,
                               sweep_convergence_threshold=1e-9, chain_convergence_threshold=1e-9)
    ch = driver.Chain(ops, opts, seed=6)
    got = ch.solve_for_multiple_levels(4)
    for g, e in zip(got, case["energies"]):
        assert abs(g - e) <= 1e-7 * abs(e)


def test_stress_levels_match_ed():
    """The stress golden values agree with exact diagonalisation of the MPO."""
    for case in KATS["stress_levels"]["cases"]:
        if case["mode"] != "least_value":
            continue
        w, _ = ed.lowest_levels(mpo.transverse_ising_reference(case["sites"], case["lambda"]), 4)
        np.testing.assert_allclose(w, case["energies"], rtol=1e-9)


def test_bandwidth_sequence():
    assert driver.compute_bandwidth_dimension_sequence(16, [2] * 10) == [1, 2, 4, 8, 16, 16, 16, 8, 4, 2, 1]
    seq = driver.compute_bandwidth_dimension_sequence(1024, [2] * 100)
    assert seq[:11] == [2 ** k for k in range(11)] and seq[50] == 1024 and seq[-1] == 1
    with pytest.raises(ValueError):
        driver.compute_bandwidth_dimension_sequence(64, [2] * 10)
