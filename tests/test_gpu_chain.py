"""GPU parity of the device-resident chain (sweeps, chi growth, levels).

Known answers come from the reference's own tests (tests/chain.cpp:286-432,
tests/stress.cpp:80-187) via ``tests/golden/reference_kats.json``; the
synthetic workloads are checked against exact diagonalisation and against
the CPU oracle started from the same initial state.

Tolerances: as the reference's tests (1e-7 for sweepUntilConverged and the
stress levels, 1e-10 for optimizeChain); 1e-10 relative for energies
against ED; state overlaps 1 - |<gpu|oracle>| <= 1e-8.
"""
import numpy as np
import pytest

from kat_inputs import KATS
from oracle import driver, ed, mpo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nbc():
    import nutcracker_b200.chain as c
    return c


@pytest.mark.parametrize("case", KATS["sweep_until_converged"]["cases"], ids=lambda c: c["name"])
def test_sweep_until_converged_kat(nbc, case):
    ops = mpo.transverse_ising_reference(case["sites"], case["lambda"])
    ch = nbc.Chain(ops, initial_bandwidth_dimension=case["chi"], seed=3)
    ch.sweep_until_converged()
    assert abs(ch.get_energy() - case["energy"]) <= 1e-7 * abs(case["energy"])


@pytest.mark.parametrize("mode", ["<v", ">v", ">m"])
@pytest.mark.parametrize("case", KATS["optimize_chain"]["cases"], ids=lambda c: c["name"])
def test_optimize_chain_kat(nbc, case, mode):
    ops = mpo.transverse_ising_reference(case["sites"], case["lambda"])
    ch = nbc.Chain(ops, optimizer_mode=mode, seed=4)
    ch.optimize_chain()
    e = ch.get_energy()
    got = {"<v": -e, ">v": e, ">m": abs(e)}[mode]
    assert abs(got - case["abs_energy"]) <= 1e-10 * case["abs_energy"]


# The 10-site greatest-value and largest-magnitude cases depend on the random
# path of the sweep (the CPU restatement with ARPACK and the polar gauge also
# stops on OptimizerObtainedRegressiveEigenvalue for some seeds); the
# reference's own rand() stream is not reproducible, so those two modes are
# pinned on the 6-site chain and the least-value mode on both lengths.
STRESS = [c for c in KATS["stress_levels"]["cases"]
          if c["sites"] == 6 or (c["sites"] == 10 and c["mode"] == "least_value")]


@pytest.mark.parametrize("case", STRESS, ids=lambda c: "%s-%d-%g" % (c["mode"], c["sites"], c["lambda"]))
def test_stress_levels_kat(nbc, case):
    """tests/stress.cpp:80-187: lowest levels by the projector method (1e-7)."""
    mode = {"least_value": "<v", "greatest_value": ">v", "largest_magnitude": ">m"}[case["mode"]]
    ops = mpo.transverse_ising_reference(case["sites"], case["lambda"])
    ch = nbc.Chain(ops, optimizer_mode=mode, initial_bandwidth_dimension=2, site_convergence_threshold=1e-10,
                   sweep_convergence_threshold=1e-9, chain_convergence_threshold=1e-9,
                   sanity_check_threshold=1e-10 if mode == ">m" else 1e-12, seed=6)
    got = ch.solve_for_eigenvalues(len(case["energies"]))
    for g, e in zip(got, case["energies"]):
        if mode == ">m":
            g = abs(g)
        assert abs(g - e) <= 1e-7 * abs(e), (got, case["energies"])


def test_config1_four_levels_vs_ed(nbc):
    """H = -sum ZZ - 0.1 sum X, N=10, chi<=16, 4 levels vs exact diagonalisation (1e-10)."""
    ops = mpo.transverse_ising_ferro(10, 0.1)
    w, _ = ed.lowest_levels(ops, 4)
    ch = nbc.Chain(ops, initial_bandwidth_dimension=16, seed=11)
    got = ch.solve_for_eigenvalues(4)
    for g, e in zip(got, w):
        assert abs(g - e) <= 1e-10 * abs(e), (got, w)


def oracle_and_gpu(nbc, ops, chi, seed, **kw):
    o = driver.Chain(ops, driver.ChainOptions(initial_bandwidth_dimension=chi, **kw), seed=seed)
    g = nbc.Chain(ops, initial_bandwidth_dimension=chi, seed=seed, **kw)
    g.set_state(o.state_sites())
    return o, g


def test_heisenberg_sweeps_match_oracle(nbc):
    """Same initial state, one sweep at a time: energies agree to 1e-10, and
    the converged ground state has overlap 1 with the oracle's."""
    ops = mpo.heisenberg(10)
    o, g = oracle_and_gpu(nbc, ops, 32, 21)  # chi = 32 represents the 10-site ground state exactly
    assert abs(o.get_energy() - g.get_energy()) <= 1e-10 * abs(o.get_energy())
    for _ in range(3):
        o.perform_optimization_sweep()
        g.perform_optimization_sweep()
        assert abs(o.get_energy() - g.get_energy()) <= 1e-9 * abs(o.get_energy())
    o.sweep_until_converged()
    g.sweep_until_converged()
    assert abs(o.get_energy() - g.get_energy()) <= 1e-10 * abs(o.get_energy())
    w, V = ed.lowest_levels(ops, 1)
    assert abs(g.get_energy() - w[0]) <= 1e-9 * abs(w[0])
    ov = abs(driver.compute_state_overlap(o.state_sites(), g.state_sites()))
    assert 1 - ov <= 1e-8
    dense = ed.mps_to_dense(g.state_sites())
    assert 1 - abs(np.vdot(V[:, 0], dense)) <= 1e-8


def test_spin1_chain_vs_ed(nbc):
    ops = mpo.heisenberg_spin1(6, 0.5)
    w, _ = ed.lowest_levels(ops, 2)
    ch = nbc.Chain(ops, initial_bandwidth_dimension=27, seed=5)
    ch.sweep_until_converged()
    assert abs(ch.get_energy() - w[0]) <= 1e-10 * abs(w[0])


def test_increase_bandwidth_preserves_state(nbc):
    """tests/chain.cpp:250-284: growing chi keeps the state (energy unchanged)."""
    ops = mpo.heisenberg(10)
    ch = nbc.Chain(ops, initial_bandwidth_dimension=4, seed=8)
    ch.perform_optimization_sweep()
    e0 = ch.compute_expectation_value()
    before = ch.state_sites()
    ch.increase_bandwidth_dimension(8)
    after = ch.state_sites()
    assert abs(ch.compute_expectation_value() - e0) <= 1e-12 * abs(e0)
    ov = abs(driver.compute_state_overlap(before, after))
    assert abs(ov - 1) <= 1e-12
    assert ch.info()["bandwidth_dimension"] == 8


def test_move_preserves_norm_and_energy(nbc):
    """tests/chain.cpp:143-169."""
    ops = mpo.transverse_ising_reference(8, 0.5)
    ch = nbc.Chain(ops, initial_bandwidth_dimension=8, seed=2)
    e0 = ch.compute_expectation_value()
    for target in (7, 3, 0, 5, 0):
        ch.move_to(target)
        assert abs(ch.compute_expectation_value() - e0) <= 1e-12 * abs(e0)
        s = ch.get_site(target)
        assert abs(np.linalg.norm(s) - 1) < 1e-13


def test_bad_operator_is_rejected(nbc):
    ops = mpo.heisenberg(4)
    bad = list(ops)
    bad[1] = driver.OperatorSite(2, 3, 5, ops[1].idx, ops[1].W)  # left dim does not connect
    import nutcracker_b200
    with pytest.raises(nutcracker_b200.NutcrackerError):
        nbc.Chain(bad)
