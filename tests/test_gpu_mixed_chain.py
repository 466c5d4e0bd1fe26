"""Precision form of the chain (3xTF32 tensor-core contractions, FP64 Krylov,
projected eigenproblem and energies, closing FP64 refinement sweeps).

Each converged energy is compared with exact diagonalisation of the same MPO
(the FP64 oracle for N <= 14): |dE|/N <= 1e-9 is the accuracy target of the
precision form, and the per-level errors are checked for the projector
method too.  Before the refinement, the mixed sweeps alone must already be
within 1e-5 relative of the exact energy.
"""
import numpy as np
import pytest

from oracle import ed, mpo

pytestmark = pytest.mark.gpu

DE_PER_SITE = 1e-9


@pytest.fixture(scope="module")
def nbc():
    import nutcracker_b200.chain as c
    return c


def test_mixed_heisenberg_ground_state_vs_ed(nbc):
    n = 10
    ops = mpo.heisenberg(n)
    w, V = ed.lowest_levels(ops, 1)
    ch = nbc.Chain(ops, initial_bandwidth_dimension=32, seed=21, precision=1)
    for _ in range(3):
        ch.perform_optimization_sweep()
    e_mixed = ch.get_energy()
    assert abs(e_mixed - w[0]) <= 1e-5 * abs(w[0]), (e_mixed, w[0])
    ch.sweep_until_converged()
    info = ch.info()
    assert info["mixed_sweeps"] >= 3 and info["precision"] == 1
    assert abs(ch.get_energy() - w[0]) / n <= DE_PER_SITE, (ch.get_energy(), w[0])
    dense = ed.mps_to_dense(ch.state_sites())
    assert 1 - abs(np.vdot(V[:, 0], dense)) <= 1e-8


def test_mixed_spin1_anisotropy_vs_ed(nbc):
    n = 6
    ops = mpo.heisenberg_spin1(n, 0.5)
    w, _ = ed.lowest_levels(ops, 1)
    ch = nbc.Chain(ops, initial_bandwidth_dimension=27, seed=5, precision=1)
    ch.sweep_until_converged()
    assert abs(ch.get_energy() - w[0]) / n <= DE_PER_SITE, (ch.get_energy(), w[0])


def test_mixed_four_levels_vs_ed(nbc):
    """Config-1 chain (H = -sum ZZ - 0.1 sum X, N=10, chi<=16), four levels by
    the projector method in the precision form, each against ED."""
    n = 10
    ops = mpo.transverse_ising_ferro(n, 0.1)
    w, _ = ed.lowest_levels(ops, 4)
    ch = nbc.Chain(ops, initial_bandwidth_dimension=16, seed=11, precision=1)
    got = ch.solve_for_eigenvalues(4)
    for g, e in zip(got, w):
        assert abs(g - e) / n <= DE_PER_SITE, (got, w)


def test_set_precision_round_trip(nbc):
    """FP64 converge, a few mixed sweeps, back to FP64: the energy returns to
    the FP64 fixed point."""
    n = 8
    ops = mpo.heisenberg(n)
    w, _ = ed.lowest_levels(ops, 1)
    ch = nbc.Chain(ops, initial_bandwidth_dimension=16, seed=3)
    ch.sweep_until_converged()
    e64 = ch.get_energy()
    ch.set_precision(1)
    for _ in range(2):
        ch.perform_optimization_sweep()
    assert abs(ch.get_energy() - e64) <= 1e-5 * abs(e64)
    ch.set_precision(0)
    ch.sweep_until_converged()
    assert abs(ch.get_energy() - e64) <= 1e-10 * abs(e64)
    assert abs(e64 - w[0]) / n <= DE_PER_SITE
