"""The at-scale oracle fixtures and the helpers that replay them (CPU only).

The ``-m gpu`` tests in ``test_gpu_scale.py`` replay the oracle's seeded
initial states without building the oracle's chain
(``scale_cases.draw_initial_states``); here that shortcut is checked against
the states the oracle's own chain holds after each reset, and every
committed fixture against the case table it was made from.
"""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import scale_cases  # noqa: E402

from oracle import mpo  # noqa: E402


@pytest.mark.parametrize("build,n,chi,levels,seed", [
    (mpo.heisenberg, 12, 8, 3, 5),
    (lambda n: mpo.heisenberg_spin1(n, 0.5), 10, 9, 2, 7),
    (lambda n: mpo.transverse_ising_ferro(n, 1.5), 9, 64, 2, 3),   # chi above the chain maximum
])
def test_draw_matches_the_oracle_chain(build, n, chi, levels, seed):
    ops = build(n)
    drawn = scale_cases.draw_initial_states(ops, chi, levels, seed)
    held = scale_cases.replay_initial_states(ops, chi, levels, seed)
    assert len(drawn) == len(held) == levels
    for a, b in zip(drawn, held):
        assert len(a) == len(b) == n
        for x, y in zip(a, b):
            assert x.shape == y.shape
            np.testing.assert_array_equal(x, y)


def test_fixtures_match_the_case_table():
    with open(os.path.join(HERE, "golden", "scale_levels.json")) as f:
        data = json.load(f)
    assert set(data) <= set(scale_cases.CASES)
    for name, fx in data.items():
        _, n, chi, levels, seed = scale_cases.CASES[name]
        assert (fx["case"], fx["sites"], fx["chi"], fx["levels"], fx["seed"]) == (name, n, chi, levels, seed)
        assert len(fx["energies"]) == len(fx["sweeps"]) == levels
        assert len(fx["entanglement_level0"]) == n - 1
        # levels in increasing order (the projector method finds them bottom-up)
        assert all(a <= b + 1e-9 * abs(b) for a, b in zip(fx["energies"], fx["energies"][1:]))
        np.testing.assert_allclose(scale_cases.fingerprint(scale_cases.initial_states(name)),
                                   fx["initial_states_fingerprint"], rtol=1e-9)


def test_tfim_fixture_is_exact():
    """The oracle's three N=100 transverse Ising levels (projector method,
    chi=32) against the exact free-fermion levels: the fixture that the GPU
    is compared with is itself pinned to an exact answer at scale."""
    with open(os.path.join(HERE, "golden", "scale_levels.json")) as f:
        fx = json.load(f)["tfim_lambda1.5_N100_chi32"]
    n, lam = fx["sites"], 1.5
    A = np.diag(np.full(n, 2.0 * lam))
    B = np.zeros((n, n))
    for i in range(n - 1):
        A[i, i + 1] = A[i + 1, i] = -1.0
        B[i, i + 1], B[i + 1, i] = -1.0, 1.0
    L = np.sort(np.abs(np.linalg.eigvalsh(np.block([[A, B], [-B, -A]]))[n:]))
    e0 = -0.5 * float(L.sum())
    exact = [e0, e0 + L[0], e0 + L[1]]
    for got, want in zip(fx["energies"], exact):
        assert abs(got - want) / n <= 1e-13, (fx["energies"], exact)
