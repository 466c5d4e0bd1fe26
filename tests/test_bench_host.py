"""Host-side helpers of bench.py (no GPU).

The serving sample checks every request against the exact levels of the
transverse-field Ising chain from its free-fermion form; that closed form is
pinned here against exact diagonalisation of the same MPO.
"""
import importlib.util
import os

import pytest

from oracle import ed, mpo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("n", [2, 3, 6, 9, 10])
@pytest.mark.parametrize("lam", [0.5, 1.0, 1.37])
def test_tfim_exact_levels_match_ed(bench, n, lam):
    w, _ = ed.lowest_levels(mpo.transverse_ising_ferro(n, lam), 4)
    ex = bench.tfim_exact_levels(n, lam, 4)
    assert len(ex) == 4
    assert max(abs(a - b) for a, b in zip(w, ex)) < 1e-12 * n
