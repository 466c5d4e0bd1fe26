"""Parity at the workload sizes, against the CPU oracle.

* The Heisenberg XXX chain at N=100 (the headline chain): the ground state
  at chi=64 and at chi=128 (FP64 and the precision form), swept to
  convergence at the reference's default thresholds from the same seeded
  initial state as the oracle.  The oracle's converged energies are
  committed fixtures (tests/golden/scale_levels.json, made by
  tests/golden/make_scale_fixtures.py): a full oracle run takes tens of
  minutes of CPU time.  FP64 energies agree to 1e-10 relative, the
  precision form's to 1e-9 per site; the ground state's entanglement
  profile (von Neumann entropy across all 99 bonds, a gauge-invariant
  fingerprint of the state) to 1e-6.
* Ground plus two excited levels by the projector method
  (chain.cpp:301-310) at N=100, on the transverse-field Ising chain at
  lambda=1.5 (chi=32), whose levels are non-degenerate and exactly known
  (free fermions): every level against the oracle to 1e-10 relative, and
  against the exact level to the truncation error.  (The excited levels of
  the Heisenberg chain form an exactly degenerate triplet, inside which
  single-site sweeps at the reference's 1e-12 threshold drift for hundreds
  of sweeps: the oracle's first excited level still changed by 1.3e-7 per
  sweep, shrinking 4% a sweep, after 13 sweeps of 42 s.)
* The spin-1 Heisenberg chain with single-ion anisotropy D=0.5 at N=64,
  chi=64, in FP64 and in the precision form (3xTF32 sweeps followed by the
  FP64 refinement): |dE|/N <= 1e-9 against the oracle.
* The H_eff product at chi=1024 (core.f95:2529-2556) against
  oracle.core.apply_heff: FP64 to 1e-12 relative, the precision form to
  5e-6 relative (3xTF32 products carry ~1e-6).
"""
import json
import os

import numpy as np
import pytest

from oracle import core

HERE = os.path.dirname(os.path.abspath(__file__))
import sys  # noqa: E402
sys.path.insert(0, os.path.join(HERE, "golden"))
import scale_cases  # noqa: E402

pytestmark = pytest.mark.gpu



def _fixture(name):
    with open(os.path.join(HERE, "golden", "scale_levels.json")) as f:
        data = json.load(f)
    if name not in data:
        pytest.skip("oracle fixture %s not generated (tests/golden/make_scale_fixtures.py %s)" % (name, name))
    return data[name]


def _same_state(profile, fx):
    """Ground states agree bond by bond in entanglement entropy to 1e-6: two
    states with overlap 1 - 1e-8 (the plain form's overlap bound) may differ
    by ~1e-4 here, so this is the stricter check."""
    diff = np.max(np.abs(np.array(profile) - np.array(fx["entanglement_level0"])))
    assert diff <= 1e-6, diff


def _solve_levels(name, precision=0):
    import nutcracker_b200.chain as nbc

    _, n, chi, levels, seed = scale_cases.CASES[name]
    inits = scale_cases.initial_states(name)
    # the replayed initial states are the ones the oracle started from
    np.testing.assert_allclose(scale_cases.fingerprint(inits), _fixture(name)["initial_states_fingerprint"],
                               rtol=1e-9)
    ch = nbc.Chain(scale_cases.operator(name), initial_bandwidth_dimension=chi, seed=seed)
    if precision:
        ch.set_precision(precision)
    energies, profile = [], None
    for k in range(levels):
        if k > 0:
            ch.construct_and_add_projector_from_state()
        ch.set_state(inits[k])
        ch.sweep_until_converged()
        energies.append(ch.get_energy())
        if k == 0:
            profile = scale_cases.entanglement_profile(ch.state_sites())
    return energies, profile


@pytest.mark.parametrize("name,precision", [("heisenberg_xxx_N100_chi64", 0), ("heisenberg_xxx_N100_chi128", 0),
                                            ("heisenberg_xxx_N100_chi128", 1)],
                         ids=["chi64_ground_fp64", "chi128_ground_fp64", "chi128_ground_precision_form"])
def test_heisenberg_N100_vs_oracle(name, precision):
    fx = _fixture(name)
    got, profile = _solve_levels(name, precision)
    n = fx["sites"]
    assert len(got) == len(fx["energies"])
    for g, e in zip(got, fx["energies"]):
        assert abs(g - e) / n <= 1e-9, (got, fx["energies"])
        if precision == 0:
            assert abs(g - e) <= 1e-10 * abs(e), (got, fx["energies"])
    _same_state(profile, fx)


def _tfim_exact_levels(n, lam, k):
    """Lowest k levels of H = -sum Z_i Z_{i+1} - lam sum X_i on n open sites
    (free fermions: the BdG matrix [[A, B], [-B, -A]] with A = 2 lam I minus
    the nearest-neighbour ones and B[i, i+1] = -1 has eigenvalues +-L_k; the
    levels are -sum(L)/2 plus sums of subsets of the L_k)."""
    A = np.diag(np.full(n, 2.0 * lam))
    B = np.zeros((n, n))
    for i in range(n - 1):
        A[i, i + 1] = A[i + 1, i] = -1.0
        B[i, i + 1], B[i + 1, i] = -1.0, 1.0
    L = np.sort(np.abs(np.linalg.eigvalsh(np.block([[A, B], [-B, -A]]))[n:]))
    e0 = -0.5 * float(L.sum())
    m = min(n, 4)
    return sorted(e0 + sum(float(L[i]) for i in range(m) if mask >> i & 1) for mask in range(1 << m))[:k]


def test_tfim_N100_ground_and_two_excited_vs_oracle():
    name = "tfim_lambda1.5_N100_chi32"
    fx = _fixture(name)
    got, profile = _solve_levels(name)
    n = fx["sites"]
    assert len(got) == len(fx["energies"]) == 3
    for g, e in zip(got, fx["energies"]):
        assert abs(g - e) <= 1e-10 * abs(e), (got, fx["energies"])
    exact = _tfim_exact_levels(n, 1.5, 3)
    assert all(abs(g - x) / n <= 1e-9 for g, x in zip(got, exact)), (got, exact)
    _same_state(profile, fx)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "precision_form"])
def test_spin1_N64_vs_oracle(precision):
    name = "spin1_heisenberg_D0.5_N64_chi64"
    fx = _fixture(name)
    got, profile = _solve_levels(name, precision)
    n = fx["sites"]
    for g, e in zip(got, fx["energies"]):
        assert abs(g - e) / n <= 1e-9, (got, fx["energies"])
        if precision == 0:
            assert abs(g - e) <= 1e-10 * abs(e), (got, fx["energies"])
    _same_state(profile, fx)


@pytest.mark.parametrize("mixed", [False, True], ids=["fp64", "precision_form"])
def test_heff_chi1024_vs_oracle(mixed):
    import ctypes as ct

    import torch

    import nutcracker_b200 as nb
    from nutcracker_b200 import operators

    chi = 1024
    op = operators.heisenberg(4)[1]
    rng = np.random.default_rng(31)

    def rc(shape):
        return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))

    L, R, x = rc((chi, chi, op.cl)), rc((chi, chi, op.cr)), rc((chi, chi, op.d))
    want = core.apply_heff(chi, chi, op.cl, op.cr, op.d, L, op.idx, op.W, R, x).ravel(order="F")

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel(order="F"))).cuda()

    W, idx = dev(op.W), dev(op.idx.astype(np.int32))
    dL, dR, dx = dev(L), dev(R), dev(x)
    y = torch.full_like(dx, float("nan"))
    fn = nb.lib.nc_heff_apply_mixed_dev if mixed else nb.lib.nc_heff_apply_dev
    p = [ct.c_void_p(t.data_ptr()) for t in (idx, W, dL, dR, dx, y)]
    assert fn(chi, chi, op.cl, op.cr, op.d, op.nnz, *p) == 0, nb.lib.nc_last_error()
    torch.cuda.synchronize()
    got = y.cpu().numpy()
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err <= (5e-6 if mixed else 1e-12), err
