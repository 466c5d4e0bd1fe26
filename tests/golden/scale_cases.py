"""At-scale parity cases: the oracle's level loop and the states it starts from.

TEST INFRASTRUCTURE.  ``make_scale_fixtures.py`` runs these cases through the
CPU oracle (``oracle/driver.py``, the restatement of the reference's chain
driver) and commits the converged energies; the ``-m gpu`` tests replay the
same seeded initial states on the device and compare.

Level loop (``chain.cpp:301-310`` solveForMultipleLevels with the chi-growth
``optimizeChain`` replaced by ``sweepUntilConverged`` at a fixed bond
dimension): level 0 starts from the chain's first random state; level k adds
the projector of level k-1 (``constructAndAddProjectorFromState``) and resets
the chain (``chain.cpp:175-237``), which draws a fresh random state and
filters it against the projectors.  The oracle's random sites come from
``InitialSiteSource(seed)`` in a fixed order, so the initial state of every
level can be replayed without solving anything (``initial_states``).
"""
from __future__ import annotations

import numpy as np

from oracle import driver, mpo

# name -> (operator builder, sites, chi, levels, seed)
CASES = {
    "heisenberg_xxx_N100_chi64": (lambda n: mpo.heisenberg(n), 100, 64, 3, 2024),
    "spin1_heisenberg_D0.5_N64_chi64": (lambda n: mpo.heisenberg_spin1(n, 0.5), 64, 64, 1, 2025),
}
ARPACK_NCV = 24


def operator(name):
    build, n, _, _, _ = CASES[name]
    return build(n)


def options(name, **kw):
    _, _, chi, _, _ = CASES[name]
    return driver.ChainOptions(initial_bandwidth_dimension=chi, arpack_ncv=ARPACK_NCV, **kw)


def initial_states(name):
    """The initial state of every level, as the oracle's level loop draws them."""
    _, _, _, levels, seed = CASES[name]
    ch = driver.Chain(operator(name), options(name), seed=seed)
    out = [[s.copy(order="F") for s in ch.state_sites()]]
    for _ in range(1, levels):
        ch.reset()
        out.append([s.copy(order="F") for s in ch.state_sites()])
    return out


def entanglement_profile(sites):
    """Von Neumann entropy of the normalised state across every bond (a
    gauge-invariant fingerprint of an MPS); sites (br, bl, d), any gauge."""
    n = len(sites)
    # left-canonicalise from site 0, reading the Schmidt values of each bond
    # from the singular values of the remainder carried to the right
    carry = np.ones((1, 1), dtype=complex)
    ent = []
    for i in range(n):
        s = np.asarray(sites[i])
        br, bl, d = s.shape
        # A(l, s, r) = sum_l' carry(l, l') S(r, l', s)
        a = np.einsum("ab,rbs->asr", carry, s).reshape(carry.shape[0] * d, br)
        q, r = np.linalg.qr(a)
        carry = r
        if i < n - 1:
            sv = np.linalg.svd(r, compute_uv=False)
            p = sv ** 2 / np.sum(sv ** 2)
            p = p[p > 1e-300]
            ent.append(float(-np.sum(p * np.log(p))))
    return ent


def run_oracle(name):
    """Energies (and sweep counts) of every level, plus the entanglement
    profile of level 0."""
    _, _, _, levels, seed = CASES[name]
    ch = driver.Chain(operator(name), options(name), seed=seed)
    energies, sweeps, profile = [], [], None
    for k in range(levels):
        if k > 0:
            ch.construct_and_add_projector_from_state()
            ch.reset()
        s0 = ch.sweeps
        ch.sweep_until_converged()
        energies.append(float(ch.get_energy()))
        sweeps.append(ch.sweeps - s0)
        if k == 0:
            profile = entanglement_profile(ch.state_sites())
    return {"energies": energies, "sweeps": sweeps, "entanglement_level0": profile}
