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
from threadpoolctl import threadpool_limits

from oracle import driver, mpo

# name -> (operator builder, sites, chi, levels, seed)
CASES = {
    "heisenberg_xxx_N100_chi64": (lambda n: mpo.heisenberg(n), 100, 64, 1, 2024),
    "heisenberg_xxx_N100_chi128": (lambda n: mpo.heisenberg(n), 100, 128, 1, 2026),
    "tfim_lambda1.5_N100_chi32": (lambda n: mpo.transverse_ising_ferro(n, 1.5), 100, 32, 3, 2027),
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
    _, _, chi, levels, seed = CASES[name]
    return draw_initial_states(operator(name), chi, levels, seed)


def draw_initial_states(ops, chi, levels, seed):
    """The sites that ``levels`` resets of ``driver.Chain(ops, seed=seed)`` at
    bond dimension ``chi`` draw from their ``InitialSiteSource``, without
    contracting any environment: each reset (chain.cpp:175-237) draws the
    right-normalised sites N-1 .. 1, then the centre site 0.  The projectors
    that the level loop adds in between draw nothing, and at these bond
    dimensions they do not raise the chain's bond dimension
    (minimum_bandwidth_dimension_for_projector_count), so the draws are the
    same.  ``replay_initial_states`` is the reference for this shortcut."""
    with threadpool_limits(1):   # small QRs: a threaded BLAS only spins
        return _draw(ops, chi, levels, seed)


def _draw(ops, chi, levels, seed):
    phys = [o.d for o in ops]
    n = len(ops)
    bw = min(driver.maximum_bandwidth_dimension(phys), chi)
    dims = driver.compute_bandwidth_dimension_sequence(bw, phys)
    rdims = list(reversed(dims))
    src = driver.InitialSiteSource(seed)
    out = []
    for _ in range(levels):
        rights = [src.right(ops[op].d, rdims[k + 1], rdims[k]) for k, op in enumerate(reversed(range(1, n)))]
        centre = src.middle(ops[0].d, dims[0], dims[1])
        out.append([np.asfortranarray(centre)] + [np.asfortranarray(s) for s in reversed(rights)])
    return out


def replay_initial_states(ops, chi, levels, seed):
    """The same states read from the oracle's own chain after each reset."""
    ch = driver.Chain(ops, driver.ChainOptions(initial_bandwidth_dimension=chi), seed=seed)
    out = [[s.copy(order="F") for s in ch.state_sites()]]
    for _ in range(1, levels):
        ch.reset()
        out.append([s.copy(order="F") for s in ch.state_sites()])
    return out


def fingerprint(states):
    """Per level, two weighted sums over every site's elements (real and
    imaginary part): enough to show a change of seed or draw order, and
    insensitive to the last-bit differences that another BLAS build or
    thread count leaves in the QRs of the random sites."""
    out = []
    for level in states:
        acc = 0j
        for i, s in enumerate(level):
            a = np.asarray(s).ravel(order="F")
            acc += (i + 1) * np.dot(np.arange(1, a.size + 1) % 7 + 1, a)
        out.append([float(acc.real), float(acc.imag)])
    return out


def entanglement_profile(sites):
    """Von Neumann entropy of the normalised state across every bond (a
    gauge-invariant fingerprint of an MPS); sites (br, bl, d), any gauge."""
    with threadpool_limits(1):
        return _entanglement_profile(sites)


def _entanglement_profile(sites):
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
