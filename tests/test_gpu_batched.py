"""Batched form: many independent XXZ chains solved concurrently on one GPU.

The batched workload is a set of chains H = sum_i J_i (X X + Y Y + Delta_i Z Z)
with per-bond couplings J_i ~ U[0.5, 1.5], Delta_i ~ U[0, 2] (seeded), each
solved for its ground state at its own bond dimension.  The chains run through
the serving engine (one worker per concurrent chain, each on its own stream
and arena), so one batch keeps many chains' kernels in flight at once.

Checked here, on a seeded batch of chains small enough for exact
diagonalisation (N <= 12, chi = 2^(N/2) represents them exactly):
  * every chain's energy matches ED (|dE|/N <= 1e-9), in both precision forms;
  * every chain's energy is the same solved alone and inside the batch
    (1e-12 relative: a result depends only on the chain's own inputs);
  * a larger member (N = 32, chi = 64) gives the same energy alone and in the
    batch, and matches a plain single-chain FP64 solve.
"""
import numpy as np
import pytest

from oracle import ed, mpo

pytestmark = pytest.mark.gpu


def _batch(seed=2024, count=12):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(8, 13))
        ops = mpo.xxz_random(n, rng)
        out.append((n, ops, 2 ** (n // 2), k % 3 == 2))   # every third chain in the precision form
    return out


def _submit(srv, batch):
    return [srv.submit(ops, levels=1, initial_bandwidth_dimension=chi, seed=11 + k, precision=int(prec))
            for k, (n, ops, chi, prec) in enumerate(batch)]


def test_batched_xxz_chains_match_ed_and_are_the_same_alone():
    from nutcracker_b200.serve import Server

    batch = _batch()
    with Server(max_inflight=1) as srv:
        alone = [srv.wait(i) for i in _submit(srv, batch)]
    with Server(max_inflight=len(batch)) as srv:
        together = [srv.wait(i) for i in _submit(srv, batch)]
        st = srv.stats()
    assert st["completed"] == len(batch) and st["failed"] == 0
    for (n, ops, chi, prec), a, t in zip(batch, alone, together):
        assert a["status"] == 0 and t["status"] == 0, (a["message"], t["message"])
        ea, et = a["energies"][0], t["energies"][0]
        assert abs(ea - et) <= 1e-12 * abs(ea), (n, prec, ea, et)
        w, _ = ed.lowest_levels(ops, 1)
        assert abs(et - w[0]) / n <= 1e-9, (n, chi, prec, et, w[0])


def test_batched_large_member_same_in_batch_and_as_single_chain():
    from nutcracker_b200.chain import Chain
    from nutcracker_b200.serve import Server

    rng = np.random.default_rng(77)
    big = mpo.xxz_random(32, rng)
    small = _batch(seed=5, count=6)
    with Server(max_inflight=8) as srv:
        rid = srv.submit(big, levels=1, initial_bandwidth_dimension=64, seed=3)
        _submit(srv, small)
        in_batch = srv.wait(rid)
        srv.drain()
    assert in_batch["status"] == 0, in_batch["message"]
    with Server(max_inflight=1) as srv:
        alone = srv.wait(srv.submit(big, levels=1, initial_bandwidth_dimension=64, seed=3))
    assert abs(in_batch["energies"][0] - alone["energies"][0]) <= 1e-12 * abs(alone["energies"][0])
    ch = Chain(big, initial_bandwidth_dimension=64, seed=3)
    e = ch.solve_levels_at_bandwidth(1)[0]
    assert abs(e - alone["energies"][0]) <= 1e-12 * abs(e)
