"""Batched form on the GPU: many XXZ chains swept in lockstep, one grouped
launch per contraction stage (nc_batch_*).

Checked against the oracle and against the single-chain engine:
  * every chain of a seeded batch small enough for exact diagonalisation
    (N <= 14, chi = 2^(N/2) represents the chain exactly) matches ED to
    |dE|/N <= 1e-9, in the complex64 form with its FP64 refinement and in the
    FP64 form;
  * every chain's energy is the same solved alone and inside the batch (its
    result depends only on its own inputs; 1e-13 relative);
  * the complex64 sweeps alone (no refinement) are within 1e-6 per site;
  * a larger member (N = 32, chi = 32) agrees with the single-chain FP64
    solve of the same operator at the same bond dimension;
  * the autotuner's measurement returns a time per tile configuration and a
    table built from it is accepted.
"""
import numpy as np
import pytest

from oracle import ed, mpo

pytestmark = pytest.mark.gpu


def _xxz_batch(seed, count, nmin=6, nmax=14):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        out.append((n, mpo.xxz_random(n, rng), 2 ** (n // 2)))
    return out


def _solve(batch, seeds, **opt):
    from nutcracker_b200.batched import Batch

    with Batch([b[1] for b in batch], [b[2] for b in batch], seeds=seeds, maximum_sweeps=200, **opt) as bt:
        res = bt.solve()
        st = bt.stats()
    return res, st


@pytest.mark.parametrize("precision", [1, 0])
def test_batch_matches_ed_and_is_the_same_alone(precision):
    batch = _xxz_batch(2024, 10)
    seeds = [100 + k for k in range(len(batch))]
    together, st = _solve(batch, seeds, precision=precision)
    assert st["chains"] == len(batch) and st["global_steps"] > 0 and st["lanczos_iterations"] > 0
    for (n, ops, chi), r in zip(batch, together):
        assert r["converged"] == 1
        w, _ = ed.lowest_levels(ops, 1)
        assert abs(r["energy"] - w[0]) / n <= 1e-9, (n, chi, precision, r["energy"], w[0])
        if precision:
            assert r["mixed_sweeps"] >= 2 and r["fp64_sweeps"] >= 2
        else:
            assert r["mixed_sweeps"] == 0 and r["fp64_sweeps"] >= 2
    for k in (0, 3, 7):
        alone, _ = _solve([batch[k]], [seeds[k]], precision=precision)
        e1, e2 = alone[0]["energy"], together[k]["energy"]
        assert abs(e1 - e2) <= 1e-13 * abs(e1), (k, e1, e2)


def test_complex64_sweeps_without_refinement():
    batch = _xxz_batch(7, 6, nmin=8, nmax=12)
    res, _ = _solve(batch, [5] * len(batch), precision=1, refine=0)
    for (n, ops, chi), r in zip(batch, res):
        w, _ = ed.lowest_levels(ops, 1)
        assert r["fp64_sweeps"] == 0
        assert abs(r["energy"] - w[0]) / n <= 1e-6, (n, r["energy"], w[0])


def test_large_member_matches_single_chain_solve():
    from nutcracker_b200.chain import Chain

    rng = np.random.default_rng(77)
    big = mpo.xxz_random(32, rng)
    batch = [(32, big, 32)] + _xxz_batch(5, 5, nmin=8, nmax=12)
    res, _ = _solve(batch, [3] * len(batch), precision=1)
    ch = Chain(big, initial_bandwidth_dimension=32, seed=3)
    e = ch.solve_levels_at_bandwidth(1)[0]
    assert abs(res[0]["energy"] - e) / 32 <= 1e-8, (res[0]["energy"], e)


def test_autotune_measurement_and_table():
    from nutcracker_b200 import batched

    doc = batched.autotune(chis=(16,), problems=32, reps=3)
    assert len(doc["entries"]) == len(batched.STAGES)
    for e in doc["entries"]:
        assert all(t > 0 for t in e["us_per_launch"])
    table = [(batched.STAGES.index(e["stage"]), e["chi"], e["D"], e["d"], e["cfg"]) for e in doc["entries"]]
    batch = _xxz_batch(11, 3, nmin=6, nmax=8)
    res, _ = _solve(batch, [1, 2, 3], precision=0, tile_table=table)
    for (n, ops, chi), r in zip(batch, res):
        w, _ = ed.lowest_levels(ops, 1)
        assert abs(r["energy"] - w[0]) / n <= 1e-9
