"""Serving loop: continuous batching of independent solves.

A stream of transverse-field Ising requests of different sizes (the serving
workload's form: H = -sum ZZ - lam sum X, several N, chi and level counts)
is solved twice: each request alone (one worker), then all of them submitted
at once to a server with several workers, so that they overlap on the device.
Each request's energies must be the same alone and in the mix (1e-12
relative: the results depend only on the request's own inputs), and match
exact diagonalisation (|dE|/N <= 1e-9; the bond dimension chi = 2^(N/2)
represents these chains exactly).  A second test checks that admission keeps
the in-flight footprint within the memory budget.
"""
import pytest

from oracle import ed, mpo

pytestmark = pytest.mark.gpu

REQUESTS = [  # (N, lam, levels, precision)
    (8, 0.5, 1, 0), (10, 1.0, 2, 0), (8, 1.5, 3, 0), (10, 0.7, 1, 1), (8, 1.2, 2, 1), (10, 1.4, 3, 0),
]


def _submit_all(srv, reqs):
    ids = []
    for n, lam, levels, prec in reqs:
        ops = mpo.transverse_ising_ferro(n, lam)
        ids.append(srv.submit(ops, levels=levels, initial_bandwidth_dimension=2 ** (n // 2), seed=7 + n,
                              precision=prec))
    return ids


def test_serving_results_same_alone_and_in_mix_and_match_ed():
    from nutcracker_b200.serve import Server

    alone = []
    with Server(max_inflight=1) as srv:
        for req in REQUESTS:
            (rid,) = _submit_all(srv, [req])
            alone.append(srv.wait(rid))
    with Server(max_inflight=6) as srv:
        ids = _submit_all(srv, REQUESTS)
        mixed = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(REQUESTS) and st["failed"] == 0
    assert st["p50_seconds"] > 0 and st["p99_seconds"] >= st["p50_seconds"]
    for (n, lam, levels, prec), a, m in zip(REQUESTS, alone, mixed):
        assert a["status"] == 0 and m["status"] == 0, (a["message"], m["message"])
        w, _ = ed.lowest_levels(mpo.transverse_ising_ferro(n, lam), levels)
        for ea, em, e in zip(a["energies"], m["energies"], w):
            assert abs(ea - em) <= 1e-12 * abs(ea), (ea, em)
            assert abs(em - e) / n <= 1e-9, (n, lam, levels, prec, em, e)


def test_admission_respects_memory_budget():
    from nutcracker_b200.serve import Server, footprint_bytes

    reqs = [(10, 1.0, 1, 0)] * 6
    one = footprint_bytes(mpo.transverse_ising_ferro(10, 1.0), levels=1, initial_bandwidth_dimension=32)
    budget = 2 * one + one // 2           # at most two requests in flight
    with Server(max_inflight=6, memory_budget_bytes=budget) as srv:
        ids = _submit_all(srv, reqs)
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert all(r["status"] == 0 for r in res)
    assert st["peak_bytes_in_flight"] <= budget
    assert st["peak_bytes_in_flight"] >= one
