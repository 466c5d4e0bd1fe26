#!/usr/bin/env python
"""Benchmark: variational-MPS sweeps per second on the Heisenberg chain,
precision form (3xTF32 tensor-core contractions) against the plain FP64 form.

Workload (the reference's headline configuration): S=1/2 Heisenberg XXX
chain H = sum (XX + YY + ZZ), N=100 open sites, d=2, MPO bond dimension 5,
state bond dimension chi=1024 (reached from a chi=256 warm start, "256 then
1024"), complex128 state, seeded random initial MPS, reference tolerances.

One step = one full optimisation sweep (Chain::performOptimizationSweep,
chain.cpp:147-163): 198 site eigen-solves, 198 gauge moves and environment
updates.  Both forms are timed from the same freshly grown chi=1024 state
(two sweeps at chi=256, then the growth, no sweep at chi=1024 yet), after W
untimed warm-up sweeps of each form that are then discarded, so the K timed
sweeps include the transient after the growth (the FP64 form's first sweep
needs ~10 H_eff products per site to reach its 1e-12 site tolerance).
``value`` is the precision form's sweeps/s over K sweeps plus its FP64 final
energy evaluation (every environment rebuilt in FP64 for the state the
mixed sweeps left, and the expectation value), which is inside the timed
window; ``fp64.value`` the plain form's.  ``accuracy`` compares that FP64
evaluation with the FP64 form's energy after the same K sweeps (target
|dE|/N <= 1e-9), and reports the closing FP64 sweep (the refinement) timed on
its own.  ``e2e`` is the precision form through the public C-ABI with the
grown state uploaded from pinned host memory (environments rebuilt) before
each sweep and the energy read back after it.  Per-site working sets
(environments 84 MB each) exceed the 126 MB L2 together with the site and
scratch tensors, so no L2 flush is inserted.

``--impl reference`` times the CPU restatement of the reference path
(numpy/scipy on all host cores: reference-ordered zgemm H_eff products,
zgesdd polar moves, sparse-MPO environment updates) on a bounded sample of
interior chi=1024 site steps and extrapolates to a sweep.

Multi-GPU: replicas only (a sweep is a sequential chain of dependent site
solves); each rank sweeps its own chain and value = all ranks' sweeps / the
slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nutcracker-1_b200"))

T_START = time.perf_counter()


def log(msg):
    """Progress line on stderr (the JSON line alone goes to stdout)."""
    sys.stderr.write("[bench %7.1fs] %s\n" % (time.perf_counter() - T_START, msg))
    sys.stderr.flush()


METRIC = "sweeps/s @N=100 \u03c7=1024 mixed vs FP64 GPU at |\u0394E|/N\u22641e-9"
UNIT = "sweeps/s"
# H_eff products per interior site step charged to the CPU sample when no
# measured sweep segment is available (the reference arm): the mean that
# ARPACK (ncv=3, tol 1e-12) needed per interior site when the oracle swept
# the converged N=100, chi=128 state on a B200 box's host (cpu_validation).
CPU_SAMPLE_MATVECS = 1.37
# DRAM traffic of one tcgen05 stage-A GEMM launch at chi=1024 (ncu, read 216.9 MB +
# write 48.0 MB; the shape's algorithmic operand bytes are 185 MB).
TC32_PROFILED_TRAFFIC = 264.9e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sites", type=int, default=100)
    ap.add_argument("--chi", type=int, default=1024)
    ap.add_argument("--chi-start", type=int, default=256)
    ap.add_argument("--presweeps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"],
                    help="both (default): time FP64 and precision-form sweeps from the same state; "
                         "value is the precision form's")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-loop sample")
    ap.add_argument("--serving-only", action="store_true", help="run only the serving-loop sample")
    ap.add_argument("--serve-requests", type=int, default=24,
                    help="requests in the serving sample (the serving workload has 20k; a bounded sample)")
    ap.add_argument("--serve-half", action="store_true",
                    help="halve the serving workload's N and chi ranges (N<=64, chi<=128)")
    ap.add_argument("--serve-no-mixed", action="store_true", help="serve the FP64 form only")
    ap.add_argument("--serve-fp64-stream", action="store_true",
                    help="also run the stream in the FP64 form (by default the FP64 form gives the plain "
                         "one-at-a-time baseline only)")
    ap.add_argument("--serve-plain", type=int, default=6,
                    help="requests of the stream timed one at a time and then all at once (the plain "
                         "per-solve baseline and the concurrency speed-up on the same requests)")
    ap.add_argument("--serve-slots", type=int, default=0, help="concurrent requests (0: min(32, 2 x cores))")
    ap.add_argument("--serve-rates", default="64",
                    help="Poisson arrival rates swept by the serving sample, requests/s (comma-separated)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-form sample")
    ap.add_argument("--no-config3", action="store_true", help="skip the spin-1 precision-form sample")
    ap.add_argument("--config3-only", action="store_true", help="run only the spin-1 precision-form sample")
    ap.add_argument("--c3-sites", type=int, default=64)
    ap.add_argument("--c3-chi", type=int, default=512)
    ap.add_argument("--c3-levels", type=int, default=2)
    ap.add_argument("--batched-only", action="store_true", help="run only the batched-form sample")
    ap.add_argument("--batch-chains", type=int, default=256,
                    help="chains in the batched sample (the batched workload has 4096; a bounded sample)")
    ap.add_argument("--batch-sweep-tol", type=float, default=1e-10,
                    help="relative sweep-energy threshold of the batched sample (batch and single-chain alike)")
    ap.add_argument("--batch-plain", type=int, default=16,
                    help="chains of the batch also solved one at a time by the single-chain engine")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-time-to-accuracy", action="store_true",
                    help="skip the untimed evaluations behind the time-to-accuracy comparison")
    ap.add_argument("--time-budget", type=float, default=780.0,
                    help="seconds after which the remaining secondary samples (serving, batched, spin-1) are "
                         "skipped and recorded as such, so that a run ends within minutes")
    ap.add_argument("--no-cpu-validation", action="store_true",
                    help="skip the oracle's measured chi=128 sweep segment that checks the extrapolation model")
    ap.add_argument("--cpu-validation-s", type=float, default=60.0)
    ap.add_argument("--phases", action="store_true",
                    help="synchronise and time each sweep phase (diagnostics; slows the sweep slightly)")
    ap.add_argument("--gauge-only", action="store_true",
                    help="time only the Householder-QR gauge move of a chi x chi site (kernel profiling)")
    ap.add_argument("--heff-only", action="store_true",
                    help="time only the effective-Hamiltonian product at --chi (kernel profiling)")
    ap.add_argument("--tc-gemm-only", action="store_true",
                    help="time only the tcgen05 3xTF32 complex GEMM of the stage-A shape at --chi "
                         "(M=chi, N=5*chi, K=chi; kernel profiling)")
    return ap.parse_args()


def run_heff_only(args):
    """W + K H_eff products of the interior Heisenberg site at --chi on
    seeded random environments (the workload of the dominant kernel)."""
    import ctypes as ct
    import torch

    import nutcracker_b200 as nb
    from nutcracker_b200 import operators

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    nb.lib.nc_set_stream(ct.c_void_p(stream.cuda_stream))
    op = operators.heisenberg(4)[1]
    chi, d, cl, cr = args.chi, 2, 5, 5
    g = torch.Generator(device="cuda").manual_seed(args.seed)
    L = torch.randn(chi * chi * cl, dtype=torch.complex128, device="cuda", generator=g)
    R = torch.randn(chi * chi * cr, dtype=torch.complex128, device="cuda", generator=g)
    x = torch.randn(chi * chi * d, dtype=torch.complex128, device="cuda", generator=g)
    y = torch.empty_like(x)
    W = torch.from_numpy(op.W.ravel(order="F")).cuda()
    idx = torch.from_numpy(op.idx.ravel(order="F").astype(np.int32)).cuda()

    def once():
        st = nb.lib.nc_heff_apply_dev(chi, chi, cl, cr, d, op.nnz, ct.c_void_p(idx.data_ptr()),
                                      ct.c_void_p(W.data_ptr()), ct.c_void_p(L.data_ptr()),
                                      ct.c_void_p(R.data_ptr()), ct.c_void_p(x.data_ptr()),
                                      ct.c_void_p(y.data_ptr()))
        if st != 0:
            nb._check()

    for _ in range(args.warmup):
        once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")
    e0.record(stream)
    for _ in range(args.steps):
        once()
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    flops = 8 * d * chi * chi * (cl * chi + cr * chi) + 8 * op.nnz * d * d * chi * chi
    print(json.dumps({"heff_chi": chi, "ms": t * 1e3, "tflops": flops / t / 1e12}), flush=True)


def run_tc_gemm_only(args):
    """W + K calls of the tcgen05 3xTF32 complex GEMM on the stage-A shape of
    the chi x chi interior site (psi_a times the five left-environment blocks),
    seeded random complex128 operands, through nc_tc_zgemm_dev."""
    import ctypes as ct
    import torch

    import nutcracker_b200 as nb

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    nb.lib.nc_set_stream(ct.c_void_p(stream.cuda_stream))
    M, N, K = args.chi, 5 * args.chi, args.chi
    g = torch.Generator(device="cuda").manual_seed(args.seed)
    A = torch.randn(K, M, dtype=torch.complex128, device="cuda", generator=g)   # column-major M x K
    B = torch.randn(N, K, dtype=torch.complex128, device="cuda", generator=g)   # column-major K x N
    C = torch.empty((N, M), dtype=torch.complex128, device="cuda")

    def once():
        if nb.lib.nc_tc_zgemm_dev(M, N, K, ct.c_void_p(A.data_ptr()), ct.c_void_p(B.data_ptr()),
                                  ct.c_void_p(C.data_ptr()), 1) != 0:
            nb._check()

    for _ in range(args.warmup):
        once()
    nb.lib.nc_profile_begin(ct.c_double(1e9))
    for _ in range(args.steps):
        once()
    n, ms, fl = ct.c_uint64(), ct.c_double(), ct.c_double()
    nb.lib.nc_profile_query(1, ct.byref(n), ct.byref(ms), ct.byref(fl))
    nb.lib.nc_profile_end(ct.byref(ct.c_uint64()), ct.byref(ct.c_double()), ct.byref(ct.c_double()))
    print(json.dumps({"tc_gemm": [M, N, K], "launches": n.value, "ms_per_launch": ms.value / max(n.value, 1),
                      "tf32_tflops": fl.value / (ms.value * 1e-3) / 1e12 if ms.value > 0 else None}), flush=True)


def tfim_exact_levels(n, lam, k):
    """Lowest k levels of the open chain H = -sum Z_i Z_{i+1} - lam sum X_i, exact
    at any N from its free-fermion form (Jordan-Wigner; Lieb, Schultz & Mattis 1961):
    with A = 2 lam I minus the nearest-neighbour ones and the antisymmetric pairing B
    (B[i,i+1] = -1), the BdG matrix [[A, B], [-B, -A]] has eigenvalues +-L_k, and the
    spectrum is -sum(L)/2 plus the sum of any subset of the L_k."""
    A = np.diag(np.full(n, 2.0 * lam))
    B = np.zeros((n, n))
    for i in range(n - 1):
        A[i, i + 1] = A[i + 1, i] = -1.0
        B[i, i + 1], B[i + 1, i] = -1.0, 1.0
    L = np.sort(np.abs(np.linalg.eigvalsh(np.block([[A, B], [-B, -A]]))[n:]))
    e0 = -0.5 * float(L.sum())
    m = min(n, 4)
    levels = sorted(e0 + sum(float(L[i]) for i in range(m) if mask >> i & 1) for mask in range(1 << m))
    return levels[:k]


def serving_sample(args):
    """Serving workload sample: transverse-field Ising solves H = -sum ZZ - lam sum X with
    lam ~ U[0.5,1.5], N ~ U{8..128}, chi ~ U{16..256} (capped at the chain's maximum bond
    dimension), 1-4 levels each, seeded, Poisson arrivals, in the plain FP64 form and in the
    precision form (precision=1: mixed sweeps and the FP64 refinement).

    The plain per-solve GPU throughput is the FP64 form solving the first `serve_plain`
    requests one at a time.  The serving loop (continuous batching with `slots` slots: a
    request starts as soon as a slot and its environments' HBM footprint are free) then
    takes the whole stream on its Poisson arrival schedule, at each rate of `serve_rates`,
    in the precision form and once in the FP64 form.  speedup_vs_plain = serving solves/s
    divided by the plain FP64 per-solve throughput; speedup_same_form divides by the same
    form's one-at-a-time throughput instead (the concurrency gain alone).  Every energy is
    checked against the exact free-fermion levels of its chain, and a request's energies
    must be the same alone and in the stream."""
    from nutcracker_b200 import operators
    from nutcracker_b200.serve import Server

    rng = np.random.default_rng(args.seed + 5)
    reqs = []
    n_hi, chi_hi = (64, 128) if args.serve_half else (128, 256)
    for _ in range(args.serve_requests):
        n = int(rng.integers(8, n_hi + 1))
        lam = float(rng.uniform(0.5, 1.5))
        chi = int(min(rng.integers(16, chi_hi + 1), 2 ** (n // 2)))
        levels = int(rng.integers(1, 5))
        reqs.append((n, lam, chi, levels))
    gaps = rng.exponential(1.0, size=len(reqs))   # unit-rate Poisson gaps, scaled per rate
    rates = [float(r) for r in args.serve_rates.split(",")]
    ops = {}

    def op(n, lam):
        if (n, lam) not in ops:
            ops[(n, lam)] = operators.ferromagnetic_transverse_ising(n, lam)
        return ops[(n, lam)]

    slots = args.serve_slots or max(1, min(32, 2 * (os.cpu_count() or 4)))

    def submit(srv, r, k, precision):
        n, lam, chi, levels = r
        return srv.submit(op(n, lam), levels=levels, initial_bandwidth_dimension=chi, seed=1000 + k,
                          precision=precision)

    def warm(srv, precision):
        w = operators.ferromagnetic_transverse_ising(16, 1.0)
        for i in [srv.submit(w, levels=1, initial_bandwidth_dimension=16, seed=1, precision=precision)
                  for _ in range(slots)]:
            srv.wait(i)

    def one_at_a_time(precision):
        with Server(max_inflight=slots) as srv:
            warm(srv, precision)
            out = []
            t0 = time.perf_counter()
            for k, r in enumerate(reqs[:args.serve_plain]):
                out.append(srv.wait(submit(srv, r, k, precision)))
            log("serving: %d requests one at a time (precision %d): %.1f s" % (len(out), precision, time.perf_counter() - t0))
            return out, time.perf_counter() - t0

    def stream(precision, rate):
        arrivals = np.cumsum(gaps / rate)
        with Server(max_inflight=slots) as srv:
            warm(srv, precision)
            start = time.perf_counter()
            ids = []
            for k, r in enumerate(reqs):
                delay = arrivals[k] - (time.perf_counter() - start)
                if delay > 0:
                    time.sleep(delay)
                ids.append(submit(srv, r, k, precision))
            res = [srv.wait(i) for i in ids]
            window = time.perf_counter() - start
            after = srv.stats()
        log("serving: stream of %d at %.0f/s (precision %d): %.1f s" % (len(reqs), rate, precision, window))
        lat = sorted(x["seconds_total"] for x in res if x["status"] == 0)
        pct = (lambda q: lat[min(len(lat) - 1, int(np.ceil(q * len(lat))) - 1)]) if lat else (lambda q: None)
        exact_err, exact_err_full_chi = [], []
        for r, x in zip(reqs, res):
            n, lam, chi, levels = r
            if x["status"] == 0:
                err = max(abs(e - ref) / n for e, ref in zip(x["energies"], tfim_exact_levels(n, lam, levels)))
                exact_err.append(err)
                if chi >= 2 ** (n // 2):   # the bond dimension represents the chain exactly
                    exact_err_full_chi.append(err)
        return res, {
            "rate_per_s": rate, "requests": len(reqs), "failed": sum(1 for x in res if x["status"] != 0),
            "solves_per_s": len(lat) / window if window > 0 else None,
            "p50_s": pct(0.5), "p99_s": pct(0.99), "mean_s": float(np.mean(lat)) if lat else None,
            "window_s": window, "peak_gb_in_flight": after["peak_bytes_in_flight"] / 1e9,
            "max_dE_per_site_vs_exact": max(exact_err) if exact_err else None,
            "max_dE_per_site_vs_exact_where_chi_is_exact": max(exact_err_full_chi) if exact_err_full_chi else None,
        }

    def same(a_list, b_list):
        return max((abs(a - b) / max(abs(a), 1e-300) for p, m in zip(a_list, b_list)
                    for a, b in zip(p["energies"], m["energies"])), default=0.0)

    plain64, t64 = one_at_a_time(0)
    plain_rate = len(plain64) / t64
    out = {
        "workload": "TFIM -ZZ - lam X: lam~U[0.5,1.5], N~U{8..%d}, chi~U{16..%d} (<= chain maximum), 1-4 levels, "
                    "Poisson arrivals; %d requests (bounded sample of the 20k-request stream)"
                    % (n_hi, chi_hi, len(reqs)),
        "slots": slots,
        "plain": {"form": "fp64", "requests": len(plain64), "solves_per_s": plain_rate, "mean_s": t64 / len(plain64)},
        "speedup_definition": "serving-loop solves/s over the stream / plain FP64 per-solve throughput (the first "
                              "plain requests one at a time); speedup_same_form: / the same form's one-at-a-time "
                              "throughput",
        "exact": "free-fermion levels of every request (truncation error included where chi < 2^(N/2))",
    }
    forms = [("mixed", 1)] if not args.serve_no_mixed else []
    if args.serve_fp64_stream or args.serve_no_mixed:
        forms.append(("fp64", 0))
    for name, prec in forms:
        if out.get("mixed") and time.perf_counter() - T_START > args.time_budget:
            out[name] = {"skipped": "time budget"}
            continue
        if prec:
            plain_f, t_f = one_at_a_time(prec)
            rate_f = len(plain_f) / t_f
        else:
            plain_f, rate_f = plain64, plain_rate
        runs = []
        for rate in (rates if prec or args.serve_no_mixed else rates[-1:]):
            if runs and time.perf_counter() - T_START > args.time_budget:
                runs.append({"rate_per_s": rate, "skipped": "time budget"})
                continue
            res, summary = stream(prec, rate)
            summary["speedup_vs_plain"] = summary["solves_per_s"] / plain_rate if summary["solves_per_s"] else None
            summary["speedup_same_form"] = summary["solves_per_s"] / rate_f if summary["solves_per_s"] else None
            summary["max_rel_diff_alone_vs_stream"] = same(plain_f, res)
            runs.append(summary)
        out[name] = {"precision": "mixed (3xTF32 sweeps + FP64 refinement)" if prec else "fp64",
                     "one_at_a_time_solves_per_s": rate_f, "streams": runs,
                     "max_rel_diff_plain_fp64_vs_form": same(plain64, plain_f)}
    best = max((r.get("speedup_vs_plain") or 0 for f in ("mixed", "fp64") if f in out
                for r in out[f].get("streams", [])),
               default=None)
    out["speedup_vs_plain_best"] = best
    return out


def guarded_sample(fn, args):
    """A secondary sample of the bench line; a failure is recorded in its
    object instead of losing the headline measurement."""
    t0 = time.perf_counter()
    if t0 - T_START > args.time_budget:
        return {"skipped": "the run had used %.0f s of its %.0f s budget before this sample (--time-budget)"
                % (t0 - T_START, args.time_budget), "sample_wall_s": 0.0}
    try:
        out = fn(args)
    except Exception as e:   # noqa: BLE001 - reported in the line
        out = {"error": "%s: %s" % (type(e).__name__, e)}
    out["sample_wall_s"] = time.perf_counter() - t0
    return out


def batched_sample(args):
    """Batched workload sample: independent XXZ chains H = sum_i J_i (XX + YY + Delta_i ZZ)
    with per-bond J_i ~ U[0.5,1.5], Delta_i ~ U[0,2], N ~ U{8..48}, chi ~ U{8..128} (capped
    at the chain's maximum bond dimension), ground state, seeded.  The batch goes through
    the lockstep engine (nc_batch: one persistent grouped launch per contraction stage
    over every chain, one CUDA-graph replay per Lanczos iteration of every chain,
    complex64 contractions with FP64 Krylov and an FP64 refinement), timed with CUDA
    events around nc_batch_solve.  The plain per-chain throughput is the single-chain
    FP64 engine solving the first `plain` chains of the batch one at a time; the same
    chains are also solved as a batch of their own, and each of them alone through the
    batched engine (the energies must be identical alone and in the batch)."""
    import torch

    from nutcracker_b200 import operators
    from nutcracker_b200.batched import Batch, load_tile_table
    from nutcracker_b200.chain import Chain

    rng = np.random.default_rng(args.seed + 11)
    chains = []
    for _ in range(args.batch_chains):
        n = int(rng.integers(8, 49))
        chi = int(min(rng.integers(8, 129), 2 ** (n // 2)))
        chains.append((n, operators.xxz_random(n, rng), chi))
    seeds = [3000 + k for k in range(len(chains))]
    table = load_tile_table()

    def run_batch(idx):
        with Batch([chains[k][1] for k in idx], [chains[k][2] for k in idx], seeds=[seeds[k] for k in idx],
                   tile_table=table, maximum_sweeps=60,
                   sweep_convergence_threshold=args.batch_sweep_tol) as b:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = b.solve()
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            st = b.stats()
        return res, st, dt

    # warm-up (module load, graph instantiation paths)
    run_batch(list(range(min(4, len(chains)))))
    res, st, window = run_batch(list(range(len(chains))))
    log("batched: %d chains in %.1f s" % (len(chains), window))
    nplain = min(args.batch_plain, len(chains))
    if nplain == 0:
        return {"chains": len(chains), "chains_per_s": len(chains) / window, "window_s": window,
                "global_steps": st["global_steps"], "lanczos_iterations": st["lanczos_iterations"],
                "unconverged": sum(1 for r in res if not r["converged"])}
    sub = list(range(nplain))
    # plain: the single-chain FP64 engine, one chain at a time
    plain_e = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in sub:
        n, op, chi = chains[k]
        ch = Chain(op, initial_bandwidth_dimension=chi, seed=seeds[k], sweep_convergence_threshold=args.batch_sweep_tol)
        plain_e.append(ch.solve_levels_at_bandwidth(1)[0])
        del ch
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    log("batched: %d chains one at a time (single-chain engine) in %.1f s" % (nplain, t_plain))
    res_sub, st_sub, window_sub = run_batch(sub)
    alone = [run_batch([k])[0][0]["energy"] for k in sub[:4]]
    same = max(abs(a - res[k]["energy"]) / abs(a) for k, a in zip(sub[:4], alone))
    dev_plain = max(abs(res[k]["energy"] - e) / chains[k][0] for k, e in zip(sub, plain_e))
    rate = len(chains) / window
    plain_rate = nplain / t_plain
    return {
        "workload": "XXZ chains sum J_i (XX + YY + Delta_i ZZ): J_i~U[0.5,1.5], Delta_i~U[0,2] per bond, "
                    "N~U{8..48}, chi~U{8..128} (<= chain maximum), ground state, sweeps until the energy "
                    "changes by < %g relative; %d chains (bounded sample of the 4096-chain batch); complex64 "
                    "contractions, FP64 Krylov, FP64 refinement sweeps" % (args.batch_sweep_tol, len(chains)),
        "engine": "nc_batch lockstep: one grouped launch per contraction stage, Lanczos iteration as "
                  "one CUDA graph replay",
        "chains": len(chains), "unconverged": sum(1 for r in res if not r["converged"]),
        "chains_per_s": rate, "window_s": window,
        "global_steps": st["global_steps"], "lanczos_iterations": st["lanczos_iterations"],
        "kernel_launches": st["kernel_launches"], "device_bytes": st["device_bytes"],
        "mean_sweeps": float(np.mean([r["sweeps"] for r in res])),
        "tile_table_entries": len(table),
        "plain_chains": nplain, "plain_chains_per_s": plain_rate,
        "plain_definition": "single-chain FP64 engine (nc_chain), the first %d chains one at a time" % nplain,
        "speedup_vs_plain": rate / plain_rate,
        "same_chains_batched_chains_per_s": nplain / window_sub,
        "same_chains_speedup": (nplain / window_sub) / plain_rate,
        "max_rel_diff_alone_vs_batch": same,
        "max_abs_dE_per_site_vs_single_chain_fp64": dev_plain,
    }


def config3_spin1_sample(args):
    """Precision form on the spin-1 chain H = sum S.S + 0.5 sum (S^z)^2 (d=3, MPO bond
    dimension 5, N=64, chi=512; the second chain of the precision-form configuration):
    both forms solve the same levels from the same chi=512 state (grown from a chi=128
    start swept twice), each level swept to convergence (the precision form: mixed sweeps,
    then its FP64 refinement), timed with CUDA events; the error of every level of the
    precision form is stated against the FP64 form's."""
    import torch

    from nutcracker_b200 import operators
    from nutcracker_b200.chain import Chain

    n, chi, levels = args.c3_sites, args.c3_chi, args.c3_levels
    ops = operators.heisenberg_spin1(n, 0.5)
    ch = Chain(ops, initial_bandwidth_dimension=min(128, chi), seed=args.seed + 3)
    for _ in range(2):
        ch.perform_optimization_sweep()
    if chi > min(128, chi):
        ch.increase_bandwidth_dimension(chi)
    start = ch.state_sites()
    out = {"workload": "spin-1 Heisenberg sum S.S + 0.5 sum (S^z)^2, N=%d, d=3, MPO bond 5, chi=%d, %d levels "
                       "(projector method), from the same chi=%d state" % (n, chi, levels, chi)}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        c = Chain(ops, initial_bandwidth_dimension=chi, seed=args.seed + 3, precision=prec)
        energies, secs, sweeps = [], [], []
        for k in range(levels):
            if k > 0:
                c.construct_and_add_projector_from_state()
                c.reset()
            else:
                c.set_state(start)
            s0 = c.info()["sweeps"]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            c.sweep_until_converged()
            torch.cuda.synchronize()
            secs.append(time.perf_counter() - t0)
            energies.append(c.get_energy())
            sweeps.append(c.info()["sweeps"] - s0)
            log("config3 %s level %d: %.1f s" % (name, k, secs[-1]))
        out[name] = {"energies": energies, "seconds": secs, "sweeps": sweeps}
    e64, emx = out["fp64"]["energies"], out["mixed"]["energies"]
    out["dE_per_site_per_level"] = [abs(a - b) / n for a, b in zip(emx, e64)]
    out["speedup_vs_fp64"] = sum(out["fp64"]["seconds"]) / max(1e-9, sum(out["mixed"]["seconds"]))
    out["note"] = ("levels >= 1 start from each chain's own random state (reset), so their sweep counts differ "
                   "between the forms; level 0 starts from the same state")
    return out


def run_gauge_only(args):
    """W + K right-moving gauge moves (norm_denorm_going_right_) of a
    (chi, chi, 2) site into its neighbour: device-resident through
    nc_gauge_move_dev, timed with CUDA events on the library's stream, and
    once through the Level-0 host entry point (host copies included)."""
    import ctypes as ct
    import time as _t

    import torch

    import nutcracker_b200 as nb

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    nb.lib.nc_set_stream(ct.c_void_p(stream.cuda_stream))
    rng = np.random.default_rng(args.seed)
    chi = args.chi
    A = np.asfortranarray(rng.standard_normal((chi, chi, 2)) + 1j * rng.standard_normal((chi, chi, 2)))
    B = np.asfortranarray(rng.standard_normal((chi, chi, 2)) + 1j * rng.standard_normal((chi, chi, 2)))
    dA = torch.from_numpy(A.ravel(order="F")).cuda()
    dB = torch.from_numpy(B.ravel(order="F")).cuda()
    oA, oB = torch.empty_like(dA), torch.empty_like(dB)
    args_dev = [ct.c_void_p(t.data_ptr()) for t in (dA, dB, oA, oB)]

    def once():
        if nb.lib.nc_gauge_move_dev(1, chi, chi, chi, 2, 2, *args_dev) != 0:
            nb._check()

    for _ in range(max(1, args.warmup)):
        once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")
    e0.record(stream)
    for _ in range(args.steps):
        once()
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    t0 = _t.perf_counter()
    nb.Core.norm_denorm_going_right(chi, chi, chi, 2, 2, A, B)
    t_host = _t.perf_counter() - t0
    m, n = 2 * chi, chi
    flops = 4.0 * (2 * m * n * n - 2.0 / 3.0 * n ** 3)
    print(json.dumps({"gauge_chi": chi, "ms": ms, "qr_equiv_tflops": flops / (ms * 1e-3) / 1e12,
                      "ms_with_host_copies": t_host * 1e3}), flush=True)


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def bond_profile(n, chi, d=2):
    mid = (n + 1) // 2
    fwd = [1]
    p = 1
    for _ in range(mid):
        p *= d
        if p >= chi:
            break
        fwd.append(p)
    return fwd + [chi] * (n + 1 - 2 * len(fwd)) + list(reversed(fwd))


def sweep_weight(n, chi):
    """Number of full-chi interior site steps a sweep is equivalent to
    (cost per site ~ bl*br*(bl+br))."""
    b = bond_profile(n, chi)
    order = list(range(1, n)) + list(range(n - 2, -1, -1))
    return sum(b[i] * b[i + 1] * (b[i] + b[i + 1]) for i in order) / (2.0 * chi ** 3)


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU sample of the reference path (oracle restatement, test infrastructure)
# ---------------------------------------------------------------------------

def cpu_site_step_seconds(chi, reps=1, matvecs=CPU_SAMPLE_MATVECS):
    """Time one interior chi x chi site step of the reference ordering:
    `matvecs` H_eff products (stage 2 + stage 3 zgemm on the dense stage-1
    tensor), compute_expectation, the zgesdd polar move and contract_sos_left."""
    from oracle import core, mpo
    rng = np.random.default_rng(7)
    op = mpo.heisenberg(4)[1]
    d, cl, cr = 2, 5, 5

    def rc(shape):
        return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))

    L, R, S, Snext = rc((chi, chi, cl)), rc((chi, chi, cr)), rc((chi, chi, d)), rc((chi, chi, d))
    S1 = core.iteration_stage_1(chi, cl, cr, d, L, op.idx, op.W)
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        core.iteration_stage_3(chi, chi, cr, d, core.iteration_stage_2(chi, chi, cr, d, S1, S), R)
        t_mv = time.perf_counter() - t0
        t0 = time.perf_counter()
        core.compute_expectation(chi, chi, cl, cr, d, L, S, op.idx, op.W, R)
        core.norm_denorm_going_right(chi, chi, chi, d, d, S, Snext)
        core.contract_sos_left(chi, chi, cl, cr, d, L, op.idx, op.W, S)
        dt = matvecs * t_mv + (time.perf_counter() - t0)
        best = dt if best is None else min(best, dt)
    return best


def cpu_validation(ops, state, budget_s=60.0):
    """The reference algorithm (oracle: ARPACK ncv=3 at tol 1e-12, reference-ordered
    H_eff products, zgesdd polar moves) sweeping the GPU chain's converged state
    from site 0, one BLAS thread, for up to `budget_s` seconds of site steps:
    measured seconds and H_eff products per site, and the same sites predicted
    by the extrapolation model (one interior site step of this bond dimension,
    weighted by bl*br*(bl+br))."""
    from threadpoolctl import threadpool_limits

    from oracle import core, driver

    count = [0]
    orig = core.iteration_stage_3

    def counted(*a):
        count[0] += 1
        return orig(*a)

    core.iteration_stage_3 = counted
    try:
        with threadpool_limits(limits=1):
            chi = max(max(x.shape[0], x.shape[1]) for x in state)
            ch = driver.Chain(ops, driver.ChainOptions(initial_bandwidth_dimension=chi),
                              source=driver.ReplaySource(state))
            steps, weights, mv = [], [], []
            t_all = time.perf_counter()
            while time.perf_counter() - t_all < budget_s and ch.current + 1 < ch.N:
                c0 = count[0]
                t0 = time.perf_counter()
                ch.optimize_site()
                ch.move("R")
                steps.append(time.perf_counter() - t0)
                br, bl, _ = ch.state_site.shape
                weights.append(bl * br * (bl + br))
                mv.append(count[0] - c0)
            interior = [m for m, w in zip(mv, weights) if w == 2 * chi ** 3]
            mean_mv = float(np.mean(interior)) if interior else float(np.mean(mv))
            t_site = cpu_site_step_seconds(chi, matvecs=mean_mv)
    finally:
        core.iteration_stage_3 = orig
    predicted = sum(t_site * w / (2.0 * chi ** 3) for w in weights)
    measured = float(sum(steps))
    return {"chi": chi, "sites": len(steps), "measured_s": measured, "model_s": predicted,
            "model_error": predicted / measured - 1.0, "arpack_matvecs_per_interior_site": mean_mv,
            "threads": 1}


def cpu_baseline(n, chi, validation=None):
    """One interior chi x chi site step of the reference ordering on all host
    cores, charged the H_eff products ARPACK (ncv=3, tol 1e-12) needs per
    interior site in the measured sweep segment (else the committed count),
    extrapolated to a sweep by the bond-profile weight."""
    from threadpoolctl import threadpool_limits

    matvecs = validation["arpack_matvecs_per_interior_site"] if validation else CPU_SAMPLE_MATVECS
    with threadpool_limits(limits=os.cpu_count()):
        t = cpu_site_step_seconds(chi, matvecs=matvecs)
    sweeps_per_s = 1.0 / (t * sweep_weight(n, chi))
    out = {
        "value": sweeps_per_s, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
        "sample": ("one interior chi=%d site step of the reference ordering (%.2f H_eff products via stage-2/3 "
                   "zgemm, compute_expectation, zgesdd polar move, contract_sos_left) = %.2f s, numpy/scipy "
                   "OpenBLAS on %d threads; sweep = %.1f full-chi site steps (bond profile), extrapolated"
                   % (chi, matvecs, t, os.cpu_count(), sweep_weight(n, chi))),
    }
    if validation:
        out["model_check"] = validation
    return out


def run_reference(args, rank):
    if rank != 0:
        return
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(os.cpu_count()))
    times = []
    for i in range(args.warmup + args.steps):
        t = cpu_site_step_seconds(args.chi)
        if i >= args.warmup:
            times.append(t)
    step = float(np.mean(times)) * sweep_weight(args.sites, args.chi)
    value = 1.0 / step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex128", "data": "synthetic",
        "config": {"workload": "heisenberg_xxx_N%d_chi%d" % (args.sites, args.chi), "sites": args.sites,
                   "chi": args.chi, "d": 2, "mpo_bond": 5, "l2": "inputs larger than L2"},
        "cpu_baseline": {"kind": "port", "cores": os.cpu_count(), "value": value, "unit": UNIT,
                         "sample": "per step: one interior chi=%d site step (%.2f H_eff products, expectation, "
                                   "zgesdd move, environment update), extrapolated to a sweep"
                                   % (args.chi, CPU_SAMPLE_MATVECS)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def max_over_ranks(x, dist, device):
    """The largest of the ranks' values (times are reported as the slowest rank's)."""
    if not dist:
        return x
    import torch
    import torch.distributed as td
    t = torch.tensor([x], device=device, dtype=torch.float64)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def replica_seed(seed, rank):
    """Each replica sweeps its own chain from its own random initial state."""
    return seed + 7919 * rank


def replica_throughput(steps, world, seconds_max):
    """Whole-job sweeps/s of `world` independent replicas that each time `steps`
    sweeps: every rank's sweeps over the slowest rank's time."""
    return steps * world / seconds_max


def time_to_accuracy(args, ops, chain, start, res):
    """Device time each form needs, from the same freshly grown state, until its
    energy of record is within 1e-9 per site of the FP64 converged energy (the
    FP64 form's energy after K+1 sweeps).  FP64: the timed per-sweep device
    times up to the first sweep whose energy qualifies.  Precision form: the
    timed per-sweep device times of its mixed sweeps up to the first sweep count
    k whose FP64 evaluation qualifies, plus the timed FP64 evaluation.  The
    evaluations are made untimed on a second chain from a copy of the state
    after k mixed sweeps (k = 1, 2, 3, 4, 6, 8, 12, 16, 20 until one qualifies,
    so the precision form's time is an upper bound)."""
    from nutcracker_b200.chain import Chain

    n = args.sites
    e_ref = res["fp64"]["energy_plus1"]
    tol = 1e-9 * n
    per64, en64 = res["fp64"]["per_sweep_s"], res["fp64"]["energies"]
    k64 = next((k + 1 for k, e in enumerate(en64) if abs(e - e_ref) <= tol), None)
    out = {"reference_energy": e_ref, "target_dE_per_site": 1e-9,
           "fp64_sweeps": k64, "fp64_s": sum(per64[:k64]) if k64 else None}
    permx = res["mixed"]["per_sweep_s"]
    checkpoints = [k for k in (1, 2, 3, 4, 6, 8, 12, 16, 20) if k <= len(permx)]
    chain.set_precision(1)
    chain.set_state(start)
    ev = Chain(ops, initial_bandwidth_dimension=args.chi, seed=args.seed + 99)
    evals = []
    done = 0
    for k in checkpoints:
        while done < k:
            chain.perform_optimization_sweep()
            done += 1
        ev.set_state(chain.state_sites())
        e = ev.get_energy()
        evals.append({"mixed_sweeps": k, "fp64_evaluation": e, "dE_per_site": abs(e - e_ref) / n})
        if abs(e - e_ref) <= tol:
            break
    del ev
    kmx = next((x["mixed_sweeps"] for x in evals if x["dE_per_site"] * n <= tol), None)
    out.update({"mixed_evaluations": evals, "mixed_sweeps": kmx,
                "mixed_s": (sum(permx[:kmx]) + res["mixed"]["eval_s"]) if kmx else None})
    if out["fp64_s"] and out["mixed_s"]:
        out["speedup"] = out["fp64_s"] / out["mixed_s"]
    return out


def run_ours(args, rank, world):
    import ctypes as ct
    import torch

    import nutcracker_b200 as nb
    from nutcracker_b200 import operators
    from nutcracker_b200.chain import Chain

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    if nb.lib.nc_set_stream(ct.c_void_p(stream.cuda_stream)) != 0:
        nb._check()
    dist = world > 1
    if dist:
        import torch.distributed as td

    def barrier():
        if dist:
            td.barrier()


    def timed_sweeps(chain, steps, finish=None):
        """K sweeps (and `finish`, when given) between CUDA events on the
        library's stream; per-sweep device times and energies."""
        barrier()
        torch.cuda.synchronize()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 2)]
        energies = []
        torch.cuda.nvtx.range_push("timed")
        evs[0].record(stream)
        for k in range(steps):
            chain.perform_optimization_sweep()
            evs[k + 1].record(stream)
            energies.append(chain.get_energy())
        if finish is not None:
            finish()
        evs[steps + 1].record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        barrier()
        total = max_over_ranks(evs[0].elapsed_time(evs[steps + 1]) / 1e3, dist, "cuda")
        per = [evs[k].elapsed_time(evs[k + 1]) / 1e3 for k in range(steps)]
        tail = evs[steps].elapsed_time(evs[steps + 1]) / 1e3
        return total, per, tail, energies

    def query(kind):
        n, ms, fl = ct.c_uint64(), ct.c_double(), ct.c_double()
        nb.lib.nc_profile_query(kind, ct.byref(n), ct.byref(ms), ct.byref(fl))
        return int(n.value), ms.value / 1e3, fl.value

    def end_profile():
        n, ms, fl = ct.c_uint64(), ct.c_double(), ct.c_double()
        nb.lib.nc_profile_end(ct.byref(n), ct.byref(ms), ct.byref(fl))

    log("start: N=%d chi %d -> %d, %d warm-up + %d timed sweeps per form" % (args.sites, args.chi_start, args.chi, args.warmup, args.steps))
    ops = operators.heisenberg(args.sites)
    chain = Chain(ops, initial_bandwidth_dimension=args.chi_start, seed=replica_seed(args.seed, rank),
                  time_phases=1 if args.phases else 0)
    for _ in range(args.presweeps):
        chain.perform_optimization_sweep()
    chain.increase_bandwidth_dimension(args.chi)
    log("grown to chi=%d" % args.chi)
    # common start of both forms: the freshly grown chi=1024 state (no sweep
    # at chi=1024 yet), so both timed windows include the transient after
    # the growth and the energy differences are due to precision alone
    start = chain.state_sites()
    n = args.sites
    want64 = args.precision in ("both", "fp64")
    wantmx = args.precision in ("both", "mixed")
    # untimed warm-up of each form from the same state (first-use allocations,
    # recorded QR graphs, tensor maps); the timed windows restart from `start`
    chain.set_precision(0)
    chain.set_state(start)
    energy_start = chain.get_energy()
    for _ in range(args.warmup if want64 else 0):
        chain.perform_optimization_sweep()
    if wantmx:
        chain.set_precision(1)
        chain.set_state(start)
        for _ in range(args.warmup):
            chain.perform_optimization_sweep()
    log("warm-up done")
    clocks = ClockSampler(local)
    clocks.start()
    res = {}

    if want64:
        chain.set_precision(0)
        chain.set_state(start)
        info0 = chain.info()
        launches0 = nb.launch_count()
        nb.lib.nc_profile_begin(ct.c_double(1e9))
        t64, per64, _, en64 = timed_sweeps(chain, args.steps)
        g64 = query(0)
        end_profile()
        info1 = chain.info()
        res["fp64"] = {"seconds": t64, "per_sweep_s": per64, "energies": en64,
                       "launches": nb.launch_count() - launches0, "gemm": g64,
                       "energy": chain.get_energy(), "info0": info0, "info1": info1}
        chain.perform_optimization_sweep()            # one more FP64 sweep: the reference for the closing sweep
        res["fp64"]["energy_plus1"] = chain.get_energy()
        log("fp64 timed: %.1f s" % t64)

    if wantmx:
        chain.set_precision(1)
        chain.set_state(start)
        info0 = chain.info()
        launches0 = nb.launch_count()
        mixed_energy = []

        def final_fp64_energy():
            # the precision form's FP64 final energy evaluation: every
            # environment rebuilt in FP64 for the state the mixed sweeps left,
            # and the FP64 expectation value at the centre site
            mixed_energy.append(chain.get_energy())
            chain.set_precision(0)

        nb.lib.nc_profile_begin(ct.c_double(1e9))
        tmx, permx, t_eval, enmx = timed_sweeps(chain, args.steps, final_fp64_energy)
        gtc = query(1)
        g64m = query(0)
        end_profile()
        info1 = chain.info()
        res["mixed"] = {"seconds": tmx, "per_sweep_s": permx, "eval_s": t_eval, "energies": enmx,
                        "launches": nb.launch_count() - launches0, "tc": gtc, "gemm": g64m,
                        "energy": mixed_energy[0], "energy_fp64_evaluation": chain.get_energy(),
                        "info0": info0, "info1": info1}
        # the closing FP64 sweep (iterative refinement), timed on its own
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        chain.perform_optimization_sweep()
        c1.record(stream)
        torch.cuda.synchronize()
        res["mixed"]["closing_sweep_s"] = c0.elapsed_time(c1) / 1e3
        res["mixed"]["energy_closed"] = chain.get_energy()
        log("mixed timed: %.1f s" % tmx)
    if want64 and wantmx and not args.no_time_to_accuracy:
        res["time_to_accuracy"] = time_to_accuracy(args, ops, chain, start, res)
        log("time to accuracy done")
    clk = clocks.stop()

    # e2e through the public API: state from pinned host memory -> sweep -> energy back
    e2e = None
    head = "mixed" if wantmx else "fp64"
    if not args.no_e2e:
        chain.set_precision(1 if head == "mixed" else 0)
        pinned = [torch.from_numpy(np.ascontiguousarray(s.ravel(order="F"))).pin_memory() for s in start]
        h2d = sum(p.numel() * 16 for p in pinned)
        bonds = [int(start[0].shape[1])] + [int(s.shape[0]) for s in start]
        b = (ct.c_uint32 * len(bonds))(*bonds)
        ptrs = (ct.c_void_p * len(pinned))(*[p.data_ptr() for p in pinned])
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            if nb.lib.nc_chain_set_state(chain._h, b, ptrs) != 0:
                nb._check()
            chain.perform_optimization_sweep()
            _ = chain.get_energy()
        if head == "mixed":
            chain.set_precision(0)   # the FP64 final energy evaluation, as in the device-timed window
            _ = chain.get_energy()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        te = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, "cuda")
        e2e = {"value": replica_throughput(args.steps, world, te), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": 8, "precision": head, "wall_s": time.perf_counter() - t0,
               "step": "upload the freshly grown state from pinned host memory (nc_chain_set_state, environments "
                       "rebuilt), one sweep, energy read back; the precision form adds its FP64 final energy "
                       "evaluation once at the end"}

    # FP64 GEMM peak measured live (MEASURED_PEAKS.json has no FP64 entry)
    a = torch.randn(4096, 4096, dtype=torch.complex128, device="cuda")
    bm = torch.randn(4096, 4096, dtype=torch.complex128, device="cuda")
    for _ in range(2):
        a @ bm
    torch.cuda.synchronize()
    q0 = torch.cuda.Event(enable_timing=True)
    q1 = torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for _ in range(5):
        a @ bm
    q1.record(stream)
    torch.cuda.synchronize()
    peak64 = 8 * 4096 ** 3 * 5 / (q0.elapsed_time(q1) / 1e3) / 1e12
    del a, bm

    if rank != 0:
        return
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak_tf32 = peaks.get("bf16_tflops", 1590.0) / 2.0
    peak_src = ("MEASURED_PEAKS.json bf16_tflops (burst) / 2: dense TF32 runs at half the dense BF16 rate"
                if "bf16_tflops" in peaks else "fallback 1.59 PFLOP/s bf16 / 2")

    def chain_stats(r):
        i0, i1 = r["info0"], r["info1"]
        solves = i1["site_solves"] - i0["site_solves"]
        out = {"energy": r["energy"], "energy_per_site": r["energy"] / n,
               "matvecs_per_site": (i1["matvecs"] - i0["matvecs"]) / max(solves, 1),
               "site_solves": solves, "failures": i1["failures"] - i0["failures"]}
        if args.phases:
            out["phase_seconds"] = {k: i1["seconds_" + k] - i0["seconds_" + k]
                                    for k in ("solve", "gauge", "environment", "projector")}
        return out

    line = {"metric": METRIC, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
            "config": {"workload": "heisenberg_xxx_N%d_chi%d" % (args.sites, args.chi), "sites": args.sites,
                       "chi": args.chi, "chi_start": args.chi_start, "d": 2, "mpo_bond": 5,
                       "precision": head, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 (84 MB environments per site)"},
            "e2e": e2e, "clocks": clk}
    if "fp64" in res:
        r = res["fp64"]
        v64 = replica_throughput(args.steps, world, r["seconds"])
        ms, fl = r["gemm"][1], r["gemm"][2]
        ach = fl / ms / 1e12 if ms > 0 else None
        line["fp64"] = {"value": v64, "ms_per_step": r["seconds"] / args.steps * 1e3,
                        "per_sweep_s": r["per_sweep_s"], "energies": r["energies"],
                        "gpu_launches": int(r["launches"]), "chain": chain_stats(r),
                        "roofline": {"bound": "tensor", "kernel": "zgemm_dmma (FP64 DMMA complex GEMM)",
                                     "achieved": ach, "peak": peak64, "unit": "TFLOP/s",
                                     "frac": ach / peak64 if ach else None,
                                     "peak_source": "cuBLAS zgemm 4096^3 measured in this run",
                                     "gemm_share_of_step": ms / r["seconds"]}}
    if "mixed" in res:
        r = res["mixed"]
        vmx = replica_throughput(args.steps, world, r["seconds"])
        ms, fl = r["tc"][1], r["tc"][2]
        ach = fl / ms / 1e12 if ms > 0 else None
        line.update({"value": vmx, "ms_per_step": r["seconds"] / args.steps * 1e3, "dtype": "3xTF32/f64",
                     "gpu_launches": int(r["launches"]),
                     "step": "one precision-form sweep (198 site solves with 3xTF32 H_eff products, FP64 Krylov "
                             "and gauge moves, 3xTF32 environment updates) from the freshly grown chi=%d state; "
                             "the FP64 final energy evaluation (all environments rebuilt in FP64, expectation "
                             "value) is inside the timed window" % args.chi,
                     "per_sweep_s": r["per_sweep_s"], "final_fp64_evaluation_s": r["eval_s"]})
        line["roofline"] = {"bound": "tensor", "kernel": "tc32_gemm_kernel (tcgen05 kind::tf32, 3xTF32 complex GEMM)",
                            "achieved": ach, "peak": peak_tf32, "unit": "TFLOP/s",
                            "frac": ach / peak_tf32 if ach else None,
                            "traffic": TC32_PROFILED_TRAFFIC, "traffic_unit": "bytes per launch",
                            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one stage-A "
                                              "launch (M=1024, N=5120, K=1024); algorithmic operand bytes of "
                                              "that launch 185 MB",
                            "flops_counted": "TF32 tensor work: 2*M*Nr*Kr per segment, 3 segments",
                            "peak_source": peak_src, "timed_gemms": r["tc"][0],
                            "gemm_share_of_step": ms / r["seconds"],
                            "fp64_gemm_share_of_step": r["gemm"][1] / r["seconds"]}
        line["chain"] = chain_stats(r)
        acc = {"energy_start_fp64": energy_start,
               "energy_mixed_sweeps": r["energy"],
               "energy_fp64_evaluation": r["energy_fp64_evaluation"],
               "closing_fp64_sweep_s": r["closing_sweep_s"],
               "energy_after_closing_fp64_sweep": r["energy_closed"]}
        if "fp64" in res:
            e64, e64p = res["fp64"]["energy"], res["fp64"]["energy_plus1"]
            acc.update({"energy_fp64_same_sweeps": e64, "energy_fp64_one_more_sweep": e64p,
                        "dE_per_site_timed_result": abs(r["energy_fp64_evaluation"] - e64) / n,
                        "dE_per_site_mixed_sweeps_own_energy": abs(r["energy"] - e64) / n,
                        "dE_per_site_after_closing_sweep": abs(r["energy_closed"] - e64p) / n,
                        "target_dE_per_site": 1e-9,
                        "meets_target": abs(r["energy_fp64_evaluation"] - e64) / n <= 1e-9,
                        "speedup_vs_fp64": vmx / line["fp64"]["value"],
                        "speedup_definition": "same K sweeps from the same freshly grown state: FP64 sweep time "
                                              "over precision-form sweep time including its FP64 final energy "
                                              "evaluation"})
        if "time_to_accuracy" in res:
            acc["time_to_accuracy"] = res["time_to_accuracy"]
        line["accuracy"] = acc
    else:
        line.update({"value": line["fp64"]["value"], "ms_per_step": line["fp64"]["ms_per_step"],
                     "dtype": "complex128", "gpu_launches": line["fp64"]["gpu_launches"],
                     "roofline": line["fp64"]["roofline"], "chain": line["fp64"]["chain"]})
    log("e2e done")
    if world == 1 and not args.no_config3:
        line["config3_spin1"] = guarded_sample(config3_spin1_sample, args)
        log("config3 sample: %.1f s" % line["config3_spin1"]["sample_wall_s"])
    if world == 1 and not args.no_batched:
        line["batched"] = guarded_sample(batched_sample, args)
        log("batched sample: %.1f s" % line["batched"]["sample_wall_s"])
    if world == 1 and not args.no_serving:
        line["serving"] = guarded_sample(serving_sample, args)
        log("serving sample: %.1f s" % line["serving"]["sample_wall_s"])
    if world == 1 and not args.no_cpu_baseline:
        validation = None
        if not args.no_cpu_validation:
            # the chain's converged state at chi=128 for the oracle's measured sweep segment
            small = Chain(ops, initial_bandwidth_dimension=128, seed=args.seed + 17)
            for _ in range(3):
                small.perform_optimization_sweep()
            validation = cpu_validation(ops, small.state_sites(), args.cpu_validation_s)
            del small
        line["cpu_baseline"] = cpu_baseline(args.sites, args.chi, validation)
        log("cpu baseline done")
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("nccl", timeout=datetime.timedelta(minutes=30))
    try:
        if args.heff_only:
            run_heff_only(args)
        elif args.tc_gemm_only:
            run_tc_gemm_only(args)
        elif args.config3_only:
            import torch
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            print(json.dumps({"config3": config3_spin1_sample(args)}), flush=True)
        elif args.batched_only:
            print(json.dumps({"batched": batched_sample(args)}), flush=True)
        elif args.serving_only:
            import torch
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            print(json.dumps({"serving": serving_sample(args)}), flush=True)
        elif args.gauge_only:
            run_gauge_only(args)
        elif args.impl == "reference":
            run_reference(args, rank)
        else:
            run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as td
            td.destroy_process_group()


if __name__ == "__main__":
    main()
