"""Batched form: many independent chains swept in lockstep on one GPU.

ctypes binding of ``nc_batch_*`` (include/nutcracker_b200.h).  Every chain
(its own operator, number of sites and bond dimension) runs the reference's
single-site sweep until its sweep energy settles; each contraction stage of
all chains is one persistent grouped launch, and one Lanczos iteration of all
chains is one CUDA graph replay.

Tile shapes come from the autotuner's table (``tuning/batched_tiles.json``,
written by :func:`autotune`): one entry per (stage, bond dimension, MPO bond
dimension, physical dimension) with the tile configuration that timed
fastest on the GPU.
"""
from __future__ import annotations

import ctypes as ct
import json
import os

from . import NutcrackerError, _check, lib
from .chain import _operator_structs, nc_operator_site

TILE_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "batched_tiles.json")
STAGES = ("heff_first", "heff_last", "env_left", "env_right_first", "env_right_last", "absorb")


class nc_batch_options(ct.Structure):
    _fields_ = [
        ("precision", ct.c_uint32),
        ("refine", ct.c_uint32),
        ("krylov_dimension", ct.c_uint32),
        ("maximum_number_of_iterations", ct.c_uint32),
        ("sanity_check_threshold", ct.c_double),
        ("site_convergence_threshold", ct.c_double),
        ("sweep_convergence_threshold", ct.c_double),
        ("maximum_sweeps", ct.c_uint32),
        ("seed", ct.c_uint64),
        ("time_phases", ct.c_uint32),
    ]


class nc_batch_chain_result(ct.Structure):
    _fields_ = [
        ("energy", ct.c_double),
        ("sweeps", ct.c_uint32), ("mixed_sweeps", ct.c_uint32), ("fp64_sweeps", ct.c_uint32),
        ("converged", ct.c_uint32), ("bandwidth_dimension", ct.c_uint32), ("reserved", ct.c_uint32),
        ("site_solves", ct.c_uint64),
    ]


class nc_batch_stats(ct.Structure):
    _fields_ = [
        ("chains", ct.c_uint32), ("reserved", ct.c_uint32),
        ("global_steps", ct.c_uint64), ("lanczos_iterations", ct.c_uint64),
        ("graph_launches", ct.c_uint64), ("kernel_launches", ct.c_uint64),
        ("device_bytes", ct.c_uint64), ("seconds", ct.c_double),
        ("seconds_moves", ct.c_double), ("seconds_solves", ct.c_double),
        ("continued_solves", ct.c_uint64), ("max_iterations_per_step", ct.c_uint64),
        ("seconds_replays", ct.c_double),
    ]


lib.nc_batch_options_init.argtypes = [ct.POINTER(nc_batch_options)]
lib.nc_batch_create.restype = ct.c_void_p
lib.nc_batch_create.argtypes = [ct.c_uint32, ct.POINTER(ct.c_uint32), ct.POINTER(ct.POINTER(nc_operator_site)),
                                ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint64), ct.POINTER(nc_batch_options)]
lib.nc_batch_free.argtypes = [ct.c_void_p]
lib.nc_batch_set_tile_table.argtypes = [ct.c_void_p, ct.POINTER(ct.c_int32), ct.c_uint32]
lib.nc_batch_solve.argtypes = [ct.c_void_p]
lib.nc_batch_get_results.argtypes = [ct.c_void_p, ct.POINTER(nc_batch_chain_result)]
lib.nc_batch_get_stats.argtypes = [ct.c_void_p, ct.POINTER(nc_batch_stats)]
lib.nc_batch_autotune_stage.argtypes = [ct.c_uint32] * 7 + [ct.POINTER(ct.c_double)]
lib.nc_batch_tile_configs.restype = ct.c_uint32
lib.nc_batch_tile_configs.argtypes = [ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int32)]


def tile_configs():
    """The tile shapes (rows, cols) of the grouped GEMM, by configuration index."""
    n = lib.nc_batch_tile_configs(None, None)
    r, c = (ct.c_int32 * n)(), (ct.c_int32 * n)()
    lib.nc_batch_tile_configs(r, c)
    return [(r[i], c[i]) for i in range(n)]


def load_tile_table(path=TILE_TABLE):
    """Entries (stage, chi, D, d, cfg) of the committed autotuner table
    ([] when the file is absent)."""
    if not os.path.exists(path):
        return []
    with open(path) as f:
        doc = json.load(f)
    ncfg = len(tile_configs())
    out = []
    for e in doc.get("entries", []):
        stage = STAGES.index(e["stage"])
        cfg = int(e["cfg"])
        if not 0 <= cfg < ncfg:
            raise ValueError("tile table entry with an unknown configuration: %r" % (e,))
        out.append((stage, int(e["chi"]), int(e["D"]), int(e["d"]), cfg))
    return out


def autotune(chis=(8, 16, 32, 64, 128), D=5, d=2, problems=256, reps=20, precision=1, path=None):
    """Times every tile configuration of every stage at each bond dimension
    (one grouped launch of `problems` interior-site products) and returns the
    table document; writes it to `path` when given."""
    shapes = tile_configs()
    entries = []
    for chi in chis:
        for si, stage in enumerate(STAGES):
            secs = (ct.c_double * len(shapes))()
            if lib.nc_batch_autotune_stage(si, int(chi), int(D), int(d), int(problems), int(reps), int(precision),
                                           secs) != 0:
                _check()
            times = [secs[i] for i in range(len(shapes))]
            best = min(range(len(shapes)), key=lambda i: times[i])
            entries.append({"stage": stage, "chi": int(chi), "D": int(D), "d": int(d), "cfg": best,
                            "tile": list(shapes[best]),
                            "us_per_launch": [round(t * 1e6, 3) for t in times]})
    doc = {"problems_per_launch": int(problems), "precision": int(precision), "entries": entries}
    if path:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(doc, f, indent=1)
            f.write("\n")
    return doc


class Batch:
    """A batch of chains.  ``operators`` is a sequence of operators (each a
    sequence of sites with d, cl, cr, idx, W), ``bandwidths`` their bond
    dimensions, ``seeds`` optional per-chain seeds."""

    def __init__(self, operators, bandwidths, seeds=None, tile_table=None, **options):
        o = nc_batch_options()
        lib.nc_batch_options_init(ct.byref(o))
        for k, v in options.items():
            if k not in dict(nc_batch_options._fields_):
                raise AttributeError(k)
            setattr(o, k, v)
        n = len(operators)
        if n == 0 or len(bandwidths) != n or (seeds is not None and len(seeds) != n):
            raise ValueError("one bond dimension (and seed) per chain")
        self._keep = []
        arrs = (ct.POINTER(nc_operator_site) * n)()
        nsites = (ct.c_uint32 * n)()
        for c, op in enumerate(operators):
            arr, keep = _operator_structs(op)
            self._keep += [arr, keep]
            arrs[c] = ct.cast(arr, ct.POINTER(nc_operator_site))
            nsites[c] = len(op)
        bw = (ct.c_uint32 * n)(*[int(b) for b in bandwidths])
        sd = (ct.c_uint64 * n)(*[int(s) for s in seeds]) if seeds is not None else None
        h = lib.nc_batch_create(n, nsites, arrs, bw, sd, ct.byref(o))
        if not h:
            _check()
            raise NutcrackerError(-1, "nc_batch_create failed")
        self._h = ct.c_void_p(h)
        self.n = n
        table = load_tile_table() if tile_table is None else list(tile_table)
        self.set_tile_table(table)

    def set_tile_table(self, entries):
        flat = [int(x) for e in entries for x in e]
        buf = (ct.c_int32 * max(1, len(flat)))(*flat)
        if lib.nc_batch_set_tile_table(self._h, buf, len(entries)) != 0:
            _check()

    def solve(self):
        if lib.nc_batch_solve(self._h) != 0:
            _check()
        return self.results()

    def results(self):
        r = (nc_batch_chain_result * self.n)()
        if lib.nc_batch_get_results(self._h, r) != 0:
            _check()
        return [{k: getattr(x, k) for k, _ in nc_batch_chain_result._fields_ if k != "reserved"} for x in r]

    def stats(self):
        s = nc_batch_stats()
        if lib.nc_batch_get_stats(self._h, ct.byref(s)) != 0:
            _check()
        return {k: getattr(s, k) for k, _ in nc_batch_stats._fields_ if k != "reserved"}

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.nc_batch_free(h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()
