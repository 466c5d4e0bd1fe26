"""Serving loop (continuous batching of independent MPO solves) over the C-ABI.

Thin ctypes binding of ``nc_server_*`` (include/nutcracker_b200.h): requests
queue in arrival order and start as soon as a worker (one host thread with its
own stream and device arena) is free and the request's estimated device
footprint fits in the memory budget next to the running requests.  Each
request solves ``levels`` levels at its ``initial_bandwidth_dimension``.
"""
from __future__ import annotations

import ctypes as ct

from . import NutcrackerError, _check, lib
from .chain import ChainOptions, _operator_structs, nc_operator_site, nc_chain_options

MAX_LEVELS = 8


class nc_server_options(ct.Structure):
    _fields_ = [("max_inflight", ct.c_uint32), ("memory_budget_bytes", ct.c_uint64)]


class nc_request_result(ct.Structure):
    _fields_ = [
        ("status", ct.c_int32),
        ("levels", ct.c_uint32),
        ("bandwidth_dimension", ct.c_uint32),
        ("energies", ct.c_double * MAX_LEVELS),
        ("seconds_queued", ct.c_double),
        ("seconds_run", ct.c_double),
        ("seconds_total", ct.c_double),
        ("footprint_bytes", ct.c_uint64),
        ("sweeps", ct.c_uint64),
        ("message", ct.c_char * 128),
    ]


class nc_server_stats(ct.Structure):
    _fields_ = [
        ("submitted", ct.c_uint64), ("completed", ct.c_uint64), ("failed", ct.c_uint64),
        ("in_flight", ct.c_uint64), ("queued", ct.c_uint64),
        ("p50_seconds", ct.c_double), ("p99_seconds", ct.c_double), ("mean_seconds", ct.c_double),
        ("solves_per_second", ct.c_double), ("window_seconds", ct.c_double),
        ("peak_bytes_in_flight", ct.c_uint64), ("memory_budget_bytes", ct.c_uint64),
    ]


lib.nc_server_options_init.argtypes = [ct.POINTER(nc_server_options)]
lib.nc_server_create.restype = ct.c_void_p
lib.nc_server_create.argtypes = [ct.POINTER(nc_server_options)]
lib.nc_server_submit.restype = ct.c_int64
lib.nc_server_submit.argtypes = [ct.c_void_p, ct.c_uint32, ct.POINTER(nc_operator_site),
                                 ct.POINTER(nc_chain_options), ct.c_uint32]
for _f in ("nc_server_poll", "nc_server_wait"):
    getattr(lib, _f).argtypes = [ct.c_void_p, ct.c_int64, ct.POINTER(nc_request_result)]
    getattr(lib, _f).restype = ct.c_int
lib.nc_server_drain.argtypes = [ct.c_void_p]
lib.nc_server_get_stats.argtypes = [ct.c_void_p, ct.POINTER(nc_server_stats)]
lib.nc_server_free.argtypes = [ct.c_void_p]
lib.nc_chain_footprint_bytes.argtypes = [ct.c_uint32, ct.POINTER(nc_operator_site),
                                         ct.POINTER(nc_chain_options), ct.c_uint32, ct.POINTER(ct.c_uint64)]


def _result(r):
    return {"status": r.status, "levels": r.levels, "bandwidth_dimension": r.bandwidth_dimension,
            "energies": list(r.energies[:r.levels]), "seconds_queued": r.seconds_queued,
            "seconds_run": r.seconds_run, "seconds_total": r.seconds_total,
            "footprint_bytes": r.footprint_bytes, "sweeps": r.sweeps, "message": r.message.decode()}


def footprint_bytes(operator, levels=1, **options):
    """Estimated device bytes of one request (nc_chain_footprint_bytes)."""
    arr, keep = _operator_structs(operator)
    o = ChainOptions(**options)
    out = ct.c_uint64()
    if lib.nc_chain_footprint_bytes(len(operator), arr, ct.byref(o._o), int(levels), ct.byref(out)) != 0:
        _check()
    return out.value


class Server:
    def __init__(self, max_inflight=16, memory_budget_bytes=0):
        o = nc_server_options()
        lib.nc_server_options_init(ct.byref(o))
        o.max_inflight = int(max_inflight)
        o.memory_budget_bytes = int(memory_budget_bytes)
        h = lib.nc_server_create(ct.byref(o))
        if not h:
            _check()
            raise NutcrackerError(-1, "nc_server_create failed")
        self._h = ct.c_void_p(h)

    def submit(self, operator, levels=1, **options):
        """Queue one solve; returns its id.  options are ChainOptions fields."""
        arr, keep = _operator_structs(operator)
        o = ChainOptions(**options)
        rid = lib.nc_server_submit(self._h, len(operator), arr, ct.byref(o._o), int(levels))
        if rid < 0:
            _check()
        return rid

    def poll(self, rid):
        r = nc_request_result()
        st = lib.nc_server_poll(self._h, ct.c_int64(rid), ct.byref(r))
        if st == 1:
            return None
        if st != 0:
            _check()
        return _result(r)

    def wait(self, rid):
        r = nc_request_result()
        if lib.nc_server_wait(self._h, ct.c_int64(rid), ct.byref(r)) != 0:
            _check()
        return _result(r)

    def drain(self):
        if lib.nc_server_drain(self._h) != 0:
            _check()

    def stats(self):
        s = nc_server_stats()
        if lib.nc_server_get_stats(self._h, ct.byref(s)) != 0:
            _check()
        return {k: getattr(s, k) for k, _ in nc_server_stats._fields_}

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.nc_server_free(h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()
