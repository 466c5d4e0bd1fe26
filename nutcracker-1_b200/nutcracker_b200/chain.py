"""Device-resident chain (ctypes over the Level-1 C-ABI).

Mirrors ``Nutcracker::Chain`` (includes/nutcracker/chain.hpp:115-235) and
``ChainOptions`` (chain_options.hpp:11-48): the operator is copied to the
GPU once, every site / environment / projector stays in HBM, and the sweep
methods run the reference's control flow over the CUDA kernels.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import C128, NutcrackerError, _check, lib


class nc_chain_options(ct.Structure):
    _fields_ = [
        ("maximum_number_of_iterations", ct.c_uint32),
        ("sanity_check_threshold", ct.c_double),
        ("site_convergence_threshold", ct.c_double),
        ("sweep_convergence_threshold", ct.c_double),
        ("chain_convergence_threshold", ct.c_double),
        ("initial_bandwidth_dimension", ct.c_uint32),
        ("bandwidth_increment", ct.c_uint32),
        ("optimizer_mode", ct.c_char * 4),
        ("krylov_dimension", ct.c_uint32),
        ("seed", ct.c_uint64),
        ("strict", ct.c_uint32),
        ("time_phases", ct.c_uint32),
        ("precision", ct.c_uint32),
        ("maximum_sweeps", ct.c_uint32),
    ]


class nc_operator_site(ct.Structure):
    _fields_ = [
        ("physical_dimension", ct.c_uint32),
        ("left_dimension", ct.c_uint32),
        ("right_dimension", ct.c_uint32),
        ("number_of_matrices", ct.c_uint32),
        ("indices", ct.POINTER(ct.c_uint32)),
        ("matrices", ct.c_void_p),
    ]


class nc_chain_info(ct.Structure):
    _fields_ = [
        ("number_of_sites", ct.c_uint32),
        ("current_site", ct.c_uint32),
        ("bandwidth_dimension", ct.c_uint32),
        ("maximum_bandwidth_dimension", ct.c_uint32),
        ("number_of_projectors", ct.c_uint32),
        ("sweeps", ct.c_uint64),
        ("site_solves", ct.c_uint64),
        ("matvecs", ct.c_uint64),
        ("moves", ct.c_uint64),
        ("failures", ct.c_uint64),
        ("last_failure", ct.c_int32),
        ("energy", ct.c_double),
        ("seconds_solve", ct.c_double),
        ("seconds_gauge", ct.c_double),
        ("seconds_environment", ct.c_double),
        ("seconds_projector", ct.c_double),
        ("mixed_sweeps", ct.c_uint64),
        ("precision", ct.c_uint32),
    ]


lib.nc_chain_create.restype = ct.c_void_p
lib.nc_chain_create.argtypes = [ct.c_uint32, ct.POINTER(nc_operator_site), ct.POINTER(nc_chain_options)]
lib.nc_chain_free.argtypes = [ct.c_void_p]
for _f in ("nc_chain_reset", "nc_chain_optimize_site", "nc_chain_perform_optimization_sweep",
           "nc_chain_sweep_until_converged", "nc_chain_optimize_chain",
           "nc_chain_construct_and_add_projector_from_state"):
    getattr(lib, _f).argtypes = [ct.c_void_p]
    getattr(lib, _f).restype = ct.c_int
lib.nc_chain_increase_bandwidth_dimension.argtypes = [ct.c_void_p, ct.c_uint32]
lib.nc_chain_move_to.argtypes = [ct.c_void_p, ct.c_uint32]
lib.nc_chain_set_precision.argtypes = [ct.c_void_p, ct.c_uint32]
lib.nc_chain_solve_for_eigenvalues.argtypes = [ct.c_void_p, ct.c_uint32, ct.POINTER(ct.c_double)]
lib.nc_chain_solve_levels_at_bandwidth.argtypes = [ct.c_void_p, ct.c_uint32, ct.POINTER(ct.c_double)]
lib.nc_chain_serialize_state.restype = ct.c_size_t
lib.nc_chain_serialize_state.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_size_t]
lib.nc_chain_deserialize_state.argtypes = [ct.c_void_p, ct.c_char_p, ct.c_size_t]
SIGNAL_FN = ct.CFUNCTYPE(None, ct.c_void_p, ct.c_int, ct.c_int64, ct.c_void_p)
lib.nc_chain_connect.restype = ct.c_int64
lib.nc_chain_connect.argtypes = [ct.c_void_p, ct.c_int, SIGNAL_FN, ct.c_void_p]
lib.nc_chain_disconnect.argtypes = [ct.c_void_p, ct.c_int64]
# signal numbers (include/nutcracker_b200.h)
SIGNALS = {"optimize_site_success": 1, "optimize_site_failure": 2, "sweep_performed": 3,
           "sweeps_converged": 4, "chain_optimized": 5, "chain_reset": 6}
lib.nc_chain_get_energy.argtypes = [ct.c_void_p, ct.POINTER(ct.c_double)]
lib.nc_chain_compute_expectation_value.argtypes = [ct.c_void_p, ct.POINTER(ct.c_double)]
lib.nc_chain_get_info.argtypes = [ct.c_void_p, ct.POINTER(nc_chain_info)]
lib.nc_chain_get_site.argtypes = [ct.c_void_p, ct.c_uint32, ct.c_void_p, ct.POINTER(ct.c_uint32)]
lib.nc_chain_set_state.argtypes = [ct.c_void_p, ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_void_p)]


class ChainOptions:
    """chain_options.cpp:21-30 defaults; keyword overrides."""

    def __init__(self, **kw):
        self._o = nc_chain_options()
        lib.nc_chain_options_init(ct.byref(self._o))
        for k, v in kw.items():
            if k == "optimizer_mode":
                v = v.encode() if isinstance(v, str) else v
            if not hasattr(self._o, k):
                raise AttributeError(k)
            setattr(self._o, k, v)

    def __getattr__(self, k):
        return getattr(self._o, k)


def _operator_structs(operator):
    keep = []
    arr = (nc_operator_site * len(operator))()
    for i, s in enumerate(operator):
        idx = np.asfortranarray(np.asarray(s.idx, dtype=np.uint32))
        W = np.asfortranarray(np.asarray(s.W, dtype=C128))
        keep += [idx, W]
        arr[i].physical_dimension = int(s.d)
        arr[i].left_dimension = int(s.cl)
        arr[i].right_dimension = int(s.cr)
        arr[i].number_of_matrices = int(W.shape[2])
        arr[i].indices = idx.ctypes.data_as(ct.POINTER(ct.c_uint32))
        arr[i].matrices = W.ctypes.data
    return arr, keep


class Chain:
    """Nutcracker::Chain on the GPU.  ``operator`` is a sequence of sites with
    attributes d, cl, cr, idx (2,nnz uint32, 1-based) and W (d,d,nnz)."""

    def __init__(self, operator, options=None, **kw):
        self.options = options if options is not None else ChainOptions(**kw)
        arr, keep = _operator_structs(operator)
        self.number_of_sites = len(operator)
        h = lib.nc_chain_create(len(operator), arr, ct.byref(self.options._o))
        if not h:
            _check()
            raise NutcrackerError(-1, "nc_chain_create failed")
        self._h = ct.c_void_p(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.nc_chain_free(h)
            self._h = None

    def _call(self, fn, *args):
        st = fn(self._h, *args)
        if st != 0:
            _check()
            raise NutcrackerError(st, "chain call failed")

    # -- checkpoint / resume (StateBuffer layout of nutcracker.proto) -----------
    def serialize_state(self):
        n = lib.nc_chain_serialize_state(self._h, None, 0)
        if n == 0:
            _check()
        buf = ct.create_string_buffer(n)
        if lib.nc_chain_serialize_state(self._h, buf, n) != n:
            _check()
        return buf.raw

    def deserialize_state(self, data):
        self._call(lib.nc_chain_deserialize_state, data, len(data))

    # -- signals (base_chain.hpp:54-60, chain.hpp:151) ------------------------
    def connect(self, signal, callback):
        """Call ``callback(value)`` on ``signal`` (a key of SIGNALS); returns a
        connection id for ``disconnect``."""
        fn = SIGNAL_FN(lambda _h, _s, value, _u: callback(value))
        cid = lib.nc_chain_connect(self._h, SIGNALS[signal], fn, None)
        if cid < 0:
            _check()
        self.__dict__.setdefault("_slots", {})[cid] = fn   # keep the trampoline alive
        return cid

    def disconnect(self, cid):
        self._call(lib.nc_chain_disconnect, ct.c_int64(cid))
        self._slots.pop(cid, None)

    # -- reference API ----------------------------------------------------
    def reset(self):
        self._call(lib.nc_chain_reset)

    def set_state(self, sites):
        """Initial state: sites (br,bl,d), site 0 the centre, others right-normalised."""
        bonds = [int(sites[0].shape[1])] + [int(s.shape[0]) for s in sites]
        keep = [np.asfortranarray(np.asarray(s, dtype=C128)) for s in sites]
        b = (ct.c_uint32 * len(bonds))(*bonds)
        ptrs = (ct.c_void_p * len(keep))(*[k.ctypes.data for k in keep])
        self._call(lib.nc_chain_set_state, b, ptrs)

    def optimize_site(self):
        self._call(lib.nc_chain_optimize_site)

    def perform_optimization_sweep(self):
        self._call(lib.nc_chain_perform_optimization_sweep)

    def sweep_until_converged(self):
        self._call(lib.nc_chain_sweep_until_converged)

    def optimize_chain(self):
        self._call(lib.nc_chain_optimize_chain)

    def increase_bandwidth_dimension(self, b):
        self._call(lib.nc_chain_increase_bandwidth_dimension, ct.c_uint32(int(b)))

    def construct_and_add_projector_from_state(self):
        self._call(lib.nc_chain_construct_and_add_projector_from_state)

    def set_precision(self, precision):
        """0: FP64 sweeps; 1: precision form (3xTF32 tensor-core contractions)."""
        self._call(lib.nc_chain_set_precision, ct.c_uint32(int(precision)))

    def move_to(self, i):
        self._call(lib.nc_chain_move_to, ct.c_uint32(int(i)))

    def solve_for_eigenvalues(self, n):
        out = (ct.c_double * n)()
        self._call(lib.nc_chain_solve_for_eigenvalues, ct.c_uint32(int(n)), out)
        return list(out)

    def solve_levels_at_bandwidth(self, n):
        """n levels at the current bond dimension (nc_chain_solve_levels_at_bandwidth)."""
        out = (ct.c_double * n)()
        self._call(lib.nc_chain_solve_levels_at_bandwidth, ct.c_uint32(int(n)), out)
        return list(out)

    def get_energy(self):
        e = ct.c_double()
        self._call(lib.nc_chain_get_energy, ct.byref(e))
        return e.value

    def compute_expectation_value(self):
        e = ct.c_double()
        self._call(lib.nc_chain_compute_expectation_value, ct.byref(e))
        return e.value

    def info(self):
        i = nc_chain_info()
        self._call(lib.nc_chain_get_info, ct.byref(i))
        return {k: getattr(i, k) for k, _ in nc_chain_info._fields_}

    def get_site(self, i):
        dims = (ct.c_uint32 * 3)()
        self._call(lib.nc_chain_get_site, ct.c_uint32(int(i)), None, dims)
        out = np.zeros((dims[0], dims[1], dims[2]), C128, order="F")
        self._call(lib.nc_chain_get_site, ct.c_uint32(int(i)), ct.c_void_p(out.ctypes.data), dims)
        return out

    def state_sites(self):
        return [self.get_site(i) for i in range(self.number_of_sites)]
