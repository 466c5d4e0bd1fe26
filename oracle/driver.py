"""CPU oracle: restatement of Nutcracker's site/sweep driver (C++ layer).

TEST INFRASTRUCTURE ONLY (see ``oracle/core.py``).  Follows:

* ``sources/common/optimizer.cpp:160-315``   optimizeStateSite + modes
* ``sources/common/base_chain.cpp:64-123``   optimizeSite / sweeps / optimizeChain
* ``sources/common/chain.cpp:37-310``        Chain (reset, move, sweeps, levels)
* ``includes/nutcracker/chain.hpp:248-315``  absorb / move
* ``includes/nutcracker/projectors.hpp:324-485`` projector formation
* ``sources/common/projectors.cpp:18-170``   applyProjectorMatrix, overlaps
* ``sources/common/states.cpp:94-207``       cursor moves, random sites
* ``sources/common/utilities.cpp:32-91``     bond-dimension sequence
* ``includes/nutcracker/utilities.hpp:264-283,418-420``
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import core

C = np.complex128


# ---------------------------------------------------------------------------
# utilities
# ---------------------------------------------------------------------------

def outside_tolerance(a, b, tol):
    """utilities.hpp:418-420."""
    return (abs(a) + abs(b)) / 2 > tol and abs(a - b) / (abs(a) + abs(b) + tol) > tol


class RequestedBandwidthDimensionTooLargeError(ValueError):
    pass


def compute_bandwidth_dimension_sequence(requested, phys):
    """utilities.cpp:32-91."""
    if requested == 0:
        raise ValueError("requested bandwidth must be > 0")
    middle = (len(phys) + 1) // 2

    def side(dims):
        out = [1]
        p = 1
        for d in dims[:middle]:
            p *= d
            if p >= requested:
                break
            out.append(p)
        return out

    fwd = side(list(phys))
    rev = side(list(reversed(phys)))
    if len(fwd) == middle + 1 or len(rev) == middle + 1:
        raise RequestedBandwidthDimensionTooLargeError(requested)
    seq = fwd + [requested] * (len(phys) + 1 - len(fwd) - len(rev)) + list(reversed(rev))
    return seq


def maximum_bandwidth_dimension(phys):
    """utilities.hpp:264-283."""
    if len(phys) == 1:
        return 1
    middle = (len(phys) + 1) // 2
    return min(int(np.prod(phys[:middle])), int(np.prod(list(reversed(phys))[:middle])))


def minimum_bandwidth_dimension_for_projector_count(phys, nproj):
    """projectors.cpp:108-133."""
    if nproj == 0:
        return 1
    b = 1
    while True:
        seq = compute_bandwidth_dimension_sequence(b, phys)
        for i, d in enumerate(phys):
            if d * seq[i] * seq[i + 1] > nproj:
                return b
        b += 1


# ---------------------------------------------------------------------------
# data model
# ---------------------------------------------------------------------------

@dataclass
class OperatorSite:
    """OperatorSite (tensors.hpp:1641-1854): W (d,d,nnz) column-major with
    W(o1,o2) = M[o2][o1] of the row-major link matrix M; idx (2,nnz) 1-based."""
    d: int
    cl: int
    cr: int
    idx: np.ndarray
    W: np.ndarray

    @property
    def nnz(self):
        return self.W.shape[2]


def make_operator_site(d, cl, cr, links):
    """constructOperatorSite (operators.cpp:83-112).  links: (from, to, M) with
    M a row-major d x d matrix (as written in YAML / ublas)."""
    nnz = len(links)
    idx = np.zeros((2, nnz), dtype=np.uint32, order="F")
    W = np.zeros((d, d, nnz), dtype=C, order="F")
    for n, (f, t, M) in enumerate(links):
        idx[0, n], idx[1, n] = f, t
        M = np.asarray(M, dtype=C)
        assert M.shape == (d, d)
        W[:, :, n] = M.T  # row-major copy into a column-major (d,d) slot
    return OperatorSite(d, cl, cr, idx, W)


@dataclass
class ProjectorMatrix:
    nproj: int = 0
    length: int = 0
    nrefl: int = 0
    orth_dim: int = 0
    reflectors: Optional[np.ndarray] = None
    tau: Optional[np.ndarray] = None
    swaps: Optional[np.ndarray] = None

    def valid(self):
        return self.reflectors is not None


@dataclass
class ProjectorSite:
    left: Optional[np.ndarray]
    middle: np.ndarray
    right: Optional[np.ndarray]


class OptimizerFailure(Exception):
    pass


class OptimizerUnableToConverge(OptimizerFailure):
    pass


class OptimizerGivenTooManyProjectors(OptimizerFailure):
    pass


class OptimizerGivenGuessInProjectorSpace(OptimizerFailure):
    pass


class OptimizerObtainedEigenvalueDifferentFromExpectationValue(OptimizerFailure):
    pass


class OptimizerObtainedComplexEigenvalue(OptimizerFailure):
    pass


class OptimizerObtainedVanishingEigenvector(OptimizerFailure):
    pass


class OptimizerObtainedEigenvectorInProjectorSpace(OptimizerFailure):
    pass


class OptimizerObtainedRegressiveEigenvalue(OptimizerFailure):
    pass


class OptimizerUnknownFailure(OptimizerFailure):
    pass


MODES = {
    "<v": ("SR", lambda f, t, tol: t > f and outside_tolerance(f, t, tol)),
    ">v": ("LR", lambda f, t, tol: t < f and outside_tolerance(f, t, tol)),
    ">m": ("LM", lambda f, t, tol: abs(t) < abs(f) and outside_tolerance(abs(f), abs(t), tol)),
}


@dataclass
class ChainOptions:
    """chain_options.cpp:21-30 defaults."""
    maximum_number_of_iterations: int = 10000
    sanity_check_threshold: float = 1e-12
    site_convergence_threshold: float = 1e-12
    sweep_convergence_threshold: float = 1e-12
    chain_convergence_threshold: float = 1e-12
    initial_bandwidth_dimension: int = 1
    compute_new_bandwidth_dimension: Callable[[int], int] = lambda b: b + 1
    optimizer_mode: str = "<v"
    # ARPACK's basis size; the reference fixes 3 (core.f95:2565).  Not a
    # reference option: larger values reach the same converged states with
    # fewer restarts, for oracle runs at bond dimension 64 and above.
    arpack_ncv: int = 3


# ---------------------------------------------------------------------------
# site algebra
# ---------------------------------------------------------------------------

def compute_expectation_value_at_site(L, S, op, R):
    br, bl, d = S.shape
    return core.compute_expectation(bl, br, op.cl, op.cr, d, L, S, op.idx, op.W, R)


def contract_sos_left(L, S, op):
    br, bl, d = S.shape
    return core.contract_sos_left(bl, br, op.cl, op.cr, d, L, op.idx, op.W, S)


def contract_sos_right(R, S, op):
    br, bl, d = S.shape
    return core.contract_sos_right(bl, br, op.cl, op.cr, d, R, op.idx, op.W, S)


def contract_vs_left(Lov, P, S):
    blo, d, bro = P.shape
    brn, bln, _ = S.shape
    return core.contract_vs_left(blo, bro, bln, brn, d, Lov, P, S)


def contract_vs_right(Rov, P, S):
    blo, d, bro = P.shape
    brn, bln, _ = S.shape
    return core.contract_vs_right(blo, bro, bln, brn, d, Rov, P, S)


def overlap_with_projectors(pm, S):
    if not pm.valid():
        return 0.0
    return core.compute_overlap_with_projectors(pm.nproj, pm.nrefl, pm.reflectors, pm.tau,
                                                pm.swaps, S.size, S)


def optimize_state_site(L, S, op, R, pm, tol, sanity, maxit, mode, ncv=3):
    """optimizer.cpp:201-315."""
    br, bl, d = S.shape
    which = MODES[mode][0]
    if pm.valid():
        args = (pm.nproj, pm.nrefl, pm.orth_dim, pm.reflectors, pm.tau, pm.swaps)
    else:
        args = (0, 0, S.size, None, None, None)
    status, iters, ev, new, normal = core.optimize(bl, br, op.cl, op.cr, d, L, op.idx, op.W, R,
                                                   *args, which, tol, maxit, S, ncv0=ncv)
    expectation = compute_expectation_value_at_site(L, new, op, R)
    overlap = overlap_with_projectors(pm, new)
    if status == -14:
        raise OptimizerUnableToConverge(iters)
    if status == 10:
        raise OptimizerGivenTooManyProjectors()
    if status == 11:
        raise OptimizerGivenGuessInProjectorSpace()
    if status != 0:
        raise OptimizerUnknownFailure(status)
    if outside_tolerance(ev, expectation, sanity):
        raise OptimizerObtainedEigenvalueDifferentFromExpectationValue(ev, expectation)
    if abs(ev) > sanity and abs(ev.imag) / abs(ev) > sanity:
        raise OptimizerObtainedComplexEigenvalue(ev)
    if normal < 1 - sanity:
        raise OptimizerObtainedVanishingEigenvector(normal)
    if overlap > sanity:
        raise OptimizerObtainedEigenvectorInProjectorSpace(overlap)
    return iters, ev.real, new


def move_site_cursor_right(middle, right):
    """states.cpp:130-164."""
    bm, bl, d1 = middle.shape
    brr, bm2, d2 = right.shape
    assert bm2 == bm
    info, n1, n2 = core.norm_denorm_going_right(bl, bm, brr, d1, d2, middle, right)
    n2 = n2 / np.linalg.norm(n2)
    return core.F(n2), n1  # (new middle, new left-normalized site)


def move_site_cursor_left(middle, left):
    """states.cpp:94-128: old_state_site_1 = left neighbor, old_state_site_2 = middle."""
    bm, bl, d1 = left.shape
    br, bm2, d2 = middle.shape
    assert bm2 == bm
    info, dn1, n2 = core.norm_denorm_going_left(bl, bm, br, d1, d2, left, middle)
    dn1 = dn1 / np.linalg.norm(dn1)
    return core.F(dn1), n2  # (new middle, new right-normalized site)


def apply_projector_matrix(pm, S):
    """projectors.cpp:18-38."""
    out = core.filter_components_outside_orthog(S.size, pm.nproj, pm.nrefl, pm.orth_dim,
                                                pm.reflectors, pm.tau, pm.swaps, S)
    out = np.reshape(out, S.shape, order="F")
    nrm = np.linalg.norm(out)
    assert nrm > 1e-7
    return core.F(out / nrm)


def form_projector_matrix(left_bounds, right_bounds, overlap_sites):
    """projectors.hpp:406-485."""
    nproj = len(left_bounds)
    if nproj == 0:
        return ProjectorMatrix()
    d = overlap_sites[0].shape[1]
    sl = left_bounds[0].shape[0]
    sr = right_bounds[0].shape[1]
    length = d * sl * sr
    vecs = np.zeros((length, nproj), dtype=C, order="F")
    for p, (Lov, Rov, P) in enumerate(zip(left_bounds, right_bounds, overlap_sites)):
        blo, _, bro = P.shape
        vecs[:, p] = core.form_overlap_vector(blo, bro, sl, sr, d, Lov, Rov, P).ravel(order="F")
    refl, rank, tau, swaps = core.convert_vectors_to_reflectors(length, nproj, vecs)
    return ProjectorMatrix(nproj, length, min(length, nproj), length - rank, refl, tau, swaps)


def compute_projector_from_state_sites(first, rest):
    """projectors.hpp:324-359 with projectors.cpp:60-89."""
    proj = []
    cur = first.copy(order="F")
    cur_right = None
    for nxt in rest:
        bm, bl, dl = cur.shape
        br, _, dr = nxt.shape
        lno, uno, dS2, rno = core.form_norm_overlap_tensors(bl, bm, br, dl, dr, cur, nxt)
        proj.append(ProjectorSite(lno, uno, cur_right))
        cur = dS2
        cur_right = rno
    br, bl, d = cur.shape
    proj.append(ProjectorSite(None, core.form_overlap_site_tensor(br, bl, d, cur), cur_right))
    return proj


def compute_state_overlap(sites_a, sites_b):
    """<a|b> for two MPS given as site lists (first..last), via overlap-site
    contraction (projectors.hpp:361-404 with the middle site at 0)."""
    Lov = np.ones((1, 1), dtype=C, order="F")
    for i, (A, B) in enumerate(zip(sites_a, sites_b)):
        br, bl, d = A.shape
        P = core.form_overlap_site_tensor(br, bl, d, A)
        Lov = contract_vs_left(Lov, P, B)
    return complex(Lov[0, 0])


# ---------------------------------------------------------------------------
# the chain
# ---------------------------------------------------------------------------

class InitialSiteSource:
    """Seeded stand-in for randomStateSiteRight / randomStateSiteMiddle
    (states.cpp:169-207) and the bandwidth-increase isometries."""

    def __init__(self, seed):
        self.rng = np.random.default_rng(seed)

    def right(self, d, bl, br):
        return core.rand_norm_state_site_tensor(br, bl, d, self.rng)

    def middle(self, d, bl, br):
        return core.rand_unnorm_state_site_tensor(br, bl, d, self.rng)


class ReplaySource:
    """A given state as the chain's initial sites: ``sites`` (br, bl, d), site 0
    the centre, the rest right-normalised (the layout ``state_sites`` returns),
    handed out in the order ``Chain.reset`` draws them (sites N-1 .. 1, then
    the centre).  Used to run the oracle from the device chain's state."""

    def __init__(self, sites):
        self.rights = [np.asfortranarray(s) for s in sites[1:]]
        self.centre = np.asfortranarray(sites[0])

    def right(self, d, bl, br):
        s = self.rights.pop()  # site N-1 first
        assert s.shape == (br, bl, d), (s.shape, (br, bl, d))
        return s

    def middle(self, d, bl, br):
        assert self.centre.shape == (br, bl, d), (self.centre.shape, (br, bl, d))
        return self.centre


@dataclass
class Neighbor:
    expectation_boundary: np.ndarray
    state_site: np.ndarray
    overlap_boundaries: list = field(default_factory=list)


class Chain:
    """chain.hpp:115-235 / chain.cpp / base_chain.cpp."""

    def __init__(self, operator, options=None, seed=0, source=None):
        self.options = options or ChainOptions()
        self.ops = operator
        self.N = len(operator)
        self.phys = [o.d for o in operator]
        self.maximum_bandwidth_dimension = maximum_bandwidth_dimension(self.phys)
        self.source = source or InitialSiteSource(seed)
        self.projectors: List[List[ProjectorSite]] = []
        self.on_site_success = []
        self.on_site_failure = []
        self.on_sweep = []
        self.reraise = True
        self.sweeps = 0
        self.site_solves = 0
        self.reset()

    # -- boundaries ---------------------------------------------------------
    def reset_boundaries(self):
        one = np.ones((1, 1, 1), dtype=C, order="F")
        self.left_exp = one.copy(order="F")
        self.right_exp = one.copy(order="F")
        self.left_ov = [np.ones((1, 1), dtype=C, order="F") for _ in self.projectors]
        self.right_ov = [np.ones((1, 1), dtype=C, order="F") for _ in self.projectors]

    def absorb(self, side, site, op_number):
        op = self.ops[op_number]
        if side == "L":
            new_exp = contract_sos_left(self.left_exp, site, op)
            new_ov = [contract_vs_left(b, p[op_number].left, site)
                      for b, p in zip(self.left_ov, self.projectors)]
            self.left_neighbors.append(Neighbor(self.left_exp, site, self.left_ov))
            self.left_exp, self.left_ov = new_exp, new_ov
        else:
            new_exp = contract_sos_right(self.right_exp, site, op)
            new_ov = [contract_vs_right(b, p[op_number].right, site)
                      for b, p in zip(self.right_ov, self.projectors)]
            self.right_neighbors.append(Neighbor(self.right_exp, site, self.right_ov))
            self.right_exp, self.right_ov = new_exp, new_ov

    def reset_projector_matrix(self):
        self.pm = form_projector_matrix(self.left_ov, self.right_ov,
                                        [p[self.current].middle for p in self.projectors])

    def move(self, side):
        self.optimized = False
        op_number = self.current
        if side == "R":
            self.current += 1
            nb = self.right_neighbors[-1]
            middle, other = move_site_cursor_right(self.state_site, nb.state_site)
            self.absorb("L", other, op_number)
            self.right_exp, self.right_ov = nb.expectation_boundary, nb.overlap_boundaries
            self.right_neighbors.pop()
        else:
            self.current -= 1
            nb = self.left_neighbors[-1]
            middle, other = move_site_cursor_left(self.state_site, nb.state_site)
            self.absorb("R", other, op_number)
            self.left_exp, self.left_ov = nb.expectation_boundary, nb.overlap_boundaries
            self.left_neighbors.pop()
        self.state_site = middle
        self.reset_projector_matrix()

    def move_to(self, n):
        while self.current > n:
            self.move("L")
        while self.current < n:
            self.move("R")

    def reset(self):
        """chain.cpp:175-237."""
        self.optimized = False
        self.bandwidth_dimension = min(
            self.maximum_bandwidth_dimension,
            max(self.options.initial_bandwidth_dimension,
                minimum_bandwidth_dimension_for_projector_count(self.phys, len(self.projectors))))
        self.current = 0
        self.left_neighbors = []
        self.right_neighbors = []
        self.reset_boundaries()
        dims = compute_bandwidth_dimension_sequence(self.bandwidth_dimension, self.phys)
        rdims = list(reversed(dims))
        for k, op_number in enumerate(reversed(range(1, self.N))):
            site = self.source.right(self.ops[op_number].d, rdims[k + 1], rdims[k])
            self.absorb("R", site, op_number)
        self.state_site = self.source.middle(self.ops[0].d, dims[0], dims[1])
        self.reset_projector_matrix()
        if self.projectors:
            while self.pm.orth_dim == 0:
                self.move("R")
            self.state_site = apply_projector_matrix(self.pm, self.state_site)
            self.move_to(0)
        ev = self.compute_expectation_value()
        if abs(ev.imag) / abs(ev) > 1e-10:
            raise RuntimeError("initial chain energy not real: %r" % ev)
        self.energy = ev.real
        self.energy_computed = True

    # -- energies -----------------------------------------------------------
    def compute_expectation_value(self):
        return compute_expectation_value_at_site(self.left_exp, self.state_site,
                                                 self.ops[self.current], self.right_exp)

    def get_energy(self):
        return self.energy

    # -- optimization -------------------------------------------------------
    def optimize_site(self):
        """base_chain.cpp:81-110."""
        o = self.options
        try:
            iters, ev, new = optimize_state_site(
                self.left_exp, self.state_site, self.ops[self.current], self.right_exp, self.pm,
                o.site_convergence_threshold, o.sanity_check_threshold,
                o.maximum_number_of_iterations, o.optimizer_mode, o.arpack_ncv)
            if MODES[o.optimizer_mode][1](self.energy, ev, o.sanity_check_threshold):
                raise OptimizerObtainedRegressiveEigenvalue(self.energy, ev)
            if ((self.energy >= 0 and ev >= 0) or (self.energy <= 0 and ev <= 0)
                    or outside_tolerance(abs(self.energy), abs(ev), o.sanity_check_threshold)):
                self.energy = ev
                self.state_site = new
            self.optimized = True
            self.site_solves += 1
            for cb in self.on_site_success:
                cb(iters)
        except OptimizerFailure as failure:
            for cb in self.on_site_failure:
                cb(failure)
            if self.reraise:
                raise

    def perform_optimization_sweep(self):
        """chain.cpp:147-163."""
        start = self.current
        if not self.optimized:
            self.optimize_site()
        while self.current + 1 < self.N:
            self.move("R")
            self.optimize_site()
        while self.current > 0:
            self.move("L")
            self.optimize_site()
        while self.current < start:
            self.move("R")
            self.optimize_site()
        self.sweeps += 1
        for cb in self.on_sweep:
            cb(self)

    def sweep_until_converged(self):
        """base_chain.cpp:112-123 (getConvergenceEnergy == getEnergy for Chain)."""
        prev = self.get_energy()
        self.perform_optimization_sweep()
        cur = self.get_energy()
        while outside_tolerance(prev, cur, self.options.sweep_convergence_threshold):
            self.perform_optimization_sweep()
            prev, cur = cur, self.get_energy()

    def increase_bandwidth_dimension(self, new_b):
        """chain.cpp:75-122."""
        self.optimized = False
        if new_b == self.bandwidth_dimension:
            return
        assert new_b > self.bandwidth_dimension and self.current == 0
        dims = compute_bandwidth_dimension_sequence(new_b, self.phys)
        dim_iter = iter(list(reversed(dims))[1:])
        old = self.right_neighbors
        first = self.state_site
        self.right_neighbors = []
        self.reset_boundaries()
        op_number = self.N - 1
        for k in range(len(old)):
            target = next(dim_iter)
            left_site = old[k + 1].state_site if op_number > 1 else first
            s1, s2 = self._increase_between(target, left_site, old[k].state_site)
            if op_number > 1:
                old[k + 1].state_site = s1
            else:
                self.state_site = s1
            self.absorb("R", s2, op_number)
            op_number -= 1
        self.bandwidth_dimension = new_b
        self.reset_projector_matrix()

    def _increase_between(self, new_dim, s1, s2):
        """states.hpp:386-440."""
        bm, bl, dl = s1.shape
        br, _, dr = s2.shape
        if new_dim > bm:
            info, a, b = core.increase_bandwidth_between(bl, bm, br, dl, dr, new_dim, s1, s2,
                                                         self.source.rng)
        else:
            info, a, b = core.norm_denorm_going_left(bl, bm, br, dl, dr, s1, s2)
        return a, b

    def optimize_chain(self):
        """base_chain.cpp:64-79."""
        o = self.options
        self.sweep_until_converged()
        prev = self.get_energy()
        self.increase_bandwidth_dimension(min(o.compute_new_bandwidth_dimension(self.bandwidth_dimension),
                                              self.maximum_bandwidth_dimension))
        self.sweep_until_converged()
        cur = self.get_energy()
        while (outside_tolerance(prev, cur, o.chain_convergence_threshold)
               and self.bandwidth_dimension < self.maximum_bandwidth_dimension):
            self.increase_bandwidth_dimension(min(o.compute_new_bandwidth_dimension(self.bandwidth_dimension),
                                                  self.maximum_bandwidth_dimension))
            self.sweep_until_converged()
            prev, cur = cur, self.get_energy()

    def state_sites(self):
        """Sites first..last (chain at site 0: middle + right neighbors reversed)."""
        assert self.current == 0
        return [self.state_site] + [nb.state_site for nb in reversed(self.right_neighbors)]

    def construct_and_add_projector_from_state(self):
        self.optimized = False
        assert self.current == 0
        sites = self.state_sites()
        self.projectors.append(compute_projector_from_state_sites(sites[0], sites[1:]))

    def solve_for_multiple_levels(self, n, states=None):
        """chain.cpp:301-310, recording (energy, state) per level."""
        energies = []
        for _ in range(n - 1):
            self.optimize_chain()
            energies.append(self.get_energy())
            if states is not None:
                states.append([s.copy(order="F") for s in self.state_sites()])
            self.construct_and_add_projector_from_state()
            self.reset()
        self.optimize_chain()
        energies.append(self.get_energy())
        if states is not None:
            states.append([s.copy(order="F") for s in self.state_sites()])
        return energies
