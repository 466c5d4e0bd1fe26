"""Chain signals (base_chain.hpp:54-60, chain.hpp:151; emitted at
base_chain.cpp:78, 104-109, 122 and chain.cpp:162, 236): counts and order of
the events of optimizeChain and solveForMultipleLevels on a small transverse
Ising chain, queries from inside a callback, and disconnection."""
import pytest

from oracle import mpo

pytestmark = pytest.mark.gpu


def test_signals_follow_the_sweeps():
    from nutcracker_b200.chain import Chain
    n = 8
    ch = Chain(mpo.transverse_ising_ferro(n, 0.7), initial_bandwidth_dimension=4, seed=5)
    events = []
    energies = []
    for name in ("optimize_site_success", "optimize_site_failure", "sweep_performed", "sweeps_converged",
                 "chain_optimized", "chain_reset"):
        ch.connect(name, lambda v, name=name: events.append((name, v)))
    ch.connect("chain_optimized", lambda v: energies.append(ch.get_energy()))
    ch.optimize_chain()
    info = ch.info()
    names = [e[0] for e in events]
    assert names[-1] == "chain_optimized" and names.count("chain_optimized") == 1
    assert names.count("sweep_performed") == info["sweeps"]
    sweeps = [v for k, v in events if k == "sweep_performed"]
    assert sweeps == list(range(1, info["sweeps"] + 1))
    solves = names.count("optimize_site_success") + names.count("optimize_site_failure")
    assert solves == info["site_solves"]
    assert sum(v for k, v in events if k == "optimize_site_success") <= info["matvecs"]
    assert names.count("sweeps_converged") >= 2   # once per bond dimension of the growth
    assert energies == [ch.get_energy()]
    # a projector level: reset emits chain_reset
    ch.construct_and_add_projector_from_state()
    ch.reset()
    assert events[-1][0] == "chain_reset"


def test_disconnect_stops_callbacks():
    from nutcracker_b200.chain import Chain
    ch = Chain(mpo.transverse_ising_ferro(6, 1.0), initial_bandwidth_dimension=4, seed=2)
    seen = []
    cid = ch.connect("sweep_performed", seen.append)
    ch.perform_optimization_sweep()
    ch.disconnect(cid)
    ch.perform_optimization_sweep()
    assert seen == [1]
    from nutcracker_b200 import NutcrackerError
    with pytest.raises(NutcrackerError):
        ch.disconnect(cid)


def test_checkpoint_and_resume_a_converged_level():
    """A converged state saved in the StateBuffer layout and loaded into a new
    chain gives the same energy, and the C API reads the same bytes as a state."""
    from nutcracker_b200 import capi
    from nutcracker_b200.chain import Chain
    ops = mpo.transverse_ising_ferro(8, 0.9)
    a = Chain(ops, initial_bandwidth_dimension=16, seed=3)
    a.sweep_until_converged()
    e = a.get_energy()
    data = a.serialize_state()
    b = Chain(ops, initial_bandwidth_dimension=2, seed=11)
    b.deserialize_state(data)
    assert abs(b.compute_expectation_value() - e) < 1e-10 * abs(e)
    assert abs(b.get_energy() - e) < 1e-10 * abs(e)
    st = capi.State.deserialize(data)
    assert abs(st.overlap(st) - 1) < 1e-10
    again = capi.State.deserialize(b.serialize_state())
    assert abs(abs(again.overlap(st)) - 1) < 1e-10
