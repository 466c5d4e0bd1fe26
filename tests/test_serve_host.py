"""Host-side logic of the serving loop (no GPU): the per-request device
footprint estimate that drives admission grows with the bond dimension, the
number of levels and the chain length, and stays in a sane range."""
from oracle import mpo


def test_footprint_estimate_monotone():
    from nutcracker_b200.serve import footprint_bytes

    ops = mpo.transverse_ising_ferro(16, 1.0)
    f16 = footprint_bytes(ops, levels=1, initial_bandwidth_dimension=16)
    f64 = footprint_bytes(ops, levels=1, initial_bandwidth_dimension=64)
    f64l3 = footprint_bytes(ops, levels=3, initial_bandwidth_dimension=64)
    longer = footprint_bytes(mpo.transverse_ising_ferro(32, 1.0), levels=1, initial_bandwidth_dimension=64)
    assert 0 < f16 < f64 < f64l3
    assert longer > f64
    # a 16-site chi=64 chain is a few MB of tensors plus a fixed 64 MiB margin
    assert (64 << 20) < f64 < (1 << 30)


def test_footprint_caps_bandwidth_at_chain_maximum():
    from nutcracker_b200.serve import footprint_bytes

    ops = mpo.transverse_ising_ferro(6, 1.0)   # maximum bond dimension 8
    assert footprint_bytes(ops, initial_bandwidth_dimension=8) == footprint_bytes(ops, initial_bandwidth_dimension=500)
