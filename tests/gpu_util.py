"""Helpers shared by the GPU parity tests."""
import numpy as np


def rand_c(rng, shape):
    return np.asfortranarray(rng.normal(size=shape) + 1j * rng.normal(size=shape))


def rel_err(got, want):
    got = np.asarray(got).ravel(order="F")
    want = np.asarray(want).ravel(order="F")
    den = max(np.linalg.norm(want), 1e-300)
    return float(np.linalg.norm(got - want) / den)


def random_mpo_site(rng, cl, cr, d, nnz):
    idx = np.asfortranarray(np.stack([rng.integers(1, cl + 1, nnz), rng.integers(1, cr + 1, nnz)]).astype(np.uint32))
    W = rand_c(rng, (d, d, nnz))
    return idx, W
