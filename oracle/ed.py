"""Exact-diagonalisation oracle (TEST INFRASTRUCTURE ONLY).

Builds the dense Hamiltonian directly from the MPO sites (so the MPO reading
is exercised as well) and returns the lowest / highest levels.  Dense
``numpy.linalg.eigh`` for 2^N <= 4096; ``scipy.sparse.linalg.eigsh`` on the
sparse matrix for larger N.  Dense vectors order site 0 as the most
significant index, matching ``mps_to_dense``.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def mpo_to_matrix(ops, sparse=False):
    """H = sum over automaton paths of the Kronecker products of the applied
    matrices M (M[o2][o1] = W(o1,o2))."""
    kron = sp.kron if sparse else np.kron
    A = [sp.identity(1, dtype=complex, format="csr") if sparse else np.eye(1, dtype=complex)]
    for o in ops:
        nxt = [None] * o.cr
        for n in range(o.nnz):
            k1, k2 = int(o.idx[0, n]) - 1, int(o.idx[1, n]) - 1
            if k1 >= len(A) or A[k1] is None:
                continue
            M = o.W[:, :, n].T
            if sparse:
                M = sp.csr_matrix(M)
            term = kron(A[k1], M)
            nxt[k2] = term if nxt[k2] is None else nxt[k2] + term
        A = nxt
    return A[0]


def lowest_levels(ops, k=4, which="SA"):
    dim = int(np.prod([o.d for o in ops]))
    if dim <= 4096:
        H = mpo_to_matrix(ops)
        w, V = np.linalg.eigh(H)
        if which == "LA":
            return w[::-1][:k], V[:, ::-1][:, :k]
        return w[:k], V[:, :k]
    H = mpo_to_matrix(ops, sparse=True).tocsr()
    w, V = spla.eigsh(H, k=k, which=which, tol=1e-14)
    order = np.argsort(w) if which == "SA" else np.argsort(-w)
    return w[order], V[:, order]


def mps_to_dense(sites):
    """Contract an MPS (sites (br,bl,d), first..last) into a dense vector."""
    v = np.ones((1, 1), dtype=complex)  # (physical prefix, bond)
    for S in sites:
        br, bl, d = S.shape
        # v_new[(P,s), r] = sum_l v[P,l] S(r,l,s)
        t = np.einsum("pl,rls->psr", v, S)
        v = t.reshape(-1, br)
    return v[:, 0]
