"""CPU oracle for the variational-MPS sweep path.

TEST INFRASTRUCTURE ONLY: a numpy/scipy restatement of the reference's
numeric core (``sources/common/core.f95``) and of its C++ sweep driver, plus
an exact-diagonalisation checker.  Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline legs of ``bench.py`` may import it; the CUDA product
path never does.
"""
