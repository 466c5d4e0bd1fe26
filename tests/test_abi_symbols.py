"""The C-ABI library loads on a CPU-only host and exports every declared symbol."""
import ctypes
import os

from abi_symbols import ROOT, declared_symbols

LIB = os.path.join(ROOT, "nutcracker-1_b200", "lib", "libnutcracker_b200.so")


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build the library first (__graft_entry__.build())"
    lib = ctypes.CDLL(LIB)
    names = declared_symbols()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_import_without_gpu():
    import nutcracker_b200 as nb
    assert "sm_100a" in nb.version()
    assert nb.lib.nc_last_status() == 0
