"""The C-ABI library loads on a CPU-only host and exports every declared symbol."""
import ctypes
import os

from ibis_b200 import build, lib


def test_library_exports_every_declared_symbol():
    path = build.build()          # no-op when the in-tree library is current
    assert os.path.exists(path)
    so = ctypes.CDLL(path)
    names = lib.declared_symbols()
    assert "ibis_step_f32" in names and "ibis_step_f64" in names
    for name in names:
        assert hasattr(so, name), name
    assert set(names) <= set(lib.SIGNATURES), set(names) - set(lib.SIGNATURES)


def test_loader_sets_prototypes():
    L = lib.load()
    assert L.ibis_step_f32.restype is ctypes.c_int
    assert len(L.ibis_step_f32.argtypes) == 11
