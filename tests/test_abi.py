"""The C-ABI library loads without a GPU and exports every symbol include/homelbm.h declares."""
import ctypes

from openhomelbm_b200 import _lib


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.declared_symbols()
    assert len(declared) >= 16
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, f"declared but not exported: {missing}"


def test_every_declared_symbol_has_a_binding_signature():
    assert set(_lib.declared_symbols()) <= set(_lib._SIGS), set(_lib.declared_symbols()) - set(_lib._SIGS)


def test_version_and_error_string_need_no_gpu():
    lib = _lib.load()
    assert b"sm_100a" in lib.hl_version()
    assert isinstance(lib.hl_last_error(), bytes)


def test_argument_errors_are_reported_without_touching_the_gpu():
    lib = _lib.load()
    w = _lib.hl_world3d()
    w.nx, w.ny, w.nz = 0, 4, 4
    rc = lib.hl_d3q27_stream_collide(ctypes.byref(w), 0.1, None, None)
    assert rc == _lib.HL_ERR_ARG
    assert b"bad dims" in lib.hl_last_error()
    w2 = _lib.hl_world2d()
    w2.nx, w2.ny = 8, 8
    rc = lib.hl_d2q9_step(ctypes.byref(w2), ctypes.byref(_lib.hl_step2d(0.1, 0.0, 0.0)), None, None, None)
    assert rc == _lib.HL_ERR_ARG
