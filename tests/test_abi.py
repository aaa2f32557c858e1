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


def test_batch_live_view_and_control_arguments_are_checked_without_the_gpu():
    """The batched, live-view and 2D control entry points reject bad arguments before any CUDA
    call: NULL buffers, empty batches, misaligned or unprepared descriptors, bad axes."""
    lib = _lib.load()
    arg = _lib.HL_ERR_ARG
    w = _lib.hl_world3d()
    w.nx, w.ny, w.nz = 16, 16, 16
    worlds = (_lib.hl_world3d * 1)(w)
    n = ctypes.c_int(0)
    assert lib.hl_d3q27_batch_bytes(0) == 0
    assert lib.hl_d3q27_batch_prepare(worlds, 0, 64, 1 << 20, ctypes.byref(n), None) == arg
    assert lib.hl_d3q27_batch_prepare(worlds, 1, 64 + 16, 1 << 20, ctypes.byref(n), None) == arg
    assert b"64-byte" in lib.hl_last_error()
    assert lib.hl_d3q27_batch_prepare(worlds, 1, 64, 8, ctypes.byref(n), None) == arg
    assert b"too small" in lib.hl_last_error()
    stor = _lib.hl_storage()
    assert lib.hl_d3q27_stream_collide_batch(4096, 1, 1, 0.02, ctypes.byref(stor), 0, None, None) == arg
    assert lib.hl_d3q27_stream_collide_batch(4096, 1, 1, 0.02, ctypes.byref(stor), 2, None, None) == arg
    assert lib.hl_d3q27_links_batch_bytes(0, 3) == 0
    solids = (_lib.hl_solids3d * 1)()
    work = ctypes.c_size_t(0)
    assert lib.hl_d3q27_links_batch_prepare(worlds, solids, 0, 0.02, 64, 1 << 20, ctypes.byref(work), None) == arg
    assert lib.hl_d3q27_links_batch_prepare(worlds, solids, 1, 0.02, 64, 1 << 20, ctypes.byref(work), None) == arg
    assert b"world" in lib.hl_last_error()  # the domain's buffers are NULL
    assert lib.hl_d3q27_solid_links_batch(64, 1, 3, 64, 1 << 20, None) == arg
    assert lib.hl_d3q27_solid_links_batch(64, 1, 0, 64, 1 << 20, None) == arg
    assert b"not prepared" in lib.hl_last_error()
    assert lib.hl_d3q27_bc_batch_bytes(0) == 0
    bcs = (_lib.hl_bc3d * 1)()
    scratch = (ctypes.c_void_p * 1)(64)
    assert lib.hl_d3q27_bc_batch_prepare(worlds, bcs, scratch, 0, 64, 1 << 20, None) == arg  # no domains
    assert lib.hl_d3q27_bc_batch_prepare(worlds, bcs, scratch, 1, 64 + 8, 1 << 20, None) == arg
    assert b"16-byte" in lib.hl_last_error()
    assert lib.hl_d3q27_bc_batch_prepare(worlds, bcs, scratch, 1, 64, 8, None) == arg
    assert b"below" in lib.hl_last_error()
    assert lib.hl_d3q27_bc_batch_prepare(worlds, bcs, scratch, 1, 64, 1 << 20, None) == arg
    assert b"NULL buffer" in lib.hl_last_error()  # the domain's buffers are NULL
    assert lib.hl_d3q27_apply_bc_batch(64, 1, 2, None) == arg
    assert lib.hl_d3q27_apply_bc_batch(64, 1, 0, None) == arg
    assert b"not prepared" in lib.hl_last_error()
    pos = (ctypes.c_int32 * 1)(3)
    assert lib.hl_d3q27_live_slices(ctypes.byref(w), pos, 1, 8, 8, 1, 0, 0, 0, 0, 64, None, None) == arg  # cur NULL
    w.cur = 64
    assert lib.hl_d3q27_live_slices(ctypes.byref(w), pos, 1, 8, 8, 1, 3, 0, 0, 0, 64, None, None) == arg
    assert b"axis" in lib.hl_last_error()
    assert lib.hl_d3q27_live_slices(ctypes.byref(w), pos, 1, 8, 8, 1, 0, 0, 0, 1, 64, None, None) == arg
    assert b"histogram" in lib.hl_last_error()
    assert lib.hl_live_rgba(None, 0, 1.0, 1.0, None, None) == _lib.HL_OK  # nothing to colour
    assert lib.hl_live_rgba(None, 4, 1.0, 1.0, None, None) == arg
    assert lib.hl_d2q9_uimg_rgba(64, 8, 8, 3, 1.0, 64, None) == arg
    assert b"render mode" in lib.hl_last_error()
    assert lib.hl_d2q9_local_force(None, None, 8, 8, 1.0, 1.0, 1.0, 1.0, 0.1, 0.0, None) == arg
    assert lib.hl_d2q9_local_force(64, 64, 0, 8, 1.0, 1.0, 1.0, 1.0, 0.1, 0.0, None) == arg


def test_round_to_storage_arguments_are_checked_without_the_gpu():
    lib = _lib.load()
    arg = _lib.HL_ERR_ARG
    assert lib.hl_round_to_storage(None, 0, 10, 1, 0, 0, None, None) == _lib.HL_OK  # nothing to round
    assert lib.hl_round_to_storage(None, 4, 10, 1, 0, 0, None, None) == arg
    assert lib.hl_round_to_storage(64, 4, 0, 1, 0, 0, 64, None) == arg
    assert lib.hl_round_to_storage(64, 4, 10, 1, -1, 0, 64, None) == arg
    assert lib.hl_round_to_storage(64, 4, 10, 9, 0, 0, 64, None) == arg
    assert b"dtype" in lib.hl_last_error()
