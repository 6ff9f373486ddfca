"""CPU-side checks of the C ABI: the library loads and exports every entry
point the public headers declare (no device calls are made here)."""
import ctypes


def test_library_exports_every_declared_symbol():
    import tt_b200
    declared = tt_b200.declared_symbols()
    assert len(declared) > 60
    missing = [s for s in declared if not hasattr(tt_b200.lib, s)]
    assert not missing, missing


def test_errors_are_reported_without_device():
    import tt_b200
    h = ctypes.c_void_p()
    rc = tt_b200.lib.tt_qtensor_rank(None, ctypes.byref(ctypes.c_int()))
    assert rc != 0
    assert b"invalid argument" in tt_b200.lib.tt_get_last_error()
