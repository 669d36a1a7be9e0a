"""CPU-only checks of the drop-in boundary: the shared library loads without a GPU, exports
every entry point the C header declares, and the Python binding covers them all."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "tomogpi_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tomo_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    from tomogpi_b200 import _lib

    lib = _lib.load()
    missing = [f for f in header_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_binding_covers_header():
    from tomogpi_b200 import _lib

    assert set(header_functions()) == set(_lib.SIGNATURES), set(header_functions()) ^ set(_lib.SIGNATURES)


def test_version_and_error_text_without_gpu():
    from tomogpi_b200 import _lib

    lib = _lib.load()
    assert b"sm_100a" in lib.tomo_version()
    assert isinstance(lib.tomo_last_error(), bytes)


def test_invalid_arguments_are_rejected_before_any_device_work():
    import ctypes

    from tomogpi_b200 import ConfigCT, _lib

    lib = _lib.load()
    out = ctypes.c_void_p()
    bad = _lib.config_struct(ConfigCT.cone_beam(16, 8).replace(projection_nb=0))
    assert lib.tomo_context_create(ctypes.byref(bad), 0, ctypes.byref(out)) == 1  # TOMO_ERR_INVALID
    assert b"positive" in lib.tomo_last_error()
    assert lib.tomo_context_create(None, 0, ctypes.byref(out)) == 1
    assert lib.tomo_project(None, 0, None, 0, None, 0, None) == 1
    huge = _lib.config_struct(ConfigCT.cone_beam(2048, 8))
    assert lib.tomo_context_create(ctypes.byref(huge), 0, ctypes.byref(out)) == 1
    with pytest.raises(_lib.TomoError):
        _lib.call("tomo_laplacian", None, None, 0, 0, 0, None)


def test_no_cpu_fallback_when_library_missing(tmp_path, monkeypatch):
    import importlib

    import tomogpi_b200._lib as L

    monkeypatch.setattr(L, "LIB_PATH", tmp_path / "missing.so")
    monkeypatch.setattr(L, "_lib", None)
    with pytest.raises(L.LibraryError):
        L.load()
    importlib.reload(L)


def test_newer_entry_points_reject_bad_arguments_without_gpu():
    """View ranges, solver phases, regulariser and host-buffer entry points return
    TOMO_ERR_INVALID (1) on bad arguments before touching a device (the reference would
    exit or crash)."""
    import ctypes

    from tomogpi_b200 import ConfigCT, _lib

    lib = _lib.load()
    out = ctypes.c_void_p()
    cfg = _lib.config_struct(ConfigCT.cone_beam(16, 8))
    for begin, count in ((-1, 4), (0, 0), (5, 4), (8, 1), (0, 9)):
        assert lib.tomo_context_create_views(ctypes.byref(cfg), 0, begin, count, ctypes.byref(out)) == 1
        assert b"view range" in lib.tomo_last_error()
    assert lib.tomo_solver_set_regularizer(None, 1, 0.1) == 1
    assert lib.tomo_solver_phase(None, None, None, 1, 1, None) == 1
    dj, nrm = ctypes.c_void_p(), ctypes.c_void_p()
    assert lib.tomo_solver_buffers(None, ctypes.byref(dj), ctypes.byref(nrm)) == 1
    two = (ctypes.c_double * 2)()
    assert lib.tomo_gg_regularization(None, None, 4, 4, 4, 0.1, 1, 2, None, None) == 1
    assert lib.tomo_huber_regularization(None, None, 4, 4, 4, 0.1, 0.5, 1, 2, None, None) == 1
    assert lib.tomo_laplacian_host(0, None, None, 4, 4, 4) == 1
    v = (ctypes.c_float * 64)()
    assert lib.tomo_regularization_host(0, 7, v, v, 4, 4, 4, 0.1, 0.0, 2.0, 1, 2, two) == 1   # unknown kind
    assert lib.tomo_regularization_host(0, 0, v, v, 0, 4, 4, 0.1, 0.0, 2.0, 1, 2, two) == 1   # empty volume
    for beta in (0.5, float("nan"), float("inf")):  # the GG shape parameter is finite and >= 1
        assert lib.tomo_regularization_host(0, 0, v, v, 4, 4, 4, 0.1, 0.0, beta, 1, 2, two) == 1
        assert b"beta" in lib.tomo_last_error()
        assert lib.tomo_gg_regularization_beta(v, two, 4, 4, 4, 0.1, beta, 1, 2, two, None) == 1
    assert lib.tomo_regularization_host(0, 1, v, v, 4, 4, 4, 0.1, -1.0, 2.0, 1, 2, two) == 1  # Huber threshold < 0
    assert lib.tomo_gg_regularization_beta(None, None, 4, 4, 4, 0.1, 1.5, 1, 2, None, None) == 1
    assert lib.tomo_solver_set_gg_beta(None, 1.5) == 1
    assert lib.tomo_solver_set_weights(None, None, 0, None) == 1
