"""tomo_project_noalloc: the RS projection for callers that cannot call cudaMalloc.

Such callers (a framework that owns all device memory, code running under stream capture,
allocation-free real-time loops) pass their own input and output buffers and the geometry;
the entry point keeps its scratch (padded volume, view tables) in static device arrays of
the library. Checked here through the C-ABI against the allocating entry point
(tomo_project on a context), on two calls in a row whose sizes differ, so that a second
call would see stale data from the first if the shared scratch were not cleared.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2_per_view

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


def _noalloc(lib, cfg, kind, vol, sino):
    from tomogpi_b200 import _lib

    st = torch.cuda.current_stream().cuda_stream
    return lib.tomo_project_noalloc(ctypes.byref(_lib.config_struct(cfg)), 0, kind, ctypes.c_void_p(vol.data_ptr()),
                                    ctypes.c_void_p(sino.data_ptr()), ctypes.c_void_p(st))


def test_noalloc_projection_matches_allocating_entry_point():
    import tomogpi_b200 as t
    from tomogpi_b200 import _lib

    lib = _lib.load()
    torch.cuda.set_device(0)
    cases = [(t.ConfigCT.cone_beam(40, 24, det=44), _lib.PROJ_RS, 1),
             (t.ConfigCT.cone_beam(24, 12, det=28, fod=30.0), _lib.PROJ_RS_UM, 2)]
    for cfg, kind, seed in cases:  # two calls in a row, the second one smaller
        g = torch.Generator(device="cuda:0").manual_seed(seed)
        vol = torch.rand(cfg.volume_shape, device="cuda:0", generator=g) + 0.5
        got = torch.full(cfg.sinogram_shape, float("nan"), device="cuda:0")
        assert _noalloc(lib, cfg, kind, vol, got) == _lib.TOMO_OK, lib.tomo_last_error()
        with t.Context(cfg) as ctx:
            ref = ctx.project(kind, vol)
        torch.cuda.synchronize()
        errs = rel_l2_per_view(got.cpu().numpy(), ref.cpu().numpy())
        assert max(errs) <= TOL, max(errs)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import tomogpi_b200 as t
    from tomogpi_b200 import _lib

    lib = _lib.load()
    big = t.ConfigCT.cone_beam(256, 8)  # 258^3 padded voxels > 8 Mi
    dummy = torch.zeros(1, device="cuda:0")
    assert _noalloc(lib, big, _lib.PROJ_RS, dummy, dummy) == 1  # TOMO_ERR_INVALID
    assert b"8 Mi" in lib.tomo_last_error()
    many = t.ConfigCT.cone_beam(16, 5000)
    assert _noalloc(lib, many, _lib.PROJ_RS, dummy, dummy) == 1
    assert _noalloc(lib, t.ConfigCT.cone_beam(16, 8), _lib.PROJ_SIDDON, dummy, dummy) == 1
