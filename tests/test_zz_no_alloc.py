"""tomo_project_noalloc: the RS projection for callers that cannot call cudaMalloc.

Such callers (a host framework whose memory pool owns every device allocation, or real-time
code that must not allocate once it runs) pass their own input and output buffers and the
geometry; the entry point keeps its scratch (padded volume, view tables) in static device
arrays of the library. Checked here through the C-ABI on two calls in a row whose sizes
differ, so that the second call would see stale data from the first if the shared scratch
were not cleared:
* against the allocating entry point (tomo_project on a context): bit-identical, since
  every RS volume layout computes the same samples with the same arithmetic;
* against the oracle (the CPU restatement of the reference's RS kernels): 1e-5 relative L2
  per projection, the tolerance of the other parity tests.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2_per_view

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


def _noalloc(lib, cfg, kind, vol, sino, device=0):
    from tomogpi_b200 import _lib

    st = torch.cuda.current_stream().cuda_stream
    return lib.tomo_project_noalloc(ctypes.byref(_lib.config_struct(cfg)), device, kind,
                                    ctypes.c_void_p(vol.data_ptr()), ctypes.c_void_p(sino.data_ptr()),
                                    ctypes.c_void_p(st))


def test_noalloc_projection_matches_allocating_entry_point_and_oracle(oracle_mod):
    import tomogpi_b200 as t
    from tomogpi_b200 import _lib

    lib = _lib.load()
    torch.cuda.set_device(0)
    cases = [(t.ConfigCT.cone_beam(40, 24, det=44), _lib.PROJ_RS, oracle_mod.RS, 1),
             (t.ConfigCT.cone_beam(24, 12, det=28, fod=30.0), _lib.PROJ_RS_UM, oracle_mod.RS_UM, 2)]
    for cfg, kind, okind, seed in cases:  # two calls in a row, the second one smaller
        g = torch.Generator(device="cuda:0").manual_seed(seed)
        vol = torch.rand(cfg.volume_shape, device="cuda:0", generator=g) + 0.5
        got = torch.full(cfg.sinogram_shape, float("nan"), device="cuda:0")
        assert _noalloc(lib, cfg, kind, vol, got) == _lib.TOMO_OK, lib.tomo_last_error()
        assert torch.cuda.current_device() == 0
        with t.Context(cfg) as ctx:
            ref = ctx.project(kind, vol)
        torch.cuda.synchronize()
        got_h, ref_h = got.cpu().numpy(), ref.cpu().numpy()
        assert np.array_equal(got_h, ref_h), float(np.abs(got_h - ref_h).max())
        errs = rel_l2_per_view(got_h, oracle_mod.project(cfg, okind, vol.cpu().numpy()))
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
    assert _noalloc(lib, t.ConfigCT.cone_beam(16, 8), _lib.PROJ_RS, dummy, dummy, device=-1) == 1
