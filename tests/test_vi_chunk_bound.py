"""The VI backprojector skips the per-sample bounds test for a chunk of 16 slices when
the first sample and vn + 16 A lie inside the detector (csrc/vi_device.cuh). This checks
the bound the way the kernel computes it, in exactly rounded FP32 (numpy float32): whenever
the chunk qualifies, every one of its 16 samples is inside, for the repeated-addition rows
(backprojection3D_kernel_16reg.cuh:410) and the k*A rows of the UM variant."""
import numpy as np

f32 = np.float32


def _qualifies(vn, A, nv):
    return (A > f32(0.25) and f32(nv) <= f32(8192) and f32(vn - f32(0.5)) > f32(-1)
            and f32(vn + f32(f32(16) * A)) < f32(nv))


def test_chunk_bound_holds_in_fp32():
    rng = np.random.default_rng(7)
    checked = 0
    for _ in range(20000):
        nv = int(rng.integers(1, 8193))
        A = f32(rng.uniform(0.25, 4.0))
        vn = f32(rng.uniform(-2.0, nv + 2.0))
        if not _qualifies(vn, A, nv):
            continue
        checked += 1
        v = vn
        for k in range(16):
            vb_add = f32(v - f32(0.5))                               # repeated addition
            vb_um = f32(f32(vn + f32(f32(k) * A)) - f32(0.5))        # k * A
            for vb in (vb_add, vb_um):
                assert vb > f32(-1) and vb < f32(nv), (nv, A, vn, k, vb)
            v = f32(v + A)
    assert checked > 1000


def test_chunk_bound_edges():
    # a chunk ending exactly at the last row does not qualify (the bound is strict and
    # conservative); one starting at the first row does
    assert not _qualifies(f32(0.6), f32(1.0), 16)         # vn + 16 A = 16.6 >= nv
    assert _qualifies(f32(0.6), f32(1.0), 17)
    assert not _qualifies(f32(-0.6), f32(1.0), 64)        # first sample below -1
    assert not _qualifies(f32(10.0), f32(0.2), 64)        # A too small for the margin
