"""Parity at the workloads' own sizes, against the reference's own kernel sources built for
the host (oracle/_ref; the oracle's restatement, pinned bit for bit to that build at small
sizes, where the build is absent).

* 256^3 plain method, in full: modified Shepp-Logan, 256 views over 360 deg, 256 x 256
  detector of pitch 2, FOD 512, FDD 1024. RS projection (texture and hybrid layouts) per
  view and VI backprojection per volume within 1e-5 relative L2, ray sample counts equal;
  and the FP32 results' error against the FP64 oracle, stated.
* 512^3 iterative workload (Shepp-Logan + 5 seeded ellipsoids, 512^2 detector of pitch 2,
  FOD 1024, FDD 2048) on 16 of its 512 views, evenly spread over 360 deg (views 0, 32, ...,
  480: a 16-view scan has bit-identical angles, checked below). RS per view on the
  texture and hybrid layouts (the hybrid layout is what the benchmark's autotuner picks at
  this size), VI of those views' partial sums for 16 and 32 slices per thread, and one
  gradient iteration of the solver against the oracle's loop.

References: RS projection_ER_kernel.cuh:57-312 (projection_ERB_kernel_v1), VI
backprojection3D_kernel_16reg.cuh:350-576 (backprojection_VIB_kernel_v2_16reg), the gradient
loop Iter3D_Algo_Gradient.cu:25-223.
"""
import numpy as np
import pytest

from conftest import rel_l2, rel_l2_per_view

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.timeout(900)]

TOL = 1e-5


def _ref_ops(o):
    """(projection, backprojection, which) of the reference build, else of the restatement."""
    if o.ref_lib() is not None:
        return (lambda c, v: o.ref_project(c, o.RS, v)), (lambda c, s: o.ref_backproject(c, s)), "reference build"
    return (lambda c, v: o.project(c, o.RS, v)), (lambda c, s: o.backproject(c, s)), "oracle restatement"


def _worst(got, ref):
    errs = rel_l2_per_view(got, ref)
    return max(errs), int(np.argmax(errs))


@pytest.fixture(scope="module")
def plain256(oracle_mod):
    from tomogpi_b200 import ConfigCT, phantoms

    o = oracle_mod
    cfg = ConfigCT.cone_beam(256, 256, det=256, pitch=2.0, fod=512.0, magnification=2.0)
    vol = o.phantom(phantoms.modified_shepp_logan(), 256, 256, 256)
    proj, back, which = _ref_ops(o)
    sino = proj(cfg, vol)
    return cfg, vol, sino, back(cfg, sino), which


def test_plain_256_rs_vi_match_reference(plain256, oracle_mod):
    import tomogpi_b200 as t

    cfg, vol, sino_ref, back_ref, which = plain256
    torch.cuda.set_device(0)
    with t.Context(cfg) as ctx:
        v = torch.from_numpy(vol).cuda()
        for layout in ("tex", "hybrid", "march"):
            ctx.set_tuning(rs_layout=layout)
            worst, at = _worst(ctx.project("RS", v).cpu().numpy(), sino_ref)
            print(f"256^3 RS {layout} vs {which}: worst view rel L2 {worst:.3g} (view {at})")
            assert worst <= TOL, (layout, worst, at)
        assert ctx.count_samples("RS") == oracle_mod.count_samples(cfg, oracle_mod.RS)
        for zc in (1, 2):
            ctx.set_tuning(vi_zc=zc)
            err = rel_l2(ctx.backproject("VI", torch.from_numpy(sino_ref).cuda()).cpu().numpy(), back_ref)
            print(f"256^3 VI zc {zc} vs {which}: rel L2 {err:.3g}")
            assert err <= TOL, (zc, err)
        torch.cuda.synchronize()
        assert ctx.errors() == 0


def test_plain_256_fp32_error_against_fp64_oracle(plain256, oracle_mod):
    """The FP32 results of the 256^3 workload, stated against the FP64 oracle. RS: the FP32
    geometry of the reference (its prologue is FP32) rounds some chord lengths L_r to the
    other integer than FP64 does, so a few rays take one sample more or less; VI has no
    integer geometry and stays at FP32 rounding."""
    import tomogpi_b200 as t

    o = oracle_mod
    cfg, vol, sino_ref, _, _ = plain256
    with t.Context(cfg) as ctx:
        ctx.set_tuning(rs_layout="hybrid")
        s32 = ctx.project("RS", torch.from_numpy(vol).cuda()).cpu().numpy()
        b32 = ctx.backproject("VI", torch.from_numpy(sino_ref).cuda()).cpu().numpy()
    s64 = o.project(cfg, o.RS, vol.astype(np.float64), fp64=True)
    b64 = o.backproject(cfg, sino_ref.astype(np.float64), fp64=True)
    rs_err, vi_err = rel_l2(s32, s64), rel_l2(b32, b64)
    worst, at = _worst(s32, s64)
    print(f"256^3 FP32 vs FP64 oracle: RS rel L2 {rs_err:.3g} (worst view {worst:.3g}, view {at}); "
          f"VI rel L2 {vi_err:.3g}")
    assert rs_err <= 2e-4  # measured 4.2e-5 on a B200 (worst view 5.4e-5)
    assert vi_err <= 1e-5  # measured 2.7e-7


@pytest.fixture(scope="module")
def iter512(oracle_mod):
    from tomogpi_b200 import ConfigCT, phantoms

    o = oracle_mod
    full = ConfigCT.cone_beam(512, 512, det=512, pitch=2.0, fod=1024.0, magnification=2.0)
    cfg = ConfigCT.cone_beam(512, 16, det=512, pitch=2.0, fod=1024.0, magnification=2.0)
    _, a16, b16 = o.geometry_f32(cfg)
    _, a512, b512 = o.geometry_f32(full)
    assert np.array_equal(a16, a512[::32]) and np.array_equal(b16, b512[::32])
    vol = o.phantom(phantoms.config_phantom(1234, 512), 512, 512, 512)
    proj, back, which = _ref_ops(o)
    sino = proj(cfg, vol)
    return cfg, vol, sino, back(cfg, sino), which


def test_iterative_512_rs_vi_match_reference(iter512, oracle_mod):
    import tomogpi_b200 as t

    cfg, vol, sino_ref, back_ref, which = iter512
    torch.cuda.set_device(0)
    with t.Context(cfg) as ctx:
        v = torch.from_numpy(vol).cuda()
        for layout in ("tex", "hybrid", "march"):
            ctx.set_tuning(rs_layout=layout)
            worst, at = _worst(ctx.project("RS", v).cpu().numpy(), sino_ref)
            print(f"512^3 (16 views) RS {layout} vs {which}: worst view rel L2 {worst:.3g} (view {at})")
            assert worst <= TOL, (layout, worst, at)
        del v
        assert ctx.count_samples("RS") == oracle_mod.count_samples(cfg, oracle_mod.RS)
        s = torch.from_numpy(sino_ref).cuda()
        for zc in (1, 2):
            ctx.set_tuning(vi_zc=zc)
            err = rel_l2(ctx.backproject("VI", s).cpu().numpy(), back_ref)
            print(f"512^3 (16 views) VI zc {zc} vs {which}: rel L2 {err:.3g}")
            assert err <= TOL, (zc, err)
        torch.cuda.synchronize()
        assert ctx.errors() == 0


def test_iterative_512_gradient_iteration_matches_oracle(iter512, oracle_mod):
    """One iteration of the solver (residual projection, VI backprojection, regulariser,
    the optimal step's projection, update) at 512^3 on the hybrid layout, against the
    oracle's loop, from a non-zero iterate (the phantom scaled by 0.9, so the residual
    projection reads every layout's data)."""
    import tomogpi_b200 as t

    o = oracle_mod
    cfg, vol, sino_ref, _, _ = iter512
    x0 = (vol * np.float32(0.9)).astype(np.float32)
    ref, ref_alpha = o.simple_gradient(cfg, o.RS, x0, sino_ref, 1, 0.01, 21)
    with t.Context(cfg) as ctx:
        ctx.set_tuning(rs_layout="hybrid", vi_zc=1)
        solver = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=1, optimal_step_iteration_nb=21,
                                                regularization_parameter=0.01))
        x = torch.from_numpy(x0).cuda()
        solver.iterate(x, torch.from_numpy(sino_ref).cuda())
        got = x.cpu().numpy()
        alphas = solver.alphas()
        solver.close()
    err = rel_l2(got - x0, ref - x0)
    print(f"512^3 (16 views) one gradient iteration: alpha {alphas[0]:.9g} vs {ref_alpha[0]:.9g}, "
          f"update rel L2 {err:.3g}, iterate rel L2 {rel_l2(got, ref):.3g}")
    assert np.allclose(alphas, ref_alpha, rtol=1e-5, atol=0)
    assert err <= 1e-4
    assert rel_l2(got, ref) <= TOL
