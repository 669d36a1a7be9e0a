"""Parity of the CUDA operators (through the C-ABI) with the reference.

* golden fixtures: outputs of the reference's own sources (tests/golden/make_golden.py);
* the oracle (the FP32 restatement pinned to those sources, and its FP64 mode) at other
  sizes, including ragged detector/volume sizes and odd view counts;
* FP32 tolerance: 1e-5 relative L2 per projection (per view of the sinogram) and per
  volume; ray sample counts (the integer part of the geometry) must be identical.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden, rel_l2, rel_l2_per_view

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def tomo():
    import tomogpi_b200 as t

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.set_device(0)
    return t


def _dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0", dtype=dtype)


def _check_sino(got, ref, tol=TOL):
    errs = rel_l2_per_view(got, ref)
    assert max(errs) <= tol, f"worst view rel L2 {max(errs):.3g} (view {int(np.argmax(errs))})"


@pytest.mark.parametrize("case", golden_cases())
def test_operators_match_reference_golden(tomo, case):
    cfg, d = load_golden(case)
    vol, sino = _dev(d["volume"]), _dev(d["sinogram"])
    with tomo.Context(cfg) as ctx:
        _check_sino(ctx.project("RS", vol).cpu().numpy(), d["rs"])
        _check_sino(ctx.project("RS_UM", vol).cpu().numpy(), d["rs_um"])
        if "siddon_ref" in d:
            _check_sino(ctx.project("SIDDON_REF", vol).cpu().numpy(), d["siddon_ref"])
        assert rel_l2(ctx.backproject("VI", sino).cpu().numpy(), d["vi"]) <= TOL
        assert rel_l2(ctx.backproject("VI_UM", sino).cpu().numpy(), d["vi_um"]) <= TOL
        torch.cuda.synchronize()
        assert ctx.errors() == 0


GEOMS = [
    dict(n=32, views=16, det=32),
    dict(n=32, views=7, det=40, pitch=1.5),                 # odd view count, wider detector
    dict(n=24, views=12, det=24, fod=26.0),                 # strong cone angle
    dict(nxy=32, nz=20, views=9, det=(36, 28)),             # ragged sizes, nz not a multiple of 16
    dict(n=64, views=32, det=64),
    dict(nxyz=(40, 28, 18), views=1, det=(48, 30)),         # one view, nx != ny != nz
]


def _cfg(spec):
    from tomogpi_b200 import ConfigCT

    if "nxyz" in spec:
        nx, ny, nz = spec["nxyz"]
        nu, nv = spec["det"]
        c = ConfigCT.cone_beam(nx, spec["views"], det=nu)
        return c.replace(y_volume_pixel_nb=ny, y_volume_size=float(ny), z_volume_pixel_nb=nz, z_volume_size=float(nz),
                         v_detector_pixel_nb=nv, v_detector_size=2.0 * nv)
    if "nxy" in spec:
        nu, nv = spec["det"]
        c = ConfigCT.cone_beam(spec["nxy"], spec["views"], det=nu)
        return c.replace(z_volume_pixel_nb=spec["nz"], z_volume_size=float(spec["nz"]), v_detector_pixel_nb=nv,
                         v_detector_size=2.0 * nv)
    return ConfigCT.cone_beam(spec["n"], spec["views"], det=spec["det"], pitch=spec.get("pitch", 2.0),
                              fod=spec.get("fod"))


@pytest.mark.parametrize("layout", ["plain", "cell8", "tex", "hybrid", "march"])
@pytest.mark.parametrize("spec", GEOMS, ids=lambda s: "-".join(f"{k}{v}" for k, v in s.items()))
def test_projectors_match_oracle(tomo, oracle_mod, spec, layout):
    o = oracle_mod
    cfg = _cfg(spec)
    rng = np.random.default_rng(7)
    vol = rng.random(cfg.volume_shape, dtype=np.float32)
    with tomo.Context(cfg) as ctx:
        ctx.set_tuning(rs_layout=layout)
        v = _dev(vol)
        for name, kind in [("RS", o.RS), ("RS_UM", o.RS_UM), ("SIDDON_REF", o.SIDDON_REF), ("SIDDON", o.SIDDON)]:
            got = ctx.project(name, v).cpu().numpy()
            _check_sino(got, o.project(cfg, kind, vol))
            assert ctx.count_samples(name) == o.count_samples(cfg, kind), name
        torch.cuda.synchronize()
        assert ctx.errors() == 0


@pytest.mark.parametrize("spec", GEOMS, ids=lambda s: "-".join(f"{k}{v}" for k, v in s.items()))
def test_backprojectors_match_oracle(tomo, oracle_mod, spec):
    o = oracle_mod
    cfg = _cfg(spec)
    sino = np.random.default_rng(8).random(cfg.sinogram_shape, dtype=np.float32)
    with tomo.Context(cfg) as ctx:
        s = _dev(sino)
        assert rel_l2(ctx.backproject("VI", s).cpu().numpy(), o.backproject(cfg, sino)) <= TOL
        assert rel_l2(ctx.backproject("VI_UM", s).cpu().numpy(), o.backproject(cfg, sino, um=True)) <= TOL


def test_operators_against_fp64_oracle(tomo, oracle_mod):
    """Each FP32 result states its error against the FP64 oracle."""
    o = oracle_mod
    from tomogpi_b200 import phantoms

    cfg = _cfg(dict(n=48, views=24, det=48))
    vol = o.phantom(phantoms.modified_shepp_logan(), 48, 48, 48)
    with tomo.Context(cfg) as ctx:
        got = ctx.project("RS", _dev(vol)).cpu().numpy()
        ref64 = o.project(cfg, o.RS, vol.astype(np.float64), fp64=True)
        assert rel_l2(got, ref64) < 2e-3  # the FP32 geometry flips the odd L_r against FP64
        sino = o.project(cfg, o.RS, vol)
        gotb = ctx.backproject("VI", _dev(sino)).cpu().numpy()
        assert rel_l2(gotb, o.backproject(cfg, sino.astype(np.float64), fp64=True)) < 1e-5


@pytest.mark.parametrize("proj,back", [("RS", "RS_ADJOINT"), ("RS_UM", "RS_UM_ADJOINT"), ("SIDDON", "SIDDON_ADJOINT")])
def test_matched_pair_adjoint(tomo, proj, back):
    """|<Ax, y> - <x, A^T y>| / (|Ax| |y|) <= 1e-5 with the matched transposes."""
    cfg = _cfg(dict(n=48, views=24, det=56))
    g = torch.Generator(device="cuda:0").manual_seed(11)
    x = torch.randn(cfg.volume_shape, device="cuda:0", generator=g)
    y = torch.randn(cfg.sinogram_shape, device="cuda:0", generator=g)
    with tomo.Context(cfg) as ctx:
        ax = ctx.project(proj, x)
        aty = ctx.backproject(back, y)
        lhs = torch.sum(ax.double() * y.double()).item()
        rhs = torch.sum(x.double() * aty.double()).item()
        denom = torch.linalg.norm(ax.double()).item() * torch.linalg.norm(y.double()).item()
    assert abs(lhs - rhs) / denom <= 1e-5


def test_adjoint_matches_oracle_transpose(tomo, oracle_mod):
    o = oracle_mod
    cfg = _cfg(dict(n=24, views=8, det=28))
    y = np.random.default_rng(4).standard_normal(cfg.sinogram_shape).astype(np.float32)
    with tomo.Context(cfg) as ctx:
        got = ctx.backproject("RS_ADJOINT", _dev(y)).cpu().numpy()
        ref = o.project_adjoint(cfg, o.RS, y.astype(np.float64), fp64=True)
        assert rel_l2(got, ref) <= 1e-5
        # Siddon's traversal switches branch where |x_det - x_s| crosses one voxel
        # (SiddonProjector_compute_C_mem_CPU.cpp:129), so FP32 and FP64 visit different voxels
        # on such rays; its transpose is checked against the FP32 restatement.
        got = ctx.backproject("SIDDON_ADJOINT", _dev(y)).cpu().numpy()
        ref = o.project_adjoint(cfg, o.SIDDON, y, fp64=False)
        assert rel_l2(got, ref) <= 1e-5


@pytest.mark.parametrize("layout", ["plain", "cell8", "tex", "hybrid", "march"])
@pytest.mark.parametrize("storage", [torch.bfloat16, torch.float16])
def test_half_storage_operators(tomo, oracle_mod, storage, layout):
    """16-bit storage, FP32 accumulation: against the oracle run on the same rounded inputs."""
    o = oracle_mod
    cfg = _cfg(dict(n=32, views=16, det=32))
    vol = np.random.default_rng(2).random(cfg.volume_shape, dtype=np.float32)
    v16 = _dev(vol, storage)
    vol_r = v16.float().cpu().numpy()
    with tomo.Context(cfg) as ctx:
        ctx.set_tuning(rs_layout=layout)
        got = ctx.project("RS", v16, dtype=torch.float32).cpu().numpy()
        _check_sino(got, o.project(cfg, o.RS, vol_r))
        got16 = ctx.project("RS", v16).float().cpu().numpy()
        eps = 2.0 ** -8 if storage == torch.bfloat16 else 2.0 ** -11
        assert rel_l2(got16, o.project(cfg, o.RS, vol_r)) <= eps
        s16 = _dev(o.project(cfg, o.RS, vol_r), storage)
        back = ctx.backproject("VI", s16, dtype=torch.float32).cpu().numpy()
        assert rel_l2(back, o.backproject(cfg, s16.float().cpu().numpy())) <= TOL


@pytest.mark.parametrize("storage", [torch.bfloat16, torch.float16])
def test_half_texture_equals_cells(tomo, storage):
    """The 16-bit texture layout (raw BF16 / FP16 bits gathered as integers) reads the same
    texel values as the cell layout and runs the same arithmetic: identical sinograms, with
    the volume given in the 16-bit type and in FP32 (converted on the device), at a size
    where the cone reaches the volume's top and bottom faces."""
    cfg = _cfg(dict(n=48, views=20, det=64))
    vol = torch.from_numpy(np.random.default_rng(4).random(cfg.volume_shape, dtype=np.float32)).cuda()
    v16 = vol.to(storage)
    out = {}
    with tomo.Context(cfg) as ctx:
        for lay in ("cell8", "tex", "hybrid", "march"):
            ctx.set_tuning(rs_layout=lay)
            # the layouts agree bit for bit: check which ran (16-bit HYBRID and MARCH run as TEX)
            assert ctx.rs_layout_in_use(storage) == ("tex" if lay in ("hybrid", "march") else lay)
            out[lay] = ctx.project("RS", v16, dtype=torch.float32).cpu().numpy()
            out[lay + "_um"] = ctx.project("RS_UM", v16, dtype=torch.float32).cpu().numpy()
    for lay in ("tex", "hybrid", "march"):
        assert np.array_equal(out["cell8"], out[lay]) and np.array_equal(out["cell8_um"], out[lay + "_um"]), lay
    assert np.abs(out["tex"]).max() > 0


@pytest.mark.parametrize("storage", [torch.float32, torch.bfloat16, torch.float16])
def test_vi_texture_layout_equals_padded(tomo, storage):
    """The VI backprojectors reading a layered texture of the sinogram (one gather per voxel
    and view), or windows of it staged in shared memory by TMA (FP32 sinograms; other types
    fall back to the padded copy), give the same volumes as reading the zero-bordered padded
    copy, for every
    chunking and both variants, on a detector smaller than the volume's shadow (footprints
    off the detector read the border)."""
    cfg = _cfg(dict(n=40, views=24, det=36))
    sino = torch.from_numpy(np.random.default_rng(6).random(cfg.sinogram_shape, dtype=np.float32)).cuda().to(storage)
    with tomo.Context(cfg) as ctx:
        for kind in ("VI", "VI_UM"):
            for zc in (1, 2, 4):
                out = {}
                for lay in ("padded", "tex", "tma"):
                    ctx.set_tuning(vi_zc=zc, vi_layout=lay)
                    out[lay] = ctx.backproject(kind, sino, dtype=torch.float32).cpu().numpy()
                assert np.array_equal(out["padded"], out["tex"]), (kind, zc)
                assert np.array_equal(out["padded"], out["tma"]), (kind, zc, "tma")
                assert np.abs(out["tex"]).max() > 0


@pytest.mark.parametrize("storage", [torch.float32, torch.bfloat16])
def test_fdk_and_ramp_filter_match_oracle(tomo, oracle_mod, storage):
    """FDK (--op=back_fdk): the ramp filter against the oracle's double-precision
    restatement of ramp_filter_TOMO8.m, the FDK-weighted backprojection against the FP64
    restatement of FDK3D_VIB_kernel_v0_16reg (which the oracle's FP32 form reproduces bit
    for bit from the reference source), and the two composed."""
    o = oracle_mod
    cfg = _cfg(dict(n=32, views=24, det=40))
    sino = np.random.default_rng(11).random(cfg.sinogram_shape, dtype=np.float32)
    s_dev = _dev(sino, storage)
    s_r = s_dev.float().cpu().numpy().astype(np.float64)  # the values as stored
    with tomo.Context(cfg) as ctx:
        filt = ctx.ramp_filter(s_dev).cpu().numpy()
        ref_f = o.ramp_filter(cfg, s_r)
        assert rel_l2(filt, ref_f) <= 1e-5
        back = ctx.backproject("FDK", s_dev, dtype=torch.float32).cpu().numpy()
        assert rel_l2(back, o.fdk_backproject(cfg, s_r, fp64=True)) <= TOL
        fdk = ctx.fdk(s_dev).cpu().numpy()
        assert rel_l2(fdk, o.fdk_backproject(cfg, ref_f, fp64=True)) <= TOL
        host = ctx.backproject_host("FDK", filt)
        assert np.array_equal(host, ctx.backproject("FDK", torch.from_numpy(filt).cuda()).cpu().numpy())


def test_fdk_reconstructs_the_phantom(tomo):
    """Filtered backprojection of a projected Shepp-Logan phantom (128 views, modest cone
    angle) correlates with the phantom."""
    from tomogpi_b200 import phantoms

    n = 48
    cfg = _cfg(dict(n=n, views=128, det=64))
    with tomo.Context(cfg) as ctx:
        truth = tomo.phantom(phantoms.modified_shepp_logan(), n, n, n)
        rec = ctx.fdk(ctx.project("RS", truth))
        a, b = truth.cpu().numpy().ravel(), rec.cpu().numpy().ravel()
    assert np.corrcoef(a, b)[0, 1] > 0.8


def test_zero_inputs_give_zero_outputs(tomo):
    """All-zero volume and sinogram: every projector, layout and backprojector returns
    exact zeros (no stale buffer content leaks into a result)."""
    cfg = _cfg(dict(n=32, views=8, det=32))
    with tomo.Context(cfg) as ctx:
        # first fill the context's cached buffers with non-zero data
        ctx.project("RS", _dev(np.ones(cfg.volume_shape, np.float32)))
        ctx.backproject("VI", _dev(np.ones(cfg.sinogram_shape, np.float32)))
        zv = torch.zeros(cfg.volume_shape, device="cuda:0")
        zs = torch.zeros(cfg.sinogram_shape, device="cuda:0")
        for lay in ("tex", "hybrid", "march", "cell8", "plain"):
            ctx.set_tuning(rs_layout=lay)
            for kind in ("RS", "RS_UM"):
                assert not ctx.project(kind, zv).any(), (kind, lay)
        for kind in ("SIDDON", "SIDDON_REF"):
            assert not ctx.project(kind, zv).any(), kind
        for kind in ("VI", "VI_UM", "FDK", "RS_ADJOINT", "SIDDON_ADJOINT"):
            assert not ctx.backproject(kind, zs).any(), kind
        assert not ctx.ramp_filter(zs).any()


def test_host_buffer_forms_match_device_forms(tomo):
    cfg = _cfg(dict(n=32, views=8, det=32))
    vol = np.random.default_rng(9).random(cfg.volume_shape, dtype=np.float32)
    with tomo.Context(cfg) as ctx:
        a = ctx.project_host("RS", vol)
        b = ctx.project("RS", _dev(vol)).cpu().numpy()
        assert np.array_equal(a, b)
        c = ctx.backproject_host("VI", a)
        d = ctx.backproject("VI", _dev(a)).cpu().numpy()
        assert np.array_equal(c, d)


def test_geometry_tables_match_oracle(tomo, oracle_mod):
    cfg = _cfg(dict(n=32, views=13, det=40, pitch=1.7)).replace(num_start_angle=1, den_start_angle=5)
    with tomo.Context(cfg) as ctx:
        s, a, b = ctx.geometry()
    s2, a2, b2 = oracle_mod.geometry_f32(cfg)
    assert np.array_equal(s, s2) and np.array_equal(a, a2) and np.array_equal(b, b2)


def test_elementwise_and_phantom(tomo, oracle_mod):
    o = oracle_mod
    from tomogpi_b200 import phantoms

    ell = phantoms.config_phantom(3, 40)
    ph = tomo.phantom(ell, 40, 36, 28).cpu().numpy()
    assert np.array_equal(ph, o.phantom(ell, 40, 36, 28))
    v = torch.randn(28, 36, 40, device="cuda:0")
    assert np.array_equal(tomo.laplacian(v).cpu().numpy(), o.laplacian(v.cpu().numpy()))
    ref = float(np.sum(v.cpu().numpy().astype(np.float64) ** 2))
    assert abs(tomo.sq_norm(v) - ref) <= 1e-12 * ref


def test_rejects_wrong_shapes_and_dtypes(tomo):
    cfg = _cfg(dict(n=16, views=4, det=16))
    with tomo.Context(cfg) as ctx:
        with pytest.raises(ValueError):
            ctx.project("RS", torch.zeros(8, 8, 8, device="cuda:0"))
        with pytest.raises(TypeError):
            ctx.project("RS", torch.zeros(cfg.volume_shape, device="cuda:0", dtype=torch.float64))


@pytest.mark.parametrize("spec", [GEOMS[3], GEOMS[5], dict(n=48, views=12, det=56)],
                         ids=lambda s: "-".join(f"{k}{v}" for k, v in s.items()))
def test_rs_warp_shapes_are_bit_identical(tomo, oracle_mod, spec):
    """The RS launch shape (rays of a warp along u: 8, 16, 32; of a block: 16 to 128)
    changes which thread computes which ray, not the arithmetic: every shape and layout
    gives the same sinogram, bit for bit, within 1e-5 of the oracle; ragged detectors leave
    partial tiles."""
    o = oracle_mod
    cfg = _cfg(spec)
    vol = np.random.default_rng(11).random(cfg.volume_shape, dtype=np.float32)
    ref = o.project(cfg, o.RS, vol)
    with tomo.Context(cfg) as ctx:
        v = _dev(vol)
        base = None
        for layout in ("tex", "hybrid", "march", "plain"):
            for wu, tu in ((8, 32), (16, 32), (32, 32), (8, 16), (16, 64), (32, 128)):
                ctx.set_tuning(rs_layout=layout, rs_warp_u=wu, rs_tile_u=tu)
                assert ctx.tuning["rs_warp_u"] == wu and ctx.tuning["rs_tile_u"] == tu
                got = ctx.project("RS", v).cpu().numpy()
                if base is None:
                    base = got
                    _check_sino(got, ref)
                assert np.array_equal(got, base), (layout, wu, tu)



@pytest.mark.parametrize("spec", [dict(n=40, views=24, det=36), dict(n=64, views=16, det=96, fod=70.0),
                                  dict(nxyz=(40, 28, 18), views=5, det=(48, 30)), dict(n=32, views=8, det=38)],
                         ids=lambda s: "-".join(f"{k}{v}" for k, v in s.items()))
def test_vi_tma_windows_match_padded(tomo, oracle_mod, spec):
    """The TMA-staged VI backprojector: bit-identical to the padded-copy kernel, within 1e-5 of
    the oracle, on a strong cone (fod 70 for a 64^3 volume: windows of some tiles exceed the
    staged box, those threads read global memory), ragged volumes (partial tiles), and a
    detector width that is not a multiple of 4 (no tensor map: the padded kernel runs)."""
    o = oracle_mod
    cfg = _cfg(spec)
    sino = np.random.default_rng(12).random(cfg.sinogram_shape, dtype=np.float32)
    with tomo.Context(cfg) as ctx:
        s = _dev(sino)
        for kind, um in (("VI", False), ("VI_UM", True)):
            ctx.set_tuning(vi_zc=1, vi_layout="padded")
            ref = ctx.backproject(kind, s).cpu().numpy()
            ctx.set_tuning(vi_layout="tma")
            got = ctx.backproject(kind, s).cpu().numpy()
            assert np.array_equal(got, ref), kind
            assert rel_l2(got, o.backproject(cfg, sino, um=um)) <= TOL, kind
            half = ctx.backproject(kind, s, dtype=torch.bfloat16).float().cpu().numpy()
            assert np.array_equal(half, torch.from_numpy(ref).to(torch.bfloat16).float().numpy()), kind
        torch.cuda.synchronize()
        assert ctx.errors() == 0


def test_vi_tma_bounded_wait_reports_timeout(tomo, oracle_mod):
    """Failure detection of the TMA-staged backprojector without a GPU fault: with the test
    stall the producer issues no copy, so the consumers' mbarrier waits (a phase that nothing
    completes) run out after their one-second bound; the kernel returns, the host reads
    ERR_TIMEOUT (bit 1) from the context's error word, and the next call on the same context
    is exact again. A tiny volume keeps it to two blocks (about one second)."""
    from tomogpi_b200 import _lib as L

    cfg = _cfg(dict(n=16, views=4, det=16))
    sino = _dev(np.random.default_rng(13).random(cfg.sinogram_shape, dtype=np.float32))
    with tomo.Context(cfg) as ctx:
        ctx.set_tuning(vi_layout="padded")
        ref = ctx.backproject("VI", sino).cpu().numpy()
        ctx.set_tuning(vi_layout="tma")
        assert ctx.errors(clear=True) == 0
        L.call("tomo_context_test_stall", ctx.handle, 1)
        ctx.backproject("VI", sino)
        torch.cuda.synchronize()
        assert ctx.errors(clear=True) & 2
        L.call("tomo_context_test_stall", ctx.handle, 0)
        got = ctx.backproject("VI", sino).cpu().numpy()
        assert ctx.errors() == 0
        assert np.array_equal(got, ref)


@pytest.mark.parametrize("spec", [dict(n=40, views=24, det=36), dict(n=33, views=19, det=50, fod=45.0),
                                  dict(nxyz=(40, 28, 18), views=13, det=(48, 30)),
                                  dict(nxyz=(17, 30, 9), views=11, det=(40, 24))],
                         ids=lambda s: "-".join(f"{k}{v}" for k, v in s.items()))
def test_march_layout_equals_hybrid(tomo, spec):
    """The MARCH layout (faces across the march axis, each sample reusing the faces it
    shares with the previous sample of its ray) reads the same texels as the HYBRID and TEX
    layouts and runs the same arithmetic: bit-identical sinograms for the box and the
    unmatched projector, with odd and unequal x / y / z sizes (faces past the data), a
    short source distance (rays that leave the volume take the checked path) and every
    view direction (x-march and y-march views)."""
    cfg = _cfg(spec)
    vol = _dev(np.random.default_rng(13).random(cfg.volume_shape, dtype=np.float32) + 0.25)
    out = {}
    with tomo.Context(cfg) as ctx:
        for lay in ("tex", "hybrid", "march"):
            ctx.set_tuning(rs_layout=lay)
            assert ctx.rs_layout_in_use(torch.float32) == lay
            for kind in ("RS", "RS_UM"):
                out[lay, kind] = ctx.project(kind, vol).cpu().numpy()
    for kind in ("RS", "RS_UM"):
        assert np.abs(out["tex", kind]).max() > 0
        assert np.array_equal(out["march", kind], out["hybrid", kind]), kind
        assert np.array_equal(out["march", kind], out["tex", kind]), kind
