"""The oracle is pinned: its FP32 restatement must reproduce, bit for bit, the golden
outputs that the reference's own sources produced (tests/golden/make_golden.py), and, where
the reference host build exists in this checkout, fresh reference runs on other inputs."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_matches_reference_golden(oracle_mod, case):
    o = oracle_mod
    cfg, d = load_golden(case)
    vol, sino = d["volume"], d["sinogram"]
    assert np.array_equal(o.project(cfg, o.RS, vol), d["rs"])
    assert np.array_equal(o.project(cfg, o.RS_UM, vol), d["rs_um"])
    assert np.array_equal(o.backproject(cfg, sino, um=False), d["vi"])
    assert np.array_equal(o.backproject(cfg, sino, um=True), d["vi_um"])
    assert np.array_equal(o.fdk_backproject(cfg, sino), d["fdk"])
    if "siddon_ref" in d:
        assert np.array_equal(o.project(cfg, o.SIDDON_REF, vol), d["siddon_ref"])


def _ref_or_skip(o):
    if o.ref_lib() is None:
        pytest.skip("reference host build not present in this checkout (oracle/_ref)")


@pytest.mark.parametrize("n,views,det,fod", [(16, 8, 16, None), (32, 8, 32, 33.0), (24, 16, 32, None)])
def test_oracle_matches_reference_fresh(oracle_mod, n, views, det, fod):
    o = oracle_mod
    _ref_or_skip(o)
    from tomogpi_b200.config import ConfigCT

    cfg = ConfigCT.cone_beam(n, views, det=det, fod=fod)
    rng = np.random.default_rng(n * 1000 + views)
    vol = rng.standard_normal(cfg.volume_shape).astype(np.float32)
    sino = rng.standard_normal(cfg.sinogram_shape).astype(np.float32)
    assert np.array_equal(o.project(cfg, o.RS, vol), o.ref_project(cfg, o.RS, vol))
    assert np.array_equal(o.project(cfg, o.RS_UM, vol), o.ref_project(cfg, o.RS_UM, vol))
    if n % 16 == 0:
        assert np.array_equal(o.backproject(cfg, sino), o.ref_backproject(cfg, sino))
        assert np.array_equal(o.backproject(cfg, sino, um=True), o.ref_backproject(cfg, sino, um=True))
        assert np.array_equal(o.fdk_backproject(cfg, sino), o.ref_fdk_backproject(cfg, sino))
    if det % 16 == 0 and views % 8 == 0:
        assert np.array_equal(o.project(cfg, o.SIDDON_REF, vol), o.ref_project(cfg, o.SIDDON_REF, vol))


def test_oracle_sample_config_geometry(oracle_mod):
    """The sample Data3D_0256 geometry (mm units, non-unit voxels) through the oracle and,
    where available, the reference build."""
    o = oracle_mod
    from tomogpi_b200.config import ConfigCT

    cfg = ConfigCT(fod=98.0, fdd=230.0, projection_nb=8, u_detector_size=14.2 / 8, v_detector_size=14.2 / 8,
                   u_detector_pixel_nb=16, v_detector_pixel_nb=16, x_volume_size=6.05 / 16, y_volume_size=6.05 / 16,
                   z_volume_size=5.86 / 16, x_volume_pixel_nb=16, y_volume_pixel_nb=16, z_volume_pixel_nb=16)
    vol = np.random.default_rng(3).random(cfg.volume_shape, dtype=np.float32)
    a = o.project(cfg, o.RS, vol)
    assert np.isfinite(a).all() and a.max() > 0
    if o.ref_lib() is not None:
        assert np.array_equal(a, o.ref_project(cfg, o.RS, vol))
        assert np.array_equal(o.project(cfg, o.SIDDON_REF, vol), o.ref_project(cfg, o.SIDDON_REF, vol))


def test_fp64_oracle_close_to_fp32(oracle_mod):
    o = oracle_mod
    cfg, d = load_golden("n32_p16_det48")
    a32 = o.project(cfg, o.RS, d["volume"])
    a64 = o.project(cfg, o.RS, d["volume"].astype(np.float64), fp64=True)
    # FP32 vs FP64 differ by rounding plus the odd sample whose count L_r flips
    assert np.linalg.norm(a32 - a64) / np.linalg.norm(a64) < 5e-3
    b32 = o.backproject(cfg, d["sinogram"])
    b64 = o.backproject(cfg, d["sinogram"].astype(np.float64), fp64=True)
    assert np.linalg.norm(b32 - b64) / np.linalg.norm(b64) < 1e-5


@pytest.mark.parametrize("kind", [0, 1, 3])
def test_oracle_adjoint_is_transpose(oracle_mod, kind):
    """<Ax, y> == <x, A^T y> for the FP64 matched transposes."""
    o = oracle_mod
    from tomogpi_b200.config import ConfigCT

    cfg = ConfigCT.cone_beam(16, 8, det=20)
    rng = np.random.default_rng(kind)
    x = rng.standard_normal(cfg.volume_shape)
    y = rng.standard_normal(cfg.sinogram_shape)
    ax = o.project(cfg, kind, x, fp64=True)
    aty = o.project_adjoint(cfg, kind, y, fp64=True)
    lhs, rhs = float((ax * y).sum()), float((x * aty).sum())
    assert abs(lhs - rhs) / (np.linalg.norm(ax) * np.linalg.norm(y)) < 1e-12


def test_laplacian_oracle_matches_numpy(oracle_mod):
    o = oracle_mod
    rng = np.random.default_rng(5)
    v = rng.standard_normal((6, 7, 8)).astype(np.float64)
    p = np.pad(v, 1)
    ref = 6 * v - (p[1:-1, 1:-1, :-2] + p[1:-1, 1:-1, 2:] + p[1:-1, :-2, 1:-1] + p[1:-1, 2:, 1:-1]
                   + p[:-2, 1:-1, 1:-1] + p[2:, 1:-1, 1:-1])
    assert np.allclose(o.laplacian(v, fp64=True), ref, rtol=0, atol=1e-12)


def test_phantom_oracle_shepp_logan(oracle_mod):
    o = oracle_mod
    from tomogpi_b200 import phantoms

    ph = o.phantom(phantoms.modified_shepp_logan(), 32, 32, 32)
    # modified Shepp-Logan intensities: outer shell 1.0, brain 0.2, small features 0.1..0.4
    vals = set(np.round(np.unique(ph).astype(np.float64), 3).tolist())
    assert {0.0, 0.2, 1.0} <= vals
    assert ph.min() >= -1e-6 and ph.max() <= 1.0 + 1e-6


def _matlab_ramp_filter(sino, oversampling, fc, du):
    """ramp_filter_TOMO8.m step by step with FFTs (the reference's own formulation), for
    checking the oracle's direct-convolution restatement. Matlab's round is half away from
    zero and its fftshift of an even length is a roll by half the length."""
    rnd = lambda x: int(np.floor(x + 0.5))  # noqa: E731
    n = sino.shape[-1]
    m = oversampling * n
    ramp = np.array([-(k - 1) + m / 2 for k in range(1, m // 2 + 2)] + [(k - 1) - m / 2 for k in range(m // 2 + 2, m + 1)])
    ramp = np.fft.fftshift(ramp)
    ramp = ramp / ramp.max()
    nr = rnd(m * fc)
    nr -= nr % 2
    hann = 0.5 * (1 - np.cos(2 * np.pi * np.arange(nr) / (nr - 1)))
    win = np.fft.fftshift(np.concatenate([np.zeros((m - nr) // 2), hann, np.zeros((m - nr) // 2)]))
    h = np.real(np.fft.ifft(ramp * win))
    down = np.concatenate([h[:rnd(n)], h[m - rnd(n):]])
    down[rnd(n / 2):rnd(3 * n / 2)] = 0
    filt = np.fft.fft(down)
    rows = sino.reshape(-1, n).astype(np.float64)
    out = np.real(np.fft.ifft(np.fft.fft(rows, 2 * n, axis=1) * filt[None, :], axis=1))[:, :n] / (2 * du)
    return out.reshape(sino.shape)


@pytest.mark.parametrize("n,det,over,fc", [(16, 40, 16, 1.0), (16, 33, 16, 1.0), (16, 24, 4, 0.5)])
def test_ramp_filter_oracle_matches_matlab_steps(oracle_mod, n, det, over, fc):
    """The ramp filter has no C source in the reference (only ramp_filter_TOMO8.m): the
    oracle's direct convolution is checked against the Matlab steps done with FFTs."""
    o = oracle_mod
    from tomogpi_b200.config import ConfigCT

    cfg = ConfigCT.cone_beam(n, 5, det=det, pitch=1.7)
    sino = np.random.default_rng(det).standard_normal(cfg.sinogram_shape)
    got = o.ramp_filter(cfg, sino, oversampling=over, cutoff=fc)
    ref = _matlab_ramp_filter(sino, over, fc, float(np.float32(cfg.u_detector_size) / np.float32(det)))
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


@pytest.mark.parametrize("shape", [(8, 9, 10), (16, 16, 16), (5, 12, 7)])
@pytest.mark.parametrize("huber", [None, 0.05, 0.4, 1e6])
@pytest.mark.parametrize("total,optimal", [(1, 4), (4, 4)])
def test_regularizer_criteria_match_reference(oracle_mod, shape, huber, total, optimal):
    """The oracle's GG (beta = 2) and Huber criteria against the reference's own
    GeneralizedGaussianRegularizer_CPU / HuberRegularizer_CPU built for the host: dJ, jReg and
    normdJProjReg bit for bit."""
    o = oracle_mod
    if o.ref_reg_lib() is None:
        pytest.skip("reference host build of the regularisers unavailable")
    rng = np.random.default_rng(sum(shape) + (0 if huber is None else int(huber * 100)))
    vol = rng.normal(0, 0.3, shape).astype(np.float32)
    dJ = rng.normal(0, 1.0, shape).astype(np.float32)
    got = o.regularizer_criterion(vol, dJ, 0.037, total, optimal, huber_threshold=huber)
    ref = o.regularizer_criterion(vol, dJ, 0.037, total, optimal, huber_threshold=huber, reference=True)
    assert np.array_equal(got[0], ref[0])
    assert got[1] == ref[1]
    assert got[2] == ref[2]
    if total < optimal:
        assert got[2] is not None and np.isfinite(got[2])


@pytest.mark.parametrize("huber", [None, 0.05])
@pytest.mark.parametrize("lam,opt,pos", [(0.01, 4, 0), (0.01, 21, 1), (0.0, 3, 0)])
def test_gradient_loop_matches_reference(oracle_mod, huber, lam, opt, pos):
    """The oracle's simple gradient against the reference's own Iter3D::doSimpleGradient
    (Iter3D_Algo_Gradient.cu:25-223) built for the host over its RS / VI kernel sources and
    GG / Huber regularisers: the iterate bit for bit."""
    from tomogpi_b200 import ConfigCT, phantoms

    o = oracle_mod
    if o.ref_iter_lib() is None:
        pytest.skip("reference host build of the gradient loop unavailable")
    cfg = ConfigCT.cone_beam(16, 12)
    truth = o.phantom(phantoms.config_phantom(0, 16), 16, 16, 16)
    g = o.project(cfg, o.SIDDON, truth)
    g = (g + np.random.default_rng(2).normal(0, 0.01 * g.max(), g.shape)).astype(np.float32)
    ours, _ = o.simple_gradient(cfg, o.RS, np.zeros(cfg.volume_shape, np.float32), g, 5, lam, opt, positivity=pos,
                                huber_threshold=huber)
    ref = o.ref_simple_gradient(cfg, np.zeros(cfg.volume_shape, np.float32), g, 5, lam, opt, positivity=pos,
                                huber_threshold=huber)
    assert np.array_equal(ours, ref)
    assert np.abs(ours).max() > 0


@pytest.mark.parametrize("shape", [(8, 9, 10), (5, 12, 7)])
@pytest.mark.parametrize("beta", [1.0, 1.2, 1.5, 1.9, 2.5])
@pytest.mark.parametrize("total,optimal", [(1, 4), (4, 4)])
def test_gg_beta_criterion_matches_reference(oracle_mod, shape, beta, total, optimal):
    """The oracle's generalised-Gaussian criterion for beta != 2 against the reference's own
    GeneralizedGaussianRegularizer_CPU.cu:158-226 built for the host, whose beta != 2 steps
    (sign of the volume, |volume|^(beta-1), product, Laplacian, beta*lambda axpy,
    beta * sum |L dJ|^beta) are the device form's (GeneralizedGaussianRegularizer_GPU.cu:
    161-225): dJ, jReg and normdJProjReg bit for bit. The volume holds exact zeros so that
    sign(0) = 0 is exercised."""
    o = oracle_mod
    if o.ref_reg_lib() is None:
        pytest.skip("reference host build of the regularisers unavailable")
    rng = np.random.default_rng(sum(shape) + int(beta * 10))
    vol = rng.normal(0, 0.3, shape).astype(np.float32)
    vol[rng.random(shape) < 0.1] = 0.0
    dJ = rng.normal(0, 1.0, shape).astype(np.float32)
    got = o.regularizer_criterion(vol, dJ, 0.037, total, optimal, beta=beta)
    ref = o.regularizer_criterion(vol, dJ, 0.037, total, optimal, beta=beta, reference=True)
    assert np.array_equal(got[0], ref[0])
    assert got[1] == ref[1] and got[2] == ref[2]
    assert np.all(np.isfinite(got[0]))
    if beta != 2.0:  # not the beta = 2 criterion
        b2 = o.regularizer_criterion(vol, dJ, 0.037, total, optimal)
        assert not np.array_equal(got[0], b2[0])


@pytest.mark.parametrize("beta,weighted", [(1.5, False), (2.0, True), (1.2, True)])
@pytest.mark.parametrize("lam,opt,pos", [(0.01, 4, 0), (0.01, 21, 1), (0.0, 3, 0)])
def test_gradient_loop_beta_weighted_matches_reference(oracle_mod, beta, weighted, lam, opt, pos):
    """The oracle's loop with the generalised Gaussian of shape beta, and the weighted
    gradient, against the reference's own Iter3D::doSimpleGradient /
    Iter3D::doWeightedGradient (Iter3D_Algo_Gradient.cu:227-373) built for the host: the
    iterate bit for bit. Weights in (0.25, 1.75) with exact zeros (masked rays)."""
    from tomogpi_b200 import ConfigCT, phantoms

    o = oracle_mod
    if o.ref_iter_lib() is None:
        pytest.skip("reference host build of the gradient loop unavailable")
    cfg = ConfigCT.cone_beam(16, 12)
    truth = o.phantom(phantoms.config_phantom(0, 16), 16, 16, 16)
    g = o.project(cfg, o.SIDDON, truth)
    rng = np.random.default_rng(3)
    g = (g + rng.normal(0, 0.01 * g.max(), g.shape)).astype(np.float32)
    w = None
    if weighted:
        w = rng.uniform(0.25, 1.75, g.shape).astype(np.float32)
        w[rng.random(g.shape) < 0.05] = 0.0
    ours, alphas = o.simple_gradient(cfg, o.RS, np.zeros(cfg.volume_shape, np.float32), g, 5, lam, opt,
                                     positivity=pos, beta=beta, weights=w)
    ref = o.ref_simple_gradient(cfg, np.zeros(cfg.volume_shape, np.float32), g, 5, lam, opt, positivity=pos,
                                beta=beta, weights=w)
    assert np.array_equal(ours, ref)
    assert np.abs(ours).max() > 0 and np.all(np.isfinite(alphas))


@pytest.mark.parametrize("lam,opt,pos", [(0.01, 4, 0), (0.05, 21, 1)])
def test_weighted_gradient_with_huber_matches_reference(oracle_mod, lam, opt, pos):
    """The weighted loop under the Huber regulariser against the reference's own
    Iter3D::doWeightedGradient built for the host: the iterate bit for bit."""
    from tomogpi_b200 import ConfigCT, phantoms

    o = oracle_mod
    if o.ref_iter_lib() is None:
        pytest.skip("reference host build of the gradient loop unavailable")
    cfg = ConfigCT.cone_beam(16, 12)
    truth = o.phantom(phantoms.config_phantom(1, 16), 16, 16, 16)
    g = o.project(cfg, o.SIDDON, truth)
    rng = np.random.default_rng(5)
    g = (g + rng.normal(0, 0.01 * g.max(), g.shape)).astype(np.float32)
    w = rng.uniform(0.25, 1.75, g.shape).astype(np.float32)
    ours, _ = o.simple_gradient(cfg, o.RS, np.zeros(cfg.volume_shape, np.float32), g, 5, lam, opt, positivity=pos,
                                huber_threshold=0.05, weights=w)
    ref = o.ref_simple_gradient(cfg, np.zeros(cfg.volume_shape, np.float32), g, 5, lam, opt, positivity=pos,
                                huber_threshold=0.05, weights=w)
    assert np.array_equal(ours, ref)
    assert np.abs(ours).max() > 0
