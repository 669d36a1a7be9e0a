"""The MATLAB-style handle API (TomoGPI_iter_mex / Iter3D.m, src/TomoGPI_mex/Mex.cu:32-613)
on a work directory written by the test: every command against the oracle."""
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _workdir(tmp_path, n=32, views=24, seed=0, gradient="Simple", lam=0.01, opt_nb=4, iters=4):
    import oracle
    from tomogpi_b200 import ConfigCT, phantoms
    from tomogpi_b200.ingest import save_raw

    wd = tmp_path / "Projections_32"
    wd.mkdir()
    truth = oracle.phantom(phantoms.config_phantom(seed, n), n, n, n)
    save_raw(tmp_path / "real.v", truth)
    cfg = ConfigCT.cone_beam(n, views).replace(real_volume_name=str(tmp_path / "real.v"))
    cfg.to_file(str(wd / "configCT"))
    (wd / "configIteration").write_text(
        f"globalIterationNb 1\ngradientIterationNb {iters}\noptimalStepIterationNb {opt_nb}\n"
        f"regularizationParameter {lam}\npenaltyFunction GGaussian\nbeta 2\ngradient {gradient}\npositivity 0\n"
        "addedNoiseValue 30\n")
    (wd / "configComputeArchitecture").write_text("precision float\nstorage mem_CPU\ncompute COMPUTE_CUDA\n"
                                                   "pair PAIR_RSVI\n")
    (wd / "configTiff").write_text("tiffName sino\n")
    g = oracle.project(cfg, oracle.SIDDON, truth)
    g = (g + np.random.default_rng(seed).normal(0, 0.01 * g.max(), g.shape)).astype(np.float32)
    save_raw(wd / "sino.s", g)
    return str(wd) + "/", cfg, truth, g


def test_handle_queries_and_data(tmp_path):
    from tomogpi_b200.iter3d import tomogpi_iter_mex as mex

    wd, cfg, truth, g = _workdir(tmp_path)
    h = mex("new", wd)
    try:
        assert mex("getXVolumePixelNb", h, wd) == 32.0 and mex("getZVolumePixelNb", h, wd) == 32.0
        assert mex("getUSinogramPixelNb", h, wd) == 32.0 and mex("getProjectionSinogramPixelNb", h, wd) == 24.0
        assert mex("getDelta_un", h, wd) == 2.0
        assert mex("getLambda", h, wd) == pytest.approx(0.01)
        mex("setLambda", h, wd, 0.5)
        assert mex("getLambda", h, wd) == 0.5
        mex("setPositivity", h, wd, 1)
        assert mex("getPositivity", h, wd) == 1.0
        assert mex("getNoiseValue", h, wd) == 30.0
        assert (mex("getGradientIterationNb", h, wd), mex("getOptimalStepIterationNb", h, wd)) == (4.0, 4.0)
        assert mex("getStorage", h, wd) == 1.0 and mex("getPrecision", h, wd) == 0.0   # swapped, as the reference
        assert mex("getOutputDirectory", h, wd).startswith(wd + "TomoIter/Results/Result_")
        np.testing.assert_array_equal(mex("getSinoReal", h, wd), g)
        np.testing.assert_array_equal(mex("CreateVolumeReal", h, wd), truth)
        assert not mex("CreateVolumeInit", h, wd).any()
        assert isinstance(mex("getVersion", h, wd), str)
        with pytest.raises(ValueError):
            mex("noSuchCommand", h, wd)
    finally:
        mex("delete", h, wd)
    with pytest.raises(ValueError):
        mex("getLambda", h, wd)


def test_handle_operators_match_oracle(tmp_path):
    import oracle
    from tomogpi_b200.iter3d import Iter3D

    wd, cfg, truth, g = _workdir(tmp_path)
    it = Iter3D(wd)
    try:
        assert rel_l2(it.doProjection(truth), oracle.project(cfg, oracle.RS, truth)) <= 1e-5
        assert rel_l2(it.doBackprojection(g), oracle.backproject(cfg, g)) <= 1e-5
        assert rel_l2(it.doBackprojection_FDK(g), oracle.fdk_backproject(cfg, g)) <= 1e-5
        filt = it.doFilter_ramp(g)
        assert rel_l2(filt, oracle.ramp_filter(cfg, g)) <= 1e-5
        assert rel_l2(it.doFDK(g), oracle.fdk_backproject(cfg, oracle.ramp_filter(cfg, g))) <= 1e-4
        out = np.zeros_like(truth)
        it.doLaplacian(truth, out)
        np.testing.assert_array_equal(out, oracle.laplacian(truth))
    finally:
        it.close()


@pytest.mark.parametrize("total,opt", [(1, 4), (5, 4)])
def test_gg_regularization_matches_oracle(tmp_path, total, opt):
    import oracle
    from tomogpi_b200.iter3d import Iter3D

    wd, cfg, truth, g = _workdir(tmp_path)
    rng = np.random.default_rng(3)
    dJ = rng.normal(0, 1, cfg.volume_shape).astype(np.float32)
    lam = 0.037
    lap = oracle.laplacian(truth)
    expect = dJ + np.float32(2.0 * float(np.float32(lam))) * oracle.laplacian(lap)   # FP32 multiply, then add
    jreg = np.zeros(1)
    nrm = np.full(1, -1.0)
    it = Iter3D(wd)
    try:
        got = dJ.copy()
        it.ApplyLaplacianRegularization_to_dJ(truth, got, jreg, nrm, lam, total, opt)
    finally:
        it.close()
    np.testing.assert_array_equal(got, expect)
    assert jreg[0] == pytest.approx(float((lap.astype(np.float64) ** 2).sum()), rel=1e-12)
    if total < opt:
        assert nrm[0] == pytest.approx(2.0 * float((oracle.laplacian(expect).astype(np.float64) ** 2).sum()), rel=1e-12)
    else:
        assert nrm[0] == -1.0


def test_do_gradient_matches_oracle_in_place(tmp_path):
    import oracle
    from tomogpi_b200.iter3d import Iter3D

    wd, cfg, truth, g = _workdir(tmp_path, iters=4, opt_nb=3)
    ref, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g, 4, 0.01, 3)
    it = Iter3D(wd)
    try:
        vol = it.CreateVolumeInit()
        it.doGradient(vol, it.getSinoReal(), it.CreateVolumeReal())
    finally:
        it.close()
    assert rel_l2(vol, ref) <= 1e-4


def test_gg_beta_criterion_and_gradient(tmp_path):
    """configIteration beta 1.5 through the handle API: ApplyLaplacianRegularization_to_dJ and
    doGradient against the oracle's generalised Gaussian of that shape."""
    import oracle
    from tomogpi_b200.iter3d import Iter3D

    wd, cfg, truth, g = _workdir(tmp_path)
    conf = Path(wd) / "configIteration"
    conf.write_text(conf.read_text().replace("beta 2", "beta 1.5"))
    it = Iter3D(wd)
    try:
        rng = np.random.default_rng(4)
        vol = rng.normal(0, 0.3, cfg.volume_shape).astype(np.float32)
        dj = rng.normal(0, 1.0, cfg.volume_shape).astype(np.float32)
        d_ref, j_ref, n_ref = oracle.regularizer_criterion(vol, dj, it.getLambda(), 1, 4, beta=1.5)
        jr, nr = np.zeros(1), np.zeros(1)
        it.ApplyLaplacianRegularization_to_dJ(vol, dj, jr, nr, it.getLambda(), 1, 4)
        assert rel_l2(dj, d_ref) <= 1e-6
        assert abs(jr[0] - j_ref) <= 1e-6 * abs(j_ref) and abs(nr[0] - n_ref) <= 1e-6 * abs(n_ref)
        v = np.zeros(cfg.volume_shape, np.float32)
        it.doGradient(v, g)
        ref, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g,
                                        int(it.getGradientIterationNb()), it.getLambda(),
                                        int(it.getOptimalStepIterationNb()), beta=1.5)
        assert rel_l2(v, ref) <= 1e-4
    finally:
        it.close()


def test_unsupported_solver_is_refused(tmp_path):
    from tomogpi_b200.iter3d import Iter3D

    wd, cfg, truth, g = _workdir(tmp_path, gradient="Conjugate")
    it = Iter3D(wd)
    try:
        with pytest.raises(NotImplementedError):
            it.doGradient(np.zeros(cfg.volume_shape, np.float32), g)
        with pytest.raises(ValueError):
            it.doProjection(np.zeros((3, 3, 3), np.float32))
    finally:
        it.close()


def _huber_d1(v, thr):
    d = v.astype(np.float64)
    return np.where(d <= -thr, np.float32(-2.0 * thr),
                    np.where(np.abs(d) < thr, (2.0 * d).astype(np.float32), np.where(d >= thr, np.float32(2.0 * thr), v)))


def _huber_d2(v, thr):
    a = np.abs(v.astype(np.float64))
    return np.where(a > thr, np.float32(0), np.where(a <= thr, np.float32(1), v)).astype(np.float32)


@pytest.mark.parametrize("total,opt", [(1, 4), (5, 4)])
def test_huber_criterion_matches_oracle(tmp_path, total, opt):
    """ApplyLaplacianRegularization_to_dJ under penaltyFunction Huber (HuberRegularizer_CPU.cu:
    206-253) against the oracle's Laplacian and the potential's branches in numpy."""
    import oracle
    from tomogpi_b200.iter3d import Iter3D

    wd, cfg, truth, g = _workdir(tmp_path)
    thr = 0.3
    it_cfg = (Path(wd) / "configIteration")
    it_cfg.write_text(it_cfg.read_text().replace("penaltyFunction GGaussian", "penaltyFunction Huber")
                      + f"huberThreshold {thr}\n")
    rng = np.random.default_rng(5)
    dJ = rng.normal(0, 1, cfg.volume_shape).astype(np.float32)
    lam = 0.037
    grad = oracle.laplacian(truth)
    expect = dJ + np.float32(lam) * oracle.laplacian(_huber_d1(grad, thr).astype(np.float32))
    a = np.abs(grad.astype(np.float64))
    jref = float(np.where(a < thr, a * a, 2.0 * thr * a - thr * thr).sum())
    s = oracle.laplacian(oracle.laplacian(_huber_d2(grad, thr) * expect)) * expect
    jreg, nrm = np.zeros(1), np.full(1, -1.0)
    it = Iter3D(wd)
    try:
        got = dJ.copy()
        it.ApplyLaplacianRegularization_to_dJ(truth, got, jreg, nrm, lam, total, opt)
    finally:
        it.close()
    np.testing.assert_array_equal(got, expect)
    assert jreg[0] == pytest.approx(jref, rel=1e-12)
    if total < opt:
        assert nrm[0] == pytest.approx(float(np.abs(s.astype(np.float64)).sum()), rel=1e-12)
    else:
        assert nrm[0] == -1.0
