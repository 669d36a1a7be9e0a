"""The command-line drop-in (tomogpi_exe, TomoGPI_exe's --pair/--op/--compute switches) on a
work directory written by the test: each operation's output file against the oracle."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
EXE = Path(__file__).resolve().parents[1] / "tomogpi_b200" / "tomogpi_exe"


def _workdir(tmp_path, n=32, views=24, penalty="GGaussian", huber=0.05, opt_nb=4, iters=4, lam=0.05, beta=2.0,
             gradient="Simple"):
    import oracle
    from tomogpi_b200 import ConfigCT, phantoms

    wd = tmp_path / f"Projections_{n}"
    wd.mkdir()
    truth = oracle.phantom(phantoms.config_phantom(1, n), n, n, n)
    truth.tofile(str(tmp_path / "real.v"))
    cfg = ConfigCT.cone_beam(n, views).replace(real_volume_name=str(tmp_path / "real.v"))
    cfg.to_file(str(wd / "configCT"))
    (wd / "configIteration").write_text(
        f"globalIterationNb 1\ngradientIterationNb {iters}\noptimalStepIterationNb {opt_nb}\n"
        f"regularizationParameter {lam}\npenaltyFunction {penalty}\nhuberThreshold {huber}\nbeta {beta}\n"
        f"gradient {gradient}\npositivity 0\n")
    (wd / "configComputeArchitecture").write_text("precision float\nstorage mem_CPU\ncompute COMPUTE_CUDA\n"
                                                   "pair PAIR_RSVI\n")
    return wd, cfg, truth


def _run(wd, *args):
    # from the work directory's parent, as TomoGPI_exe runs next to Projections_N: operator
    # outputs land in the current directory, as the reference's do
    res = subprocess.run([str(EXE), "0", f"--workdir={wd}", *args], capture_output=True, text=True, timeout=240,
                         cwd=str(Path(wd).parent))
    return res


def _load(path, shape):
    return np.fromfile(str(path), np.float32).reshape(shape)


def test_cli_proj_back_fdk(tmp_path):
    import oracle

    wd, cfg, truth = _workdir(tmp_path)
    r = _run(wd, "--op=proj")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Time computation" in r.stdout
    sino = _load(tmp_path / "proj.s", cfg.sinogram_shape)
    assert rel_l2(sino, oracle.project(cfg, oracle.RS, truth)) <= 1e-5
    assert (tmp_path / "proj.s.hdr").read_text().split("\n")[1] == "shape 24 32 32"
    # the measured sinogram is <workdir>/<tiffName>.s (configTiff)
    (wd / "configTiff").write_text("tiffName measured\n")
    sino.tofile(str(wd / "measured.s"))
    r = _run(wd, "--op=back")
    assert r.returncode == 0, r.stdout + r.stderr
    assert rel_l2(_load(tmp_path / "back.v", cfg.volume_shape), oracle.backproject(cfg, sino)) <= 1e-5
    r = _run(wd, "--op=back_fdk")
    assert r.returncode == 0, r.stdout + r.stderr
    assert rel_l2(_load(tmp_path / "back_fdk.v", cfg.volume_shape), oracle.fdk_backproject(cfg, sino)) <= 1e-5


def test_cli_siddon_pair_and_mem_gpu(tmp_path):
    import oracle

    wd, cfg, truth = _workdir(tmp_path)
    r = _run(wd, "--op=proj", "--pair=SiddonVI")
    assert r.returncode == 0, r.stdout + r.stderr
    assert rel_l2(_load(tmp_path / "proj.s", cfg.sinogram_shape), oracle.project(cfg, oracle.SIDDON_REF, truth)) <= 1e-5
    r = _run(wd, "--op=proj", "--storage=mem_GPU")
    assert r.returncode == 0, r.stdout + r.stderr
    assert rel_l2(_load(tmp_path / "proj.s", cfg.sinogram_shape), oracle.project(cfg, oracle.RS_UM, truth)) <= 1e-5


@pytest.mark.parametrize("penalty", ["GGaussian", "Huber"])
def test_cli_gradient(tmp_path, penalty):
    import oracle

    wd, cfg, truth = _workdir(tmp_path, penalty=penalty)
    g = oracle.project(cfg, oracle.SIDDON, truth)
    g.tofile(str(wd / "proj.s"))
    r = _run(wd)
    assert r.returncode == 0, r.stdout + r.stderr
    finals = sorted(wd.glob("TomoIter/Results/Result_*/finalVolume.v"))
    assert len(finals) == 1, finals
    got = _load(finals[0], cfg.volume_shape)
    ref, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g, 4, 0.05, 4,
                                    huber_threshold=0.05 if penalty == "Huber" else None)
    assert rel_l2(got, ref) <= 1e-4


def test_cli_weighted_gradient_with_beta(tmp_path):
    """configIteration gradient Weighted (Iter3D::doWeightedGradient; the weight sinogram from
    <workdir>/weightedSinogram.s or --weights) with the generalised Gaussian of shape 1.5,
    against the oracle's weighted loop."""
    import oracle

    wd, cfg, truth = _workdir(tmp_path, beta=1.5, gradient="Weighted")
    g = oracle.project(cfg, oracle.SIDDON, truth)
    g.tofile(str(wd / "proj.s"))
    w = np.random.default_rng(5).uniform(0.5, 1.5, g.shape).astype(np.float32)
    assert _run(wd).returncode != 0  # no weight sinogram yet
    w.tofile(str(tmp_path / "w.s"))
    r = _run(wd, f"--weights={tmp_path / 'w.s'}")
    assert r.returncode == 0, r.stdout + r.stderr
    finals = sorted(wd.glob("TomoIter/Results/Result_*/finalVolume.v"))
    assert len(finals) == 1, finals
    got = _load(finals[0], cfg.volume_shape)
    ref, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g, 4, 0.05, 4, beta=1.5,
                                    weights=w)
    assert rel_l2(got, ref) <= 1e-4


def test_cli_refusals(tmp_path):
    wd, cfg, truth = _workdir(tmp_path)
    for args in (["--op=proj", "--compute=OCL"], ["--op=proj", "--precision=double"], ["--op=nonsense"]):
        r = _run(wd, *args)
        assert r.returncode != 0, args
    (wd / "configIteration").write_text("gradientIterationNb 2\noptimalStepIterationNb 2\nregularizationParameter 0\n"
                                        "gradient Conjugate\n")
    np.zeros(cfg.sinogram_shape, np.float32).tofile(str(wd / "proj.s"))
    assert _run(wd).returncode != 0


@pytest.mark.parametrize("penalty", ["GGaussian", "Huber"])
def test_cli_laplacien_and_reg(tmp_path, penalty):
    """--op=laplacien and --op=reg_GG (Iter3D_main.cu:215-272) against the oracle, which is
    pinned to the reference's own regulariser sources; reg_GG applies the criterion twice to
    dJ = 0, as the reference's timing loop does."""
    import oracle

    wd, cfg, truth = _workdir(tmp_path, penalty=penalty, huber=0.3)
    r = _run(wd, "--op=laplacien")
    assert r.returncode == 0, r.stdout + r.stderr
    np.testing.assert_array_equal(_load(tmp_path / "laplacien.v", cfg.volume_shape), oracle.laplacian(truth))
    r = _run(wd, "--op=reg_GG")
    assert r.returncode == 0, r.stdout + r.stderr
    thr = 0.3 if penalty == "Huber" else None
    dj = np.zeros(cfg.volume_shape, np.float32)
    for _ in range(2):
        dj, _, _ = oracle.regularizer_criterion(truth, dj, 0.05, 1, 4, huber_threshold=thr)
    np.testing.assert_array_equal(_load(tmp_path / "GG.v", cfg.volume_shape), dj)


def test_cli_reg_gg_beta(tmp_path):
    """--op=reg_GG with configIteration beta 1.5 against the oracle's criterion of that shape
    (pinned bit for bit to the reference's regulariser source): the power is taken in FP64
    and rounded, so the device and host results agree to a few FP32 ulps."""
    import oracle

    wd, cfg, truth = _workdir(tmp_path, beta=1.5)
    r = _run(wd, "--op=reg_GG")
    assert r.returncode == 0, r.stdout + r.stderr
    dj = np.zeros(cfg.volume_shape, np.float32)
    for _ in range(2):
        dj, _, _ = oracle.regularizer_criterion(truth, dj, 0.05, 1, 4, beta=1.5)
    got = _load(tmp_path / "GG.v", cfg.volume_shape)
    assert rel_l2(got, dj) <= 1e-6
    assert np.abs(dj).max() > 0
