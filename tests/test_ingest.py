"""Real-data ingest (--op=tiff5 / tiff4) on the host: the library's
tomo_tiff_negative_log_sinogram and the CLI against the reference's own ingest compiled
for the host (ConfigTiff.hpp:287-420, ImageTiff.cu:18-94) and against the numpy
restatement in the oracle, on synthetic detector files written by the tests.

Bars: white levels equal (FP64 sums of integers); the library's sinogram bit-equal to the
reference build (both FP32 division and C logf); the numpy restatement within 1 FP32 ulp
(FP64 log rounded to FP32)."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from tomogpi_b200 import _lib, ingest

EXE = Path(__file__).resolve().parents[1] / "tomogpi_b200" / "tomogpi_exe"

CONFIG_CT = """FOD 20
FDD 40
projectionNb 4
numStartAngle 0
denStartAngle 1
numStopAngle 2
denStopAngle 1
horizontalDetectorSize 8
verticalDetectorSize 8
horizontalDetectorPixelNb 8
verticalDetectorPixelNb 8
xVolumeSize 8
yVolumeSize 8
zVolumeSize 8
xVolumePixelNb 8
yVolumePixelNb 8
zVolumePixelNb 8
"""


def _need_ref():
    if oracle.ref_tiff_lib() is None:
        pytest.skip("reference host build of the ingest unavailable")


def _write_image(path: Path, img: np.ndarray, header=(7, 0, 13, 0)) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    np.concatenate([np.array(header, np.uint16), img.astype(np.uint16).ravel()]).tofile(str(path))


def make_case(root: Path, *, total=6, used=3, ui=40, vi=24, uf=16, vf=10, uc=20, vc=12, cu=32, cv=18, energies=3,
              digits=5, seed=0, zero_pixel=True):
    """A work directory <root>/Projections_8 with configCT and configTiff, detector files in
    <root>/tif and a calibration file in <root>/Calibration. Returns (workdir, fields)."""
    rng = np.random.default_rng(seed)
    wd = root / "Projections_8"
    wd.mkdir(parents=True, exist_ok=True)
    (wd / "configCT").write_text(CONFIG_CT)
    t = dict(total_projection_nb=total, used_projection_nb=used, u_initial_nb=ui, v_initial_nb=vi, u_final_nb=uf,
             v_final_nb=vf, u_center_final=uc, v_center_final=vc, u_calibration_nb=cu, v_calibration_nb=cv,
             calibration_energy_nb=energies, digits=digits)
    (wd / "configTiff").write_text(
        f"tiffName scan\ntotalProjectionNb {total}\nusedProjectionNb {used}\n"
        f"uDetectorPixelInitialNb {ui}\nvDetectorPixelInitialNb {vi}\nuDetectorPixelFinalNb {uf}\n"
        f"vDetectorPixelFinalNb {vf}\nuDetectorCenterFinal {uc}\nvDetectorCenterFinal {vc}\n"
        f"uCalibrationImagePixelNb {cu}\nvCalibrationImagePixelNb {cv}\nCalibrationEnergyNb {energies}\n"
        f"calibrationTiffName white.tif\nnormalizationFactor 1.0\n")
    _write_image(root / "Calibration" / "white.tif", rng.integers(20000, 60000, size=(cv, cu)))
    fmt = "_%05d.tif" if digits == 5 else "_%04d.tif"
    for p in range(1, total + 2):
        img = rng.integers(50, 65535, size=(vi, ui))
        if zero_pixel and p == total + 1:
            img[vc, uc] = 0          # -log(0) = +inf, kept as the reference computes it
        _write_image(root / "tif" / ("scan" + fmt % p), img)
    return wd, t


def _lib_sinogram(root: Path, t: dict) -> np.ndarray:
    cfg = ingest.TiffConfig(**t, tiff_name="scan", calibration_tiff_name="white.tif")
    return ingest.negative_log_sinogram(cfg, root / "tif", root / "Calibration" / "white.tif")


@pytest.mark.parametrize("kw", [
    dict(),                                        # rate 2, window inside the file
    dict(total=10, used=3),                        # rate 3 with a remainder: files 11, 8, 5
    dict(total=4, used=4, digits=4),               # every file, 4-digit names
    dict(uf=15, vf=9),                             # odd window: the last column/row stays 0
    dict(energies=1, cv=7),                        # whole calibration image is white
    dict(energies=4, cv=18),                       # rows (E-1)*ny/E rounded down
    dict(uc=4, vc=3),                              # window starts before column/row 0 (wraps)
    dict(uc=38, vc=22),                            # window runs past the file's edge
])
def test_library_matches_reference_build(tmp_path, kw):
    _need_ref()
    wd, t = make_case(tmp_path, **kw)
    ref = oracle.ref_tiff_negative_log_sinogram(wd, t["digits"], (t["used_projection_nb"], t["v_final_nb"],
                                                                   t["u_final_nb"]))
    got = _lib_sinogram(tmp_path, t)
    np.testing.assert_array_equal(got, ref)
    port = oracle.tiff_negative_log_sinogram(t, tmp_path / "tif", "scan", tmp_path / "Calibration" / "white.tif")
    np.testing.assert_array_max_ulp(got, port, maxulp=1)


def test_white_mean_three_ways(tmp_path):
    _need_ref()
    wd, t = make_case(tmp_path, cv=19, energies=3)
    f = tmp_path / "Calibration" / "white.tif"
    ref = oracle.ref_tiff_lib().ref_tiff_white_mean(str(f).encode(), 32, 19, 3)
    assert ingest.white_mean(f, 32, 19, 3) == ref
    assert oracle.tiff_white_mean(f, 32, 19, 3) == ref


def test_view_order_and_window(tmp_path):
    """Views run from file total+1 downwards; view 0 of the sinogram is that file's window."""
    wd, t = make_case(tmp_path, zero_pixel=False)
    got = _lib_sinogram(tmp_path, t)
    img = oracle.read_detector_file(tmp_path / "tif" / "scan_00007.tif", 40, 24)
    white = np.float32(oracle.tiff_white_mean(tmp_path / "Calibration" / "white.tif", 32, 18, 3))
    expect = -np.log((img[7:17, 12:28].astype(np.float32) / white).astype(np.float64))
    np.testing.assert_allclose(got[0], expect, rtol=2e-7)
    assert np.isfinite(got).all()


def test_missing_short_and_bad_inputs(tmp_path):
    wd, t = make_case(tmp_path)
    (tmp_path / "tif" / "scan_00005.tif").unlink()
    with pytest.raises(_lib.TomoError) as e:
        _lib_sinogram(tmp_path, t)
    assert e.value.status == 7 and "scan_00005.tif" in str(e.value)
    _write_image(tmp_path / "tif" / "scan_00005.tif", np.ones((3, 40)))          # too short
    with pytest.raises(_lib.TomoError) as e:
        _lib_sinogram(tmp_path, t)
    assert e.value.status == 7
    for bad in (dict(used_projection_nb=0), dict(used_projection_nb=9), dict(digits=3), dict(u_final_nb=0)):
        with pytest.raises(_lib.TomoError) as e:
            _lib_sinogram(tmp_path, {**t, **bad})
        assert e.value.status == 1
    with pytest.raises(_lib.TomoError) as e:
        ingest.white_mean(tmp_path / "Calibration" / "absent.tif", 32, 18, 3)
    assert e.value.status == 7


@pytest.mark.parametrize("op,digits", [("tiff5", 5), ("tiff4", 4)])
def test_cli_tiff_op(tmp_path, op, digits):
    if not EXE.exists():
        pytest.skip("tomogpi_exe not built")
    wd, t = make_case(tmp_path, digits=digits)
    res = subprocess.run([str(EXE), "8", f"--op={op}", f"--workdir={wd}"], capture_output=True, text=True,
                         timeout=60)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "Real sinogram from tiff created" in res.stdout
    got = ingest.load_raw(wd / "scan.s")
    assert got.shape == (3, 10, 16)
    np.testing.assert_array_equal(got, _lib_sinogram(tmp_path, t))
    py = ingest.ingest_workdir(wd, digits=digits, save=False)
    np.testing.assert_array_equal(py, got)


def test_raw_sidecar_round_trip(tmp_path):
    a = np.arange(24, dtype=np.float32).reshape(2, 3, 4)
    ingest.save_raw(tmp_path / "x.v", a)
    np.testing.assert_array_equal(ingest.load_raw(tmp_path / "x.v"), a)
    a.tofile(str(tmp_path / "plain.s"))                  # a reference file: no sidecar
    np.testing.assert_array_equal(ingest.load_raw(tmp_path / "plain.s", shape=(2, 3, 4)), a)
    with pytest.raises(ValueError):
        ingest.load_raw(tmp_path / "plain.s")
    with pytest.raises(ValueError):
        ingest.load_raw(tmp_path / "plain.s", shape=(5, 5))


def test_config_reader_first_match(tmp_path):
    f = tmp_path / "configTiff"
    f.write_text("# tiffName comment\ntiffName a b\ntiffName c\n")
    assert ingest.read_config_field(f, "tiffName") == "comment"   # first token match, as the reference
    assert ingest.read_config_field(f, "absent", "dflt") == "dflt"
    with pytest.raises(KeyError):
        ingest.read_config_field(f, "absent")
    assert ctypes.sizeof(_lib.TomoTiffConfig) == 12 * 4
