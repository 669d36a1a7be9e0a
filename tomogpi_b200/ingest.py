"""Real-data ingest: detector files to the normalised negative-log sinogram.

The reference's ``--op=tiff5`` / ``--op=tiff4`` (Iter3D_main.cu:317-336) reads
``<workdir>/configTiff`` (ConfigTiff.cpp:13-26), the white level of
``<workdir>/../Calibration/<calibrationTiffName>`` and the projections
``<workdir>/../tif/<tiffName>_<nnnnn>.tif``, and saves ``<workdir>/<tiffName>.s`` (FP32,
view-major, Iter3D.cu:27-30). The arithmetic runs in libtomogpi_b200
(``tomo_tiff_negative_log_sinogram``); this module reads the configuration and calls it.

Raw ``.s`` / ``.v`` files carry no header in the reference (Sinogram3D.cu:138-184,
Volume.cu:248-272). ``save_raw`` writes the same bytes plus a ``<file>.hdr`` sidecar with the
dtype and shape, and ``load_raw`` uses the sidecar when it is there.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib


def read_config_field(path, name: str, default=None) -> str:
    """First whitespace-separated token equal to `name`, then the next token
    (Config::getConfigFileField, Config.cpp:35-69). KeyError if absent and no default."""
    with open(path) as f:
        for row in f:
            toks = row.split()
            for i, tok in enumerate(toks):
                if tok == name:
                    return toks[i + 1] if i + 1 < len(toks) else ""
    if default is not None:
        return default
    raise KeyError(f"field {name} not found in {path}")


@dataclass
class TiffConfig:
    """The detector-file fields of configTiff (ConfigTiff.cpp:13-26)."""
    total_projection_nb: int
    used_projection_nb: int
    u_initial_nb: int
    v_initial_nb: int
    u_final_nb: int
    v_final_nb: int
    u_center_final: int
    v_center_final: int
    u_calibration_nb: int
    v_calibration_nb: int
    calibration_energy_nb: int
    digits: int = 5
    tiff_name: str = ""
    calibration_tiff_name: str = ""

    FIELDS = {
        "total_projection_nb": "totalProjectionNb", "used_projection_nb": "usedProjectionNb",
        "u_initial_nb": "uDetectorPixelInitialNb", "v_initial_nb": "vDetectorPixelInitialNb",
        "u_final_nb": "uDetectorPixelFinalNb", "v_final_nb": "vDetectorPixelFinalNb",
        "u_center_final": "uDetectorCenterFinal", "v_center_final": "vDetectorCenterFinal",
        "u_calibration_nb": "uCalibrationImagePixelNb", "v_calibration_nb": "vCalibrationImagePixelNb",
        "calibration_energy_nb": "CalibrationEnergyNb",
    }

    @classmethod
    def from_file(cls, path, digits: int = 5) -> "TiffConfig":
        kw = {k: int(read_config_field(path, v)) for k, v in cls.FIELDS.items()}
        return cls(**kw, digits=digits, tiff_name=read_config_field(path, "tiffName"),
                   calibration_tiff_name=read_config_field(path, "calibrationTiffName"))

    @property
    def sinogram_shape(self):
        return (self.used_projection_nb, self.v_final_nb, self.u_final_nb)

    def struct(self) -> _lib.TomoTiffConfig:
        return _lib.TomoTiffConfig(*[int(getattr(self, n)) for n, _ in _lib.TomoTiffConfig._fields_])


def white_mean(calibration_file, nx: int, ny: int, energy_nb: int) -> float:
    """White level of a calibration file (ImageCalibration::getWhiteMeanValue)."""
    out = ctypes.c_double()
    _lib.call("tomo_tiff_white_mean", str(calibration_file).encode(), nx, ny, energy_nb, ctypes.byref(out))
    return out.value


def negative_log_sinogram(cfg: TiffConfig, tif_dir, calibration_file) -> np.ndarray:
    """The normalised negative-log sinogram [used][v_final][u_final] (FP32) of the files
    <tif_dir>/<tiff_name>_<p+1>.tif. TomoError TOMO_ERR_INVALID for a bad configuration
    (digits other than 4 or 5 included), TOMO_ERR_IO for a missing or short file."""
    out = np.empty(cfg.sinogram_shape, np.float32)
    st = cfg.struct()
    _lib.call("tomo_tiff_negative_log_sinogram", ctypes.byref(st), str(tif_dir).encode(),
              cfg.tiff_name.encode(), str(calibration_file).encode(), out.ctypes.data)
    return out


def ingest_workdir(workdir, digits: int = 5, save: bool = True) -> np.ndarray:
    """--op=tiff5 (digits 5) / --op=tiff4 (digits 4) on a reference work directory: reads
    configTiff, builds the sinogram and (save=True) writes <workdir>/<tiffName>.s."""
    wd = Path(workdir)
    cfg = TiffConfig.from_file(wd / "configTiff", digits=digits)
    sino = negative_log_sinogram(cfg, wd / ".." / "tif", wd / ".." / "Calibration" / cfg.calibration_tiff_name)
    if save:
        save_raw(wd / f"{cfg.tiff_name}.s", sino)
    return sino


def save_raw(path, array: np.ndarray) -> None:
    """The reference's raw file (values only, native byte order) plus a text sidecar
    <path>.hdr: "dtype <numpy dtype>" and "shape <d0> <d1> ...", slowest axis first."""
    a = np.ascontiguousarray(array)
    a.tofile(str(path))
    Path(str(path) + ".hdr").write_text(f"dtype {a.dtype.str}\nshape {' '.join(map(str, a.shape))}\n")


def load_raw(path, shape=None, dtype=np.float32) -> np.ndarray:
    """A raw file; dtype and shape from its <path>.hdr sidecar when present, else the
    arguments (reference files have no sidecar). A size mismatch raises ValueError."""
    hdr = Path(str(path) + ".hdr")
    if hdr.exists():
        meta = dict(line.split(None, 1) for line in hdr.read_text().splitlines() if line.strip())
        dtype = np.dtype(meta["dtype"])
        shape = tuple(int(x) for x in meta["shape"].split())
    if shape is None:
        raise ValueError(f"{path}: no .hdr sidecar, give the shape")
    a = np.fromfile(str(path), dtype=dtype)
    if a.size != int(np.prod(shape)):
        raise ValueError(f"{path}: {a.size} values, expected {int(np.prod(shape))} for shape {tuple(shape)}")
    return a.reshape(shape)
