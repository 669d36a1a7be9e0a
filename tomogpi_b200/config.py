"""configCT / configIteration / configComputeArchitecture readers.

Mirrors TomoGPI's key/value configuration files (``Config::getConfigFileField``,
src/TomoGPI_lib/src/CPP/Config/Config.cpp:35-69): each file is scanned line by line,
every whitespace-separated token is compared with the requested field name, and the
token that follows the FIRST match is the value. A missing field is an error (the
reference calls ``exit``; this reader raises ``ConfigError``).

``ConfigCT`` carries exactly the fields that ConfigCT::createUniformAcquisition,
createDetector and createVolume* read (ConfigCT.cpp:43-54,110-147).
"""
from __future__ import annotations

import dataclasses
import math
import os
import re
from dataclasses import dataclass, field
from typing import Optional


class ConfigError(RuntimeError):
    pass


def read_field(path: str, name: str, cast=str):
    """Config::getConfigFileField: value token after the first token equal to ``name``."""
    try:
        with open(path, "r", encoding="utf-8", errors="replace") as fh:
            for row in fh:
                toks = row.split()
                for i, tok in enumerate(toks):
                    if tok == name:
                        if i + 1 >= len(toks):
                            raise ConfigError(f"field {name} has no value in {path}")
                        val = toks[i + 1]
                        if cast is int:
                            # istream >> int stops at the first non-digit ("256mm" -> 256)
                            j = 1 if val[:1] in "+-" else 0
                            while j < len(val) and val[j].isdigit():
                                j += 1
                            return int(val[:j])
                        if cast is float:
                            return float(_numeric_prefix(val))
                        return val
    except FileNotFoundError as exc:
        raise ConfigError(f"Unable to open file {path}") from exc
    raise ConfigError(f"Unable to find field {name} in {path}")


_NUM = re.compile(r"^[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?")


def _numeric_prefix(tok: str) -> str:
    """istream >> double: the longest leading decimal number of the token."""
    m = _NUM.match(tok)
    if not m:
        raise ConfigError(f"not a number: {tok}")
    return m.group(0)


@dataclass
class ConfigCT:
    """Acquisition, detector and volume description (configCT).

    Units are whatever the file uses (the sample files use mm; the benchmarks use voxel
    units with unit voxels). Angles: phi_p = (p + start) * pi * (stop - start) / P with
    start = numStartAngle/denStartAngle and stop = numStopAngle/denStopAngle, i.e. in
    units of pi (Acquisition.cpp:90-97, ConfigCT.cpp:112-121).
    """

    fod: float
    fdd: float
    projection_nb: int
    u_detector_size: float
    v_detector_size: float
    u_detector_pixel_nb: int
    v_detector_pixel_nb: int
    x_volume_size: float
    y_volume_size: float
    z_volume_size: float
    x_volume_pixel_nb: int
    y_volume_pixel_nb: int
    z_volume_pixel_nb: int
    num_start_angle: float = 0.0
    den_start_angle: float = 1.0
    num_stop_angle: float = 2.0
    den_stop_angle: float = 1.0
    real_volume_name: str = "none"
    init_volume_name: str = "none"

    @classmethod
    def from_file(cls, path: str) -> "ConfigCT":
        f = lambda n, t=float: read_field(path, n, t)  # noqa: E731
        return cls(
            fod=f("FOD", float), fdd=f("FDD", float), projection_nb=f("projectionNb", int),
            num_start_angle=f("numStartAngle"), den_start_angle=f("denStartAngle"),
            num_stop_angle=f("numStopAngle"), den_stop_angle=f("denStopAngle"),
            u_detector_size=f("horizontalDetectorSize"), v_detector_size=f("verticalDetectorSize"),
            u_detector_pixel_nb=f("horizontalDetectorPixelNb", int),
            v_detector_pixel_nb=f("verticalDetectorPixelNb", int),
            x_volume_size=f("xVolumeSize"), y_volume_size=f("yVolumeSize"), z_volume_size=f("zVolumeSize"),
            x_volume_pixel_nb=f("xVolumePixelNb", int), y_volume_pixel_nb=f("yVolumePixelNb", int),
            z_volume_pixel_nb=f("zVolumePixelNb", int),
            real_volume_name=_opt(path, "realVolumeName"), init_volume_name=_opt(path, "initVolumeName"),
        )

    def to_file(self, path: str) -> None:
        """Writes a configCT file with the field names ConfigCT::ConfigCT reads."""
        rows = [("FOD", self.fod), ("FDD", self.fdd), ("projectionNb", self.projection_nb),
                ("numStartAngle", self.num_start_angle), ("denStartAngle", self.den_start_angle),
                ("numStopAngle", self.num_stop_angle), ("denStopAngle", self.den_stop_angle),
                ("horizontalDetectorSize", self.u_detector_size), ("verticalDetectorSize", self.v_detector_size),
                ("horizontalDetectorPixelNb", self.u_detector_pixel_nb),
                ("verticalDetectorPixelNb", self.v_detector_pixel_nb),
                ("xVolumeSize", self.x_volume_size), ("yVolumeSize", self.y_volume_size),
                ("zVolumeSize", self.z_volume_size), ("xVolumePixelNb", self.x_volume_pixel_nb),
                ("yVolumePixelNb", self.y_volume_pixel_nb), ("zVolumePixelNb", self.z_volume_pixel_nb),
                ("realVolumeName", self.real_volume_name), ("initVolumeName", self.init_volume_name)]
        with open(path, "w") as f:
            for k, v in rows:
                f.write(f"{k} {v if isinstance(v, str) else repr(v)}\n")  # repr: exact round trip

    @classmethod
    def cone_beam(cls, n: int, views: int, det: Optional[int] = None, pitch: float = 2.0,
                  fod: Optional[float] = None, magnification: float = 2.0) -> "ConfigCT":
        """Voxel-unit circular cone-beam set-up: n^3 unit voxels, det x det detector of the
        given pitch, FOD = 2n unless given, FDD = magnification * FOD, views over 2*pi."""
        det = n if det is None else det
        fod = 2.0 * n if fod is None else fod
        return cls(fod=fod, fdd=magnification * fod, projection_nb=views,
                   u_detector_size=pitch * det, v_detector_size=pitch * det,
                   u_detector_pixel_nb=det, v_detector_pixel_nb=det,
                   x_volume_size=float(n), y_volume_size=float(n), z_volume_size=float(n),
                   x_volume_pixel_nb=n, y_volume_pixel_nb=n, z_volume_pixel_nb=n)

    # shapes in the reference layouts
    @property
    def volume_shape(self):
        return (self.z_volume_pixel_nb, self.y_volume_pixel_nb, self.x_volume_pixel_nb)

    @property
    def sinogram_shape(self):
        return (self.projection_nb, self.v_detector_pixel_nb, self.u_detector_pixel_nb)

    @property
    def voxel_ray_updates(self) -> int:
        """Work of one operator call: Nx*Ny*Nz*P voxel-ray updates."""
        return self.x_volume_pixel_nb * self.y_volume_pixel_nb * self.z_volume_pixel_nb * self.projection_nb

    def replace(self, **kw) -> "ConfigCT":
        return dataclasses.replace(self, **kw)

    def phi(self):
        start = self.num_start_angle / self.den_start_angle
        stop = self.num_stop_angle / self.den_stop_angle
        step = math.pi * (stop - start) / self.projection_nb
        return [(p + start) * step for p in range(self.projection_nb)]


def _opt(path: str, name: str) -> str:
    try:
        return read_field(path, name)
    except ConfigError:
        return "none"


@dataclass
class ConfigIteration:
    """configIteration fields used by the gradient-descent loop (ConfigIteration.cpp:12-22)."""

    gradient_iteration_nb: int = 10
    optimal_step_iteration_nb: int = 10
    regularization_parameter: float = 0.01
    penalty_function: str = "GGaussian"
    gradient: str = "Simple"
    positivity: int = 0
    beta: float = 2.0
    global_iteration_nb: int = 1
    huber_threshold: float = 0.0

    @classmethod
    def from_file(cls, path: str) -> "ConfigIteration":
        return cls(
            gradient_iteration_nb=read_field(path, "gradientIterationNb", int),
            optimal_step_iteration_nb=read_field(path, "optimalStepIterationNb", int),
            regularization_parameter=read_field(path, "regularizationParameter", float),
            penalty_function=read_field(path, "penaltyFunction"),
            gradient=read_field(path, "gradient"),
            positivity=read_field(path, "positivity", int),
            beta=read_field(path, "beta", float),
            global_iteration_nb=read_field(path, "globalIterationNb", int),
            huber_threshold=_get(path, "huberThreshold", float, 0.0),
        )


@dataclass
class ConfigComputeArchitecture:
    """configComputeArchitecture: precision/storage/compute/pair switches plus the
    reference's launch-shape fields (kept for compatibility; the B200 kernels choose their
    own shapes through the autotuner)."""

    precision: str = "float"
    storage: str = "mem_CPU"
    compute: str = "COMPUTE_CUDA"
    architecture: str = "ARCHITECTURE_GPU"
    pair: str = "PAIR_RSVI"
    gpu_nb_proj: int = 1
    streams_nb_proj: int = 1
    gpu_nb_back: int = 1
    streams_nb_back: int = 1
    extra: dict = field(default_factory=dict)

    @classmethod
    def from_file(cls, path: str) -> "ConfigComputeArchitecture":
        g = lambda n, t=str, d=None: _get(path, n, t, d)  # noqa: E731
        return cls(
            precision=g("precision", str, "float"), storage=g("storage", str, "mem_CPU"),
            compute=g("compute", str, "COMPUTE_CUDA"), architecture=g("architecture", str, "ARCHITECTURE_GPU"),
            pair=g("pair", str, "PAIR_RSVI"), gpu_nb_proj=g("gpuNbP", int, 1), streams_nb_proj=g("streamsNbP", int, 1),
            gpu_nb_back=g("gpuNbBP", int, 1), streams_nb_back=g("streamsNbBP", int, 1),
        )


def _get(path, name, cast, default):
    try:
        return read_field(path, name, cast)
    except ConfigError:
        if default is None:
            raise
        return default


def config_dir_files(directory: str):
    """The three files TomoGPI_exe reads from a Projections_N directory."""
    return (os.path.join(directory, "configCT"), os.path.join(directory, "configIteration"),
            os.path.join(directory, "configComputeArchitecture"))
