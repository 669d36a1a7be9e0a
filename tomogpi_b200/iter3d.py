"""Handle API of the reference's MATLAB binding, for Python callers.

The reference exposes its Iter3D object to MATLAB through one MEX function,
``TomoGPI_iter_mex(cmd, handle, workdirectory, args...)`` (src/TomoGPI_mex/Mex.cu:32-613,
TomoGPI_iter_mex.cu:135-...), wrapped by the handle class ``Matlab/Tomo8/Iter3D.m``. This
module gives the same two forms:

* ``Iter3D(workdirectory)``: the handle class, with the MATLAB method names;
* ``tomogpi_iter_mex(cmd, *args)``: the command dispatcher, handles being small integers
  ("new" returns one, "delete" releases it).

Arrays are numpy float32 in the reference's memory order: a MATLAB u x v x p sinogram is the
C-order array [p][v][u], a MATLAB x x y x z volume is [z][y][x]. Commands that fill a
caller's MATLAB array in place (doLaplacian's output, doGradient's volume,
ApplyLaplacianRegularization_to_dJ's dJ / JReg / normdJProjReg) write into the numpy array
given. Every computation runs in libtomogpi_b200 on the GPU.
"""
from __future__ import annotations

import os
import time
from pathlib import Path
from typing import Dict

import numpy as np

from . import _lib as L
from .config import ConfigCT, ConfigComputeArchitecture, ConfigIteration, read_field
from .ingest import load_raw

PRECISION_CODES = {"half": 0, "float": 1, "double": 2}        # kind_precision, ComputingArchitecture.cuh:31
STORAGE_CODES = {"mem_CPU": 0, "mem_GPU": 1, "mem_MGPU": 2}   # kind_storage, ComputingArchitecture.cuh:32


def _opt(path, name, cast, default):
    try:
        return read_field(str(path), name, cast)
    except Exception:
        return default


class Iter3D:
    """One reconstruction set-up read from a Projections_N directory (Iter3D.cu:13-120)."""

    def __init__(self, workdirectory, device: int = 0):
        import torch  # noqa: F401  (device buffers of the context)

        from .operators import Context

        wd = str(workdirectory)
        self.workdirectory = wd
        self.cfg = ConfigCT.from_file(os.path.join(wd, "configCT"))
        it_path = os.path.join(wd, "configIteration")
        self.iteration = ConfigIteration.from_file(it_path)
        self.arch = ConfigComputeArchitecture.from_file(os.path.join(wd, "configComputeArchitecture"))
        self.lam = float(self.iteration.regularization_parameter)
        self.positivity = int(self.iteration.positivity)
        self.noise_value = _opt(it_path, "addedNoiseValue", int, 0)
        tiff_name = _opt(os.path.join(wd, "configTiff"), "tiffName", str, None)
        # <workdir>/<tiffName>.s (Iter3D.cu:27-30)
        self.sinogram_directory = None if tiff_name is None else f"{wd}/{tiff_name}.s"
        # <workdir>TomoIter/Results/Result_<date>/ (Iter3D.cu:100-118), created as the reference does
        self.output_directory = wd + time.strftime("TomoIter/Results/Result_%Y_%m_%d_%Hh%M/")
        os.makedirs(self.output_directory, exist_ok=True)
        mem_gpu = self.arch.storage == "mem_GPU"
        siddon = self.arch.pair in ("PAIR_SIDDONVI", "SiddonVI", "SIDDONVI")
        self.projector = "RS_UM" if mem_gpu else ("SIDDON_REF" if siddon else "RS")
        self.backprojector = "VI_UM" if mem_gpu else "VI"
        self.ctx = Context(self.cfg, device)

    def close(self) -> None:
        if self.ctx is not None:
            self.ctx.close()
            self.ctx = None

    # ---- queries (Mex.cu:36-370) ----
    def getVersion(self) -> str:
        v = L.load().tomo_version().decode()
        print(f"TomoGPI version {v}")
        return v

    def getOutputDirectory(self) -> str:
        return self.output_directory

    def getWorkDirectory(self) -> str:
        return self.workdirectory

    def getDelta_un(self) -> float:
        return float(np.float32(self.cfg.u_detector_size) / np.float32(self.cfg.u_detector_pixel_nb))

    def getStorage(self) -> float:
        # the reference answers getStorage with the precision code and getPrecision with the
        # storage code (Mex.cu:165-189); kept for callers that rely on it
        return float(PRECISION_CODES.get(self.arch.precision, 1))

    def getPrecision(self) -> float:
        return float(STORAGE_CODES.get(self.arch.storage, 0))

    def getLambda(self) -> float:
        return self.lam

    def setLambda(self, lam) -> None:
        self.lam = float(lam)

    def getPositivity(self) -> float:
        return float(self.positivity)

    def setPositivity(self, positivity) -> None:
        self.positivity = int(positivity)

    def getNoiseValue(self) -> float:
        return float(self.noise_value)

    def getGlobalIterationNb(self) -> float:
        return float(self.iteration.global_iteration_nb)

    def getGradientIterationNb(self) -> float:
        return float(self.iteration.gradient_iteration_nb)

    def getOptimalStepIterationNb(self) -> float:
        return float(self.iteration.optimal_step_iteration_nb)

    def getUSinogramPixelNb(self) -> float:
        return float(self.cfg.u_detector_pixel_nb)

    def getVSinogramPixelNb(self) -> float:
        return float(self.cfg.v_detector_pixel_nb)

    def getProjectionSinogramPixelNb(self) -> float:
        return float(self.cfg.projection_nb)

    def getXVolumePixelNb(self) -> float:
        return float(self.cfg.x_volume_pixel_nb)

    def getYVolumePixelNb(self) -> float:
        return float(self.cfg.y_volume_pixel_nb)

    def getZVolumePixelNb(self) -> float:
        return float(self.cfg.z_volume_pixel_nb)

    # ---- data ----
    def getSinoReal(self) -> np.ndarray:
        """The measured sinogram <workdir>/<tiffName>.s (Mex.cu:43-65)."""
        if self.sinogram_directory is None:
            raise FileNotFoundError(f"{self.workdirectory}: no configTiff, so no sinogram name")
        return load_raw(self.sinogram_directory, self.cfg.sinogram_shape)

    def _volume_from(self, name) -> np.ndarray:
        if name == "none":
            return np.zeros(self.cfg.volume_shape, np.float32)
        return load_raw(name, self.cfg.volume_shape)

    def CreateVolumeInit(self) -> np.ndarray:
        """initVolumeName loaded, or zeros for "none" (Mex.cu:67-95)."""
        return self._volume_from(self.cfg.init_volume_name)

    def CreateVolumeReal(self) -> np.ndarray:
        """realVolumeName loaded, or zeros for "none" (Mex.cu:97-121)."""
        return self._volume_from(self.cfg.real_volume_name)

    # ---- operators ----
    def doProjection(self, volume) -> np.ndarray:
        return self.ctx.project_host(self.projector, self._vol(volume))

    def doBackprojection(self, sinogram) -> np.ndarray:
        return self.ctx.backproject_host(self.backprojector, self._sino(sinogram))

    def doBackprojection_FDK(self, sinogram) -> np.ndarray:
        """FDK-weighted backprojection of an already filtered sinogram (Mex.cu:406-439)."""
        return self.ctx.backproject_host("FDK", self._sino(sinogram))

    def doFilter_ramp(self, sinogram, cutoff: float = 1.0) -> np.ndarray:
        """ramp_filter_TOMO8(sinogram, 16, cutoff, delta_un) (Iter3D.m doFilter_ramp)."""
        import torch

        s = torch.from_numpy(self._sino(sinogram)).cuda(self.ctx.device)
        return self.ctx.ramp_filter(s, oversampling=16, cutoff=float(cutoff)).cpu().numpy()

    def doFDK(self, sinogram, cutoff: float = 1.0) -> np.ndarray:
        return self.doBackprojection_FDK(self.doFilter_ramp(sinogram, cutoff))

    def doLaplacian(self, volume_in, volume_out) -> np.ndarray:
        """volume_out = L volume_in, {-1, 2, -1} on each axis (Mex.cu:478-503)."""
        import torch

        from .operators import laplacian

        vin = torch.from_numpy(self._vol(volume_in)).cuda(self.ctx.device)
        volume_out[...] = laplacian(vin).cpu().numpy()
        return volume_out

    def ApplyLaplacianRegularization_to_dJ(self, volume, dJ, JReg, normdJProjReg, lam, total_iteration_idx,
                                           optimal_step_iteration_nb):
        """Regulariser criterion (Mex.cu:505-531), the generalised Gaussian with configIteration
        beta (dJ += 2*lam L(L volume) for beta = 2, beta*lam L(sign(volume) |volume|^(beta-1))
        otherwise) or Huber (dJ += lam L(psi'(L volume))) as configIteration selects, dJ updated
        in place; JReg[0] and, when total_iteration_idx < optimal_step_iteration_nb,
        normdJProjReg[0] are written."""
        import torch

        from .operators import gg_regularization, huber_regularization

        v = torch.from_numpy(self._vol(volume)).cuda(self.ctx.device)
        d = torch.from_numpy(self._vol(dJ)).cuda(self.ctx.device)
        lam32 = float(np.float32(lam))
        if self.iteration.penalty_function == "Huber":   # Mex.cu:526-527
            j, n = huber_regularization(v, d, lam32, self.iteration.huber_threshold, int(total_iteration_idx),
                                        int(optimal_step_iteration_nb))
        else:
            j, n = gg_regularization(v, d, lam32, int(total_iteration_idx), int(optimal_step_iteration_nb),
                                     beta=float(self.iteration.beta))
        dJ[...] = d.cpu().numpy()
        JReg[0] = j
        if n is not None:
            normdJProjReg[0] = n
        return j, n

    def doGradient(self, volume, sinogram, real_volume=None) -> np.ndarray:
        """gradientIterationNb iterations of the simple gradient on `volume`, in place
        (Mex.cu:533-560, Iter3D_Algo_Gradient.cu:25-223)."""
        from .operators import GradientParams, Solver

        if self.iteration.gradient != "Simple":
            raise NotImplementedError(f"gradient {self.iteration.gradient}: only Simple is part of this library")
        huber = self.iteration.penalty_function == "Huber"
        vol = self._vol(volume)
        prm = GradientParams(gradient_iteration_nb=int(self.iteration.gradient_iteration_nb),
                             optimal_step_iteration_nb=int(self.iteration.optimal_step_iteration_nb),
                             regularization_parameter=self.lam, positivity=self.positivity,
                             projector=self.projector, backprojector=self.backprojector)
        s = Solver(self.ctx, prm)
        try:
            if huber:
                s.set_regularizer("huber", self.iteration.huber_threshold)
            else:
                s.set_regularizer("gg", beta=float(self.iteration.beta))
            s.iterate_host(vol, self._sino(sinogram))
        finally:
            s.close()
        if vol is not volume:
            volume[...] = vol
        return volume

    # ---- checks ----
    def _vol(self, a) -> np.ndarray:
        a = np.asarray(a)
        if a.size != int(np.prod(self.cfg.volume_shape)) or a.dtype != np.float32:
            raise ValueError(f"expected a float32 volume of {self.cfg.volume_shape}")
        return a.reshape(self.cfg.volume_shape) if a.flags.c_contiguous else np.ascontiguousarray(a).reshape(
            self.cfg.volume_shape)

    def _sino(self, a) -> np.ndarray:
        a = np.asarray(a)
        if a.size != int(np.prod(self.cfg.sinogram_shape)) or a.dtype != np.float32:
            raise ValueError(f"expected a float32 sinogram of {self.cfg.sinogram_shape}")
        return np.ascontiguousarray(a).reshape(self.cfg.sinogram_shape)


_handles: Dict[int, Iter3D] = {}
_next_handle = [1]


def tomogpi_iter_mex(cmd: str, *args):
    """TomoGPI_iter_mex: "new"(workdirectory) -> handle; "delete"(handle, ...);
    any Iter3D method name (handle, workdirectory, args...) -> its result."""
    if cmd == "new":
        if len(args) < 1:
            raise ValueError("new: the work directory is expected")
        h = _next_handle[0]
        _next_handle[0] += 1
        _handles[h] = Iter3D(args[0])
        return h
    if len(args) < 1 or args[0] not in _handles:
        raise ValueError(f"{cmd}: unknown handle")
    obj = _handles[args[0]]
    if cmd == "delete":
        _handles.pop(args[0]).close()
        return None
    fn = getattr(obj, cmd, None) if not cmd.startswith("_") else None
    if fn is None or not callable(fn):
        raise ValueError(f"{cmd}: unknown command")
    return fn(*args[2:])
