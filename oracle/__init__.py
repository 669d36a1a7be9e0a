"""The oracle -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``libtomo_oracle.so`` (the CPU restatement of the reference's
arithmetic, ``tomo_oracle.cpp``) and, where it has been built, to ``_ref/libtomo_ref.so``
(the reference's own kernel sources and Siddon C file compiled for the host through the
shims in ``ref_shim``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use this
package, and only as the checker / the timed CPU baseline. The product library never
imports it.

Every function takes a configCT-like object exposing the fields of ``CONFIG_FIELDS``
(``tomogpi_b200.ConfigCT`` does) and numpy arrays in the reference layouts:
volume ``[z][y][x]`` and sinogram ``[phi][v][u]``.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import build as _build

HERE = Path(__file__).resolve().parent

# Projector kinds, numbered as in the product C-ABI.
RS, RS_UM, SIDDON_REF, SIDDON = 0, 1, 2, 3

CONFIG_FIELDS = [
    ("fod", ctypes.c_double),
    ("fdd", ctypes.c_double),
    ("num_start_angle", ctypes.c_double),
    ("den_start_angle", ctypes.c_double),
    ("num_stop_angle", ctypes.c_double),
    ("den_stop_angle", ctypes.c_double),
    ("projection_nb", ctypes.c_int32),
    ("u_detector_size", ctypes.c_float),
    ("v_detector_size", ctypes.c_float),
    ("u_detector_pixel_nb", ctypes.c_int32),
    ("v_detector_pixel_nb", ctypes.c_int32),
    ("x_volume_size", ctypes.c_float),
    ("y_volume_size", ctypes.c_float),
    ("z_volume_size", ctypes.c_float),
    ("x_volume_pixel_nb", ctypes.c_int32),
    ("y_volume_pixel_nb", ctypes.c_int32),
    ("z_volume_pixel_nb", ctypes.c_int32),
]


class _Cfg(ctypes.Structure):
    _fields_ = CONFIG_FIELDS


def _cfg(c) -> _Cfg:
    return _Cfg(*[getattr(c, name) for name, _ in CONFIG_FIELDS])


_lib = None
_ref = None
_P = np.ctypeslib.ndpointer
_F32 = _P(dtype=np.float32, flags="C_CONTIGUOUS")
_F64 = _P(dtype=np.float64, flags="C_CONTIGUOUS")
_CFGP = ctypes.POINTER(_Cfg)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(_build.build_oracle()))
        sig = {
            "oracle_geometry_f32": (None, [_CFGP, _F32, _F32, _F32]),
            "oracle_project_f32": (None, [_CFGP, ctypes.c_int, _F32, _F32]),
            "oracle_project_f64": (None, [_CFGP, ctypes.c_int, _F64, _F64]),
            "oracle_backproject_f32": (None, [_CFGP, ctypes.c_int, _F32, _F32]),
            "oracle_backproject_f64": (None, [_CFGP, ctypes.c_int, _F64, _F64]),
            "oracle_fdk_backproject_f32": (None, [_CFGP, _F32, _F32]),
            "oracle_fdk_backproject_f64": (None, [_CFGP, _F64, _F64]),
            "oracle_ramp_filter": (None, [_CFGP, ctypes.c_int, ctypes.c_double, _F64, _F64]),
            "oracle_project_adjoint_f32": (None, [_CFGP, ctypes.c_int, _F32, _F32]),
            "oracle_project_adjoint_f64": (None, [_CFGP, ctypes.c_int, _F64, _F64]),
            "oracle_count_samples": (ctypes.c_ulonglong, [_CFGP, ctypes.c_int]),
            "oracle_laplacian_f32": (None, [_F32, _F32, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
            "oracle_laplacian_f64": (None, [_F64, _F64, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
            "oracle_sino_sq_norm_f32": (ctypes.c_double, [_F32, ctypes.c_long]),
            "oracle_vol_sq_norm_f32": (ctypes.c_double, [_F32, ctypes.c_long]),
            "oracle_simple_gradient_f32": (None, [_CFGP, ctypes.c_int, ctypes.c_int, _F32, _F32, ctypes.c_int,
                                                  ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64]),
            "oracle_simple_gradient_f64": (None, [_CFGP, ctypes.c_int, ctypes.c_int, _F64, _F64, ctypes.c_int,
                                                  ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64]),
            "oracle_gg_criterion_f32": (None, [_F32, _F32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                               ctypes.c_int, ctypes.c_int, _F64]),
            "oracle_huber_criterion_f32": (None, [_F32, _F32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_float, ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64]),
            "oracle_gg_criterion_beta_f32": (None, [_F32, _F32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_float, ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64]),
            "oracle_gradient_f32": (None, [_CFGP, ctypes.c_int, ctypes.c_int, _F32, _F32, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
            "oracle_gradient_f64": (None, [_CFGP, ctypes.c_int, ctypes.c_int, _F64, _F64, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
            "oracle_simple_gradient_reg_f32": (None, [_CFGP, ctypes.c_int, ctypes.c_int, _F32, _F32, ctypes.c_int,
                                                      ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64,
                                                      ctypes.c_int, ctypes.c_double]),
            "oracle_simple_gradient_reg_f64": (None, [_CFGP, ctypes.c_int, ctypes.c_int, _F64, _F64, ctypes.c_int,
                                                      ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64,
                                                      ctypes.c_int, ctypes.c_double]),
            "oracle_phantom_f32": (None, [_F64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def ref_lib():
    """The reference's own sources built for the host, or None if never built here."""
    global _ref
    if _ref is None:
        so = _build.build_reference()
        if so is None or not Path(so).exists():
            return None
        _ref = ctypes.CDLL(str(so))
        for name in ("ref_rs_box_project", "ref_rs_um_project", "ref_siddon_project"):
            getattr(_ref, name).argtypes = [_CFGP, _F32, _F32]
        for name in ("ref_vi_backproject", "ref_vi_um_backproject", "ref_fdk_backproject"):
            getattr(_ref, name).argtypes = [_CFGP, _F32, _F32]
    return _ref


def _vol_shape(c):
    return (c.z_volume_pixel_nb, c.y_volume_pixel_nb, c.x_volume_pixel_nb)


def _sino_shape(c):
    return (c.projection_nb, c.v_detector_pixel_nb, c.u_detector_pixel_nb)


def geometry_f32(c):
    """(scalars, alpha, beta): fod, fdd, gamma, du, dv, uc, vc, dx, xc, yc, zc as float32."""
    s = np.zeros(13, np.float32)
    a = np.zeros(c.projection_nb, np.float32)
    b = np.zeros(c.projection_nb, np.float32)
    lib().oracle_geometry_f32(ctypes.byref(_cfg(c)), s, a, b)
    return s[:11], a, b


def project(c, kind: int, vol: np.ndarray, fp64: bool = False) -> np.ndarray:
    dt = np.float64 if fp64 else np.float32
    vol = np.ascontiguousarray(vol, dtype=dt)
    out = np.zeros(_sino_shape(c), dt)
    fn = lib().oracle_project_f64 if fp64 else lib().oracle_project_f32
    fn(ctypes.byref(_cfg(c)), kind, vol, out)
    return out


def backproject(c, sino: np.ndarray, um: bool = False, fp64: bool = False) -> np.ndarray:
    dt = np.float64 if fp64 else np.float32
    sino = np.ascontiguousarray(sino, dtype=dt)
    out = np.zeros(_vol_shape(c), dt)
    fn = lib().oracle_backproject_f64 if fp64 else lib().oracle_backproject_f32
    fn(ctypes.byref(_cfg(c)), int(um), sino, out)
    return out


def fdk_backproject(c, sino: np.ndarray, fp64: bool = False) -> np.ndarray:
    """FDK-weighted VI backprojection (FDK3D_kernel_16reg.cuh:24-349) of a filtered sinogram."""
    dt = np.float64 if fp64 else np.float32
    sino = np.ascontiguousarray(sino, dtype=dt)
    out = np.zeros(_vol_shape(c), dt)
    (lib().oracle_fdk_backproject_f64 if fp64 else lib().oracle_fdk_backproject_f32)(ctypes.byref(_cfg(c)), sino, out)
    return out


def ramp_filter(c, sino: np.ndarray, oversampling: int = 16, cutoff: float = 1.0) -> np.ndarray:
    """The ramp filter of ramp_filter_TOMO8.m, in double."""
    sino = np.ascontiguousarray(sino, dtype=np.float64)
    out = np.zeros(_sino_shape(c), np.float64)
    lib().oracle_ramp_filter(ctypes.byref(_cfg(c)), int(oversampling), float(cutoff), sino, out)
    return out


def project_adjoint(c, kind: int, sino: np.ndarray, fp64: bool = True) -> np.ndarray:
    dt = np.float64 if fp64 else np.float32
    sino = np.ascontiguousarray(sino, dtype=dt)
    out = np.zeros(_vol_shape(c), dt)
    fn = lib().oracle_project_adjoint_f64 if fp64 else lib().oracle_project_adjoint_f32
    fn(ctypes.byref(_cfg(c)), kind, sino, out)
    return out


def count_samples(c, kind: int) -> int:
    return int(lib().oracle_count_samples(ctypes.byref(_cfg(c)), kind))


def laplacian(vol: np.ndarray, fp64: bool = False) -> np.ndarray:
    dt = np.float64 if fp64 else np.float32
    vol = np.ascontiguousarray(vol, dtype=dt)
    out = np.zeros_like(vol)
    nz, ny, nx = vol.shape
    (lib().oracle_laplacian_f64 if fp64 else lib().oracle_laplacian_f32)(vol, out, nx, ny, nz)
    return out


def sino_sq_norm(s: np.ndarray) -> float:
    s = np.ascontiguousarray(s, dtype=np.float32)
    return float(lib().oracle_sino_sq_norm_f32(s, s.size))


def vol_sq_norm(v: np.ndarray) -> float:
    v = np.ascontiguousarray(v, dtype=np.float32)
    return float(lib().oracle_vol_sq_norm_f32(v, v.size))


def simple_gradient(c, proj_kind: int, vol0: np.ndarray, real_sino: np.ndarray, iterations: int,
                    lam: float, optimal_step_nb: int, positivity: int = 0, back_um: bool = False,
                    fp64: bool = False, huber_threshold=None, beta: float = 2.0, weights=None):
    """Iter3D::doSimpleGradient, or Iter3D::doWeightedGradient when `weights` (a sinogram)
    is given; returns (volume, per-iteration alpha). Regulariser: the generalised Gaussian of
    shape `beta`, or the Huber potential when `huber_threshold` is given."""
    dt = np.float64 if fp64 else np.float32
    vol = np.array(vol0, dtype=dt, copy=True, order="C")
    sino = np.ascontiguousarray(real_sino, dtype=dt)
    alphas = np.zeros(max(iterations, 1), np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=dt)
    if w is not None and w.size != sino.size:
        raise ValueError("weights must have the sinogram's size")
    fn = lib().oracle_gradient_f64 if fp64 else lib().oracle_gradient_f32
    fn(ctypes.byref(_cfg(c)), proj_kind, int(back_um), vol, sino, iterations, float(lam), optimal_step_nb,
       positivity, alphas, 0 if huber_threshold is None else 1, float(huber_threshold or 0.0), float(beta),
       None if w is None else w.ctypes.data_as(ctypes.c_void_p))
    return vol, alphas[:iterations]


def phantom(ellipsoids: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    e = np.ascontiguousarray(ellipsoids, dtype=np.float64).reshape(-1, 10)
    out = np.zeros((nz, ny, nx), np.float32)
    lib().oracle_phantom_f32(e, e.shape[0], nx, ny, nz, out)
    return out


# --- the reference's own sources, host build -------------------------------------
def ref_project(c, kind: int, vol: np.ndarray) -> np.ndarray:
    r = ref_lib()
    if r is None:
        raise RuntimeError("reference host build unavailable (oracle/_ref not built)")
    vol = np.ascontiguousarray(vol, dtype=np.float32)
    if kind == SIDDON_REF:
        # The Siddon C file addresses voxels modulo 256 per axis (which, below 256, can reach
        # past the volume); give it a zero-filled buffer that covers every such address.
        nx, ny = c.x_volume_pixel_nb, c.y_volume_pixel_nb
        span = max(vol.size, 256 + 255 * nx + 255 * nx * ny)
        padded = np.zeros(span, np.float32)
        padded[: vol.size] = vol.ravel()
        vol = padded
    out = np.zeros(_sino_shape(c), np.float32)
    fn = {RS: r.ref_rs_box_project, RS_UM: r.ref_rs_um_project, SIDDON_REF: r.ref_siddon_project}[kind]
    fn(ctypes.byref(_cfg(c)), vol, out)
    return out


def ref_backproject(c, sino: np.ndarray, um: bool = False) -> np.ndarray:
    r = ref_lib()
    if r is None:
        raise RuntimeError("reference host build unavailable (oracle/_ref not built)")
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    out = np.zeros(_vol_shape(c), np.float32)
    (r.ref_vi_um_backproject if um else r.ref_vi_backproject)(ctypes.byref(_cfg(c)), sino, out)
    return out


def ref_fdk_backproject(c, sino: np.ndarray) -> np.ndarray:
    r = ref_lib()
    if r is None:
        raise RuntimeError("reference host build unavailable (oracle/_ref not built)")
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    out = np.zeros(_vol_shape(c), np.float32)
    r.ref_fdk_backproject(ctypes.byref(_cfg(c)), sino, out)
    return out


# ---- detector-file ingest (--op=tiff5 / tiff4) ----

def read_detector_file(path, nx: int, ny: int) -> np.ndarray:
    """One detector file as the reference reads it (ImageTiff::loadTiffImage,
    ImageTiff.cu:18-38; ConfigTiff.hpp:327-330): four 16-bit header words, then ny rows of
    nx 16-bit pixels."""
    raw = np.fromfile(path, dtype=np.uint16)
    if raw.size < 4 + nx * ny:
        raise ValueError(f"{path}: {raw.size} words, expected {4 + nx * ny}")
    return raw[4:4 + nx * ny].reshape(ny, nx)


def tiff_white_mean(path, nx: int, ny: int, energy_nb: int) -> float:
    """ImageCalibration::getWhiteMeanValue (ImageTiff.cu:81-94): FP64 sum over rows
    [(E-1)*ny/E, ny) (integer row bound), divided by nx*ny/E."""
    img = read_detector_file(path, nx, ny)
    y0 = (energy_nb - 1) * ny // energy_nb
    return float(img[y0:].astype(np.float64).sum()) / (float(nx) * ny / float(energy_nb))


def tiff_negative_log_sinogram(t: dict, tif_dir, tiff_name: str, calibration_file) -> np.ndarray:
    """ConfigTiff::createNormalizedMeanNegativeLogSinogram_5dig / _4dig
    (ConfigTiff.hpp:287-356 and the 4-digit twin): files p+1 for p = total, total - rate, ...
    while p > total - rate * used (rate = total // used, ConfigTiff.cpp:24), the window
    [centre - final/2, centre + final/2) of each (unsigned-short bounds, :293-296), every
    pixel mapped to -log(float(pixel) / float(white)) in FP32 (:334). `t` holds the fields
    of the product's tomo_tiff_config. Pixels of the window outside the file stay 0."""
    white = np.float32(tiff_white_mean(calibration_file, t["u_calibration_nb"], t["v_calibration_nb"],
                                       t["calibration_energy_nb"]))
    ushort = lambda x: int(x) & 0xFFFF  # noqa: E731
    inf_u = ushort(t["u_center_final"] - t["u_final_nb"] // 2)
    inf_v = ushort(t["v_center_final"] - t["v_final_nb"] // 2)
    sup_u = ushort(t["u_center_final"] + t["u_final_nb"] // 2)
    sup_v = ushort(t["v_center_final"] + t["v_final_nb"] // 2)
    total, used = t["total_projection_nb"], t["used_projection_nb"]
    rate = total // used
    nu, nv = t["u_final_nb"], t["v_final_nb"]
    out = np.zeros((used, nv, nu), np.float32)
    fmt = "_%05d.tif" if t["digits"] == 5 else "_%04d.tif"
    phi = 0
    p = total
    while p > total - rate * used:
        img = read_detector_file(Path(tif_dir) / (tiff_name + fmt % (p + 1)), t["u_initial_nb"], t["v_initial_nb"])
        v1, u1 = min(sup_v, t["v_initial_nb"]), min(sup_u, t["u_initial_nb"])
        if v1 > inf_v and u1 > inf_u:
            win = img[inf_v:v1, inf_u:u1].astype(np.float32) / white
            # float64 log rounded to FP32: within one FP32 ulp of a C logf
            with np.errstate(divide="ignore"):  # a 0 pixel gives +inf, as in the reference
                out[phi, :v1 - inf_v, :u1 - inf_u] = (-np.log(win.astype(np.float64))).astype(np.float32)
        phi += 1
        p -= rate
    return out


_ref_tiff = None


def ref_tiff_lib():
    """The reference's own detector-file ingest built for the host, or None."""
    global _ref_tiff
    if _ref_tiff is None:
        so = _build.build_reference_tiff()
        if so is None or not Path(so).exists():
            return None
        _ref_tiff = ctypes.CDLL(str(so))
        _ref_tiff.ref_tiff_sinogram.restype = ctypes.c_long
        _ref_tiff.ref_tiff_sinogram.argtypes = [ctypes.c_char_p, ctypes.c_int, _F32, ctypes.c_long]
        _ref_tiff.ref_tiff_white_mean.restype = ctypes.c_double
        _ref_tiff.ref_tiff_white_mean.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    return _ref_tiff


def ref_tiff_negative_log_sinogram(config_dir, digits: int, shape) -> np.ndarray:
    """The reference's ingest on <config_dir>/configTiff (files in <config_dir>/../tif and
    ../Calibration). The reference exits the process on a missing file: call it only on
    complete inputs."""
    r = ref_tiff_lib()
    if r is None:
        raise RuntimeError("reference host build unavailable (oracle/_ref not built)")
    out = np.zeros(shape, np.float32)
    d = str(config_dir).rstrip("/") + "/"
    n = r.ref_tiff_sinogram(d.encode(), int(digits), out, out.size)
    if n != out.size:
        raise ValueError(f"reference sinogram has {n} values, expected {out.size}")
    return out


# ---- regularisation criteria (GG beta = 2, Huber) ----

def regularizer_criterion(vol: np.ndarray, dJ: np.ndarray, lam: float, total: int, optimal: int,
                          huber_threshold=None, reference: bool = False, beta: float = 2.0):
    """One call of the regulariser's getLaplacianRegularizationCriterion on FP32 volumes
    (the generalised Gaussian of shape `beta`, or Huber when `huber_threshold` is given):
    returns (dJ updated, jReg, normdJProjReg or None). reference=True runs the reference's
    own source built for the host (oracle/_ref) instead of the restatement."""
    vol = np.ascontiguousarray(vol, dtype=np.float32)
    d = np.array(dJ, dtype=np.float32, copy=True, order="C")
    out = np.full(2, np.nan)
    nz, ny, nx = vol.shape
    if reference:
        r = ref_reg_lib()
        if r is None:
            raise RuntimeError("reference host build unavailable (oracle/_ref not built)")
        if huber_threshold is None:
            r.ref_gg_criterion(vol, d, nx, ny, nz, float(lam), float(beta), total, optimal, out)
        else:
            r.ref_huber_criterion(vol, d, nx, ny, nz, float(lam), float(huber_threshold), total, optimal, out)
    elif huber_threshold is None:
        lib().oracle_gg_criterion_beta_f32(vol, d, nx, ny, nz, float(lam), float(beta), total, optimal, out)
    else:
        lib().oracle_huber_criterion_f32(vol, d, nx, ny, nz, float(lam), float(huber_threshold), total, optimal, out)
    return d, float(out[0]), (float(out[1]) if total < optimal else None)


_ref_reg = None


def ref_reg_lib():
    """The reference's regularisation criteria built for the host, or None."""
    global _ref_reg
    if _ref_reg is None:
        so = _build.build_reference_reg()
        if so is None or not Path(so).exists():
            return None
        _ref_reg = ctypes.CDLL(str(so))
        _ref_reg.ref_gg_criterion.argtypes = [_F32, _F32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                              ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64]
        _ref_reg.ref_huber_criterion.argtypes = [_F32, _F32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_float, ctypes.c_double, ctypes.c_int, ctypes.c_int, _F64]
    return _ref_reg


_ref_iter = None


def ref_iter_lib():
    """The reference's simple gradient loop built for the host, or None."""
    global _ref_iter
    if _ref_iter is None:
        so = _build.build_reference_iter()
        if so is None or not Path(so).exists():
            return None
        _ref_iter = ctypes.CDLL(str(so))
        _ref_iter.ref_gradient.argtypes = [_CFGP, _F32, _F32, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_void_p]
    return _ref_iter


def ref_simple_gradient(c, vol0: np.ndarray, real_sino: np.ndarray, iterations: int, lam: float,
                        optimal_step_nb: int, positivity: int = 0, huber_threshold=None, beta: float = 2.0,
                        weights=None) -> np.ndarray:
    """The reference's own Iter3D::doSimpleGradient, or Iter3D::doWeightedGradient when
    `weights` is given (RS / VI kernel sources, GG of shape `beta` or Huber regulariser),
    built for the host; returns the iterate."""
    r = ref_iter_lib()
    if r is None:
        raise RuntimeError("reference host build unavailable (oracle/_ref not built)")
    vol = np.array(vol0, dtype=np.float32, copy=True, order="C")
    sino = np.ascontiguousarray(real_sino, dtype=np.float32)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
    if w is not None and w.size != sino.size:
        raise ValueError("weights must have the sinogram's size")
    r.ref_gradient(ctypes.byref(_cfg(c)), vol, sino, iterations, float(lam), optimal_step_nb, positivity,
                   0 if huber_threshold is None else 1, float(huber_threshold or 0.0), float(beta),
                   None if w is None else w.ctypes.data_as(ctypes.c_void_p))
    return vol
