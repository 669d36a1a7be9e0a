"""Python host layer over the C-ABI: contexts, operators and the gradient solver.

Device memory is held in torch CUDA tensors (torch is used for allocation and streams
only); every computation runs in libtomogpi_b200.so. Layouts follow the reference:
volume ``[z][y][x]`` and sinogram ``[phi][v][u]``.
"""
from __future__ import annotations

import ctypes
import weakref
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib as L
from .config import ConfigCT

try:  # torch is only needed for the device-pointer forms
    import torch
except ImportError:  # pragma: no cover
    torch = None

PROJECTORS = {"RS": L.PROJ_RS, "RS_UM": L.PROJ_RS_UM, "SIDDON_REF": L.PROJ_SIDDON_REF, "SIDDON": L.PROJ_SIDDON}
LAYOUTS = {"plain": L.RS_LAYOUT_PLAIN, "cell8": L.RS_LAYOUT_CELL8, "tex": L.RS_LAYOUT_TEX, "hybrid": L.RS_LAYOUT_HYBRID,
           "march": L.RS_LAYOUT_MARCH}
LAYOUT_NAMES = {v: k for k, v in LAYOUTS.items()}
VI_LAYOUTS = {"padded": 0, "tex": 1, "tma": 2}
VI_LAYOUT_NAMES = {v: k for k, v in VI_LAYOUTS.items()}
BACKPROJECTORS = {"VI": L.BACK_VI, "VI_UM": L.BACK_VI_UM, "RS_ADJOINT": L.BACK_RS_ADJOINT,
                  "SIDDON_ADJOINT": L.BACK_SIDDON_ADJOINT, "RS_UM_ADJOINT": L.BACK_RS_UM_ADJOINT, "FDK": L.BACK_FDK}


def _dtype_code(t) -> int:
    m = {torch.float32: L.F32, torch.bfloat16: L.BF16, torch.float16: L.F16}
    if t.dtype not in m:
        raise TypeError(f"unsupported storage dtype {t.dtype}")
    return m[t.dtype]


def _ptr(t) -> ctypes.c_void_p:
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream=None) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _kind(k, table) -> int:
    return table[k] if isinstance(k, str) else int(k)


class Context:
    """A geometry on one device (tomo_context): per-view tables and operator scratch."""

    def __init__(self, cfg: ConfigCT, device: int = 0, views=None):
        """views=(begin, count): a context over those views of the acquisition only
        (tomo_context_create_views); its sinograms hold `count` views."""
        L.load()
        self.cfg = cfg
        self.device = device
        h = ctypes.c_void_p()
        if views is None:
            self.views = (0, cfg.projection_nb)
            L.call("tomo_context_create", ctypes.byref(L.config_struct(cfg)), device, ctypes.byref(h))
        else:
            self.views = (int(views[0]), int(views[1]))
            L.call("tomo_context_create_views", ctypes.byref(L.config_struct(cfg)), device, self.views[0],
                   self.views[1], ctypes.byref(h))
        self.sinogram_shape = (self.views[1], cfg.v_detector_pixel_nb, cfg.u_detector_pixel_nb)
        self._h = h
        self._solvers = weakref.WeakSet()

    def close(self) -> None:
        for s in list(getattr(self, "_solvers", ())):
            s.close()  # solvers go before their context
        if getattr(self, "_h", None) and self._h.value:
            L.call("tomo_context_destroy", self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    # --- launch / layout choices ---------------------------------------------------
    @property
    def tuning(self) -> dict:
        t = L.TomoTuning()
        L.call("tomo_context_get_tuning", self._h, ctypes.byref(t))
        return {"rs_layout": LAYOUT_NAMES[t.rs_layout], "vi_zc": int(t.vi_zc),
                "vi_layout": VI_LAYOUT_NAMES[t.vi_layout], "rs_warp_u": int(t.rs_warp_u) or 8,
                "rs_tile_u": int(t.rs_tile_u) or 32}

    def rs_layout_in_use(self, dtype=None) -> str:
        """The RS input layout a projection of a volume of `dtype` uses."""
        out = ctypes.c_int32()
        code = {torch.float32: L.F32, torch.bfloat16: L.BF16, torch.float16: L.F16}[dtype or torch.float32]
        L.call("tomo_context_rs_layout", self._h, code, ctypes.byref(out))
        return LAYOUT_NAMES[out.value]

    def set_tuning(self, rs_layout=None, vi_zc=None, vi_layout=None, rs_warp_u=None, rs_tile_u=None) -> None:
        """rs_layout: "tex" | "hybrid" | "march" | "cell8" | "plain"; vi_zc: 1 | 2 | 4; vi_layout: "tex" | "padded" | "tma";
        rs_warp_u: 8 | 16 | 32 (rays of an RS warp along u); rs_tile_u: 16 | 32 | 64 | 128 (of a block)."""
        t = L.TomoTuning()
        L.call("tomo_context_get_tuning", self._h, ctypes.byref(t))
        if rs_warp_u is not None:
            t.rs_warp_u = int(rs_warp_u)
        if rs_tile_u is not None:
            t.rs_tile_u = int(rs_tile_u)
        if rs_layout is not None:
            t.rs_layout = LAYOUTS.get(rs_layout, rs_layout)
        if vi_zc is not None:
            t.vi_zc = int(vi_zc)
        if vi_layout is not None:
            t.vi_layout = VI_LAYOUTS.get(vi_layout, vi_layout)
        L.call("tomo_context_set_tuning", self._h, ctypes.byref(t))

    # --- operators on device tensors -------------------------------------------
    def project(self, kind, volume, out=None, dtype=None, stream=None):
        """sinogram := H volume  (Projector::doProjection)."""
        if out is None:
            out = torch.empty(self.sinogram_shape, dtype=dtype or volume.dtype, device=volume.device)
        self._check(volume, self.cfg.volume_shape)
        self._check(out, self.sinogram_shape)
        L.call("tomo_project", self._h, _kind(kind, PROJECTORS), _ptr(volume), _dtype_code(volume), _ptr(out),
               _dtype_code(out), _stream(stream))
        return out

    def backproject(self, kind, sinogram, out=None, dtype=None, stream=None):
        """volume := H^T sinogram  (BackProjector::doBackProjection)."""
        if out is None:
            out = torch.empty(self.cfg.volume_shape, dtype=dtype or sinogram.dtype, device=sinogram.device)
        self._check(sinogram, self.sinogram_shape)
        self._check(out, self.cfg.volume_shape)
        L.call("tomo_backproject", self._h, _kind(kind, BACKPROJECTORS), _ptr(sinogram), _dtype_code(sinogram),
               _ptr(out), _dtype_code(out), _stream(stream))
        return out

    # --- the mem_CPU form: host float32 buffers, copies inside ------------------
    def ramp_filter(self, sinogram, out=None, oversampling: int = 16, cutoff: float = 1.0, stream=None):
        """Ramp filter of filtered backprojection (ramp_filter_TOMO8.m): FP32 sinogram out."""
        self._check(sinogram, self.sinogram_shape)
        if out is None:
            out = torch.empty(self.sinogram_shape, dtype=torch.float32, device=sinogram.device)
        L.call("tomo_ramp_filter", self._h, _ptr(sinogram), _dtype_code(sinogram), _ptr(out), int(oversampling),
               float(cutoff), _stream(stream))
        return out

    def fdk(self, sinogram, oversampling: int = 16, cutoff: float = 1.0, dtype=None, stream=None):
        """Filtered backprojection: the ramp filter, then the FDK-weighted VI backprojection."""
        return self.backproject("FDK", self.ramp_filter(sinogram, oversampling=oversampling, cutoff=cutoff,
                                                        stream=stream), dtype=dtype, stream=stream)

    def project_host(self, kind, volume: np.ndarray, out: Optional[np.ndarray] = None) -> np.ndarray:
        vol = np.ascontiguousarray(volume, dtype=np.float32)
        if vol.shape != self.cfg.volume_shape:
            raise ValueError(f"volume shape {vol.shape} != {self.cfg.volume_shape}")
        if out is None:
            out = np.empty(self.sinogram_shape, np.float32)
        L.call("tomo_project_host", self._h, _kind(kind, PROJECTORS), vol.ctypes.data_as(ctypes.c_void_p),
               out.ctypes.data_as(ctypes.c_void_p))
        return out

    def backproject_host(self, kind, sinogram: np.ndarray, out: Optional[np.ndarray] = None) -> np.ndarray:
        sino = np.ascontiguousarray(sinogram, dtype=np.float32)
        if sino.shape != self.sinogram_shape:
            raise ValueError(f"sinogram shape {sino.shape} != {self.sinogram_shape}")
        if out is None:
            out = np.empty(self.cfg.volume_shape, np.float32)
        L.call("tomo_backproject_host", self._h, _kind(kind, BACKPROJECTORS), sino.ctypes.data_as(ctypes.c_void_p),
               out.ctypes.data_as(ctypes.c_void_p))
        return out

    def count_samples(self, kind, stream=None) -> int:
        n = ctypes.c_ulonglong()
        L.call("tomo_count_samples", self._h, _kind(kind, PROJECTORS), ctypes.byref(n),
               _stream(stream) if torch is not None and torch.cuda.is_available() else None)
        return int(n.value)

    def geometry(self):
        s = np.zeros(11, np.float32)
        a = np.zeros(self.cfg.projection_nb, np.float32)
        b = np.zeros(self.cfg.projection_nb, np.float32)
        L.call("tomo_context_geometry", self._h, s.ctypes.data_as(ctypes.c_void_p),
               a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p))
        return s, a, b

    def errors(self, clear: bool = True) -> int:
        bits = ctypes.c_uint()
        L.call("tomo_context_errors", self._h, ctypes.byref(bits), int(clear))
        return int(bits.value)

    @staticmethod
    def _check(t, shape):
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"shape {tuple(t.shape)} != {tuple(shape)}")


@dataclass
class GradientParams:
    """configIteration for Iter3D::doSimpleGradient (the regulariser and the weighted form are
    chosen on the Solver: set_regularizer, set_weights)."""

    gradient_iteration_nb: int = 20
    optimal_step_iteration_nb: int = 21
    regularization_parameter: float = 0.01
    positivity: int = 0
    projector: str = "RS"
    backprojector: str = "VI"
    storage: str = "f32"  # f32 | bf16 | f16: storage of the operator inputs/outputs
    real_f32: bool = False  # the real (measured) sinogram stays FP32 whatever the storage

    def struct(self) -> L.TomoGradientParams:
        st = {"f32": L.F32, "bf16": L.BF16, "f16": L.F16}[self.storage]
        return L.TomoGradientParams(_kind(self.projector, PROJECTORS), _kind(self.backprojector, BACKPROJECTORS), st,
                                    self.gradient_iteration_nb, self.optimal_step_iteration_nb,
                                    float(self.regularization_parameter), int(self.positivity), int(self.real_f32))

    def real_dtype(self):
        """numpy dtype name of the real sinogram the solver and the batch read."""
        return "f32" if self.real_f32 else self.storage


def _check_real(real_sinogram, params: GradientParams) -> None:
    """The real sinogram must be in the type the solver reads (the storage type, or FP32
    with real_f32): the library takes a raw pointer and cannot tell."""
    want = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[params.real_dtype()]
    if real_sinogram.dtype != want or not real_sinogram.is_contiguous():
        raise TypeError(f"the real sinogram must be a contiguous {want} tensor for storage {params.storage}"
                        f"{' with real_f32' if params.real_f32 else ''}, got {real_sinogram.dtype}")


class Solver:
    """Device-resident simple gradient descent (tomo_solver)."""

    def __init__(self, ctx: Context, params: GradientParams):
        self.ctx = ctx
        self.params = params
        h = ctypes.c_void_p()
        L.call("tomo_solver_create", ctx.handle, ctypes.byref(params.struct()), ctypes.byref(h))
        self._h = h
        ctx._solvers.add(self)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.call("tomo_solver_destroy", self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def iterate(self, volume, real_sinogram, first: int = 1, count: Optional[int] = None, stream=None):
        """Runs iterations [first, first+count) in place on the FP32 volume tensor."""
        if volume.dtype != torch.float32:
            raise TypeError("the master iterate is FP32")
        _check_real(real_sinogram, self.params)
        count = self.params.gradient_iteration_nb - first + 1 if count is None else count
        L.call("tomo_solver_iterate", self._h, _ptr(volume), _ptr(real_sinogram), int(first), int(count),
               _stream(stream))
        return volume

    def iterate_host(self, volume: np.ndarray, real_sinogram: np.ndarray, first: int = 1,
                     count: Optional[int] = None, stream=None) -> np.ndarray:
        """Host-buffer form: FP32 iterate and real sinogram (storage dtype, or FP32 with real_f32) in host memory,
        copied in and out around the iterations (pinned buffers make the copies async)."""
        if volume.dtype != np.float32 or not volume.flags.c_contiguous:
            raise TypeError("the host iterate must be a contiguous float32 array")
        want = {"f32": np.float32, "f16": np.float16}.get(self.params.real_dtype())
        if want is not None and real_sinogram.dtype != want:
            raise TypeError(f"real sinogram must be {want.__name__} for storage {self.params.storage}"
                            f"{' (real_f32)' if self.params.real_f32 else ''}")
        count = self.params.gradient_iteration_nb - first + 1 if count is None else count
        L.call("tomo_solver_iterate_host", self._h, volume.ctypes.data_as(ctypes.c_void_p),
               real_sinogram.ctypes.data_as(ctypes.c_void_p), int(first), int(count),
               _stream(stream) if torch is not None else None)
        return volume

    def set_regularizer(self, kind: str = "gg", huber_threshold: float = 0.0, beta: float = 2.0) -> None:
        """"gg" (generalised Gaussian with shape parameter beta >= 1, 2 by default) or "huber"
        with its threshold (configIteration penaltyFunction / huberThreshold / beta)."""
        code = {"gg": 0, "ggaussian": 0, "huber": 1}.get(str(kind).lower())
        if code is None:
            raise ValueError(f"unknown regulariser {kind!r}")
        L.call("tomo_solver_set_regularizer", self._h, code, float(huber_threshold))
        if code == 0:
            L.call("tomo_solver_set_gg_beta", self._h, float(beta))

    def set_weights(self, weights, stream=None) -> None:
        """The weighted gradient (Iter3D::doWeightedGradient, Iter3D_Algo_Gradient.cu:227-373):
        the residual is multiplied by `weights` (an FP32 sinogram of the solver's views, a
        device tensor or a host array; the solver keeps a copy) before each backprojection,
        and alpha_min starts at -999999999999. None returns to the simple gradient. Before
        the first iteration only."""
        if weights is None:
            L.call("tomo_solver_set_weights", self._h, None, 0, _stream(stream))
            return
        shape = self.ctx.sinogram_shape
        if isinstance(weights, np.ndarray):
            w = np.ascontiguousarray(weights, dtype=np.float32)
            if w.shape != tuple(shape):
                raise ValueError(f"weights of shape {w.shape}, the solver's sinogram is {tuple(shape)}")
            L.call("tomo_solver_set_weights", self._h, w.ctypes.data_as(ctypes.c_void_p), 1, None)
            return
        if weights.dtype != torch.float32 or not weights.is_contiguous() or tuple(weights.shape) != tuple(shape):
            raise TypeError(f"weights must be a contiguous float32 tensor of shape {tuple(shape)}")
        L.call("tomo_solver_set_weights", self._h, _ptr(weights), 0, _stream(stream))

    PHASE_GRADIENT, PHASE_NORMS, PHASE_UPDATE = 1, 2, 4

    def phase(self, volume, real_sinogram, iteration: int, phases: int, stream=None) -> None:
        """One iteration's phases (tomo_solver_phase) on the FP32 volume tensor; real_sinogram
        is read by PHASE_GRADIENT only (may be None otherwise)."""
        L.call("tomo_solver_phase", self._h, _ptr(volume),
               _ptr(real_sinogram) if real_sinogram is not None else None, int(iteration), int(phases),
               _stream(stream))

    def buffers(self):
        """(dJ, norms) as torch tensors viewing the solver's device buffers (no copy): the
        FP32 gradient volume and its 8 FP64 norm slots."""
        dj, nrm = ctypes.c_void_p(), ctypes.c_void_p()
        L.call("tomo_solver_buffers", self._h, ctypes.byref(dj), ctypes.byref(nrm))
        shape = self.ctx.cfg.volume_shape
        return (_device_view(dj.value, shape, "<f4", self.ctx.device),
                _device_view(nrm.value, (8,), "<f8", self.ctx.device))

    def set_timing(self, enable: bool = True) -> None:
        L.call("tomo_solver_set_timing", self._h, int(enable))

    def stats(self, reset: bool = False, stream=None) -> dict:
        st = L.TomoSolverStats()
        L.call("tomo_solver_get_stats", self._h, ctypes.byref(st), int(reset), _stream(stream))
        return {"proj_ms": st.proj_ms, "proj_launches": st.proj_launches, "back_ms": st.back_ms,
                "back_launches": st.back_launches, "kernel_launches": int(st.kernel_launches)}

    def alphas(self, stream=None) -> np.ndarray:
        n = max(self.params.gradient_iteration_nb, 1)
        out = np.zeros(n, np.float64)
        w = ctypes.c_int32()
        L.call("tomo_solver_alphas", self._h, out.ctypes.data_as(ctypes.c_void_p), n, ctypes.byref(w), _stream(stream))
        return out[: w.value]

    def get_state(self, stream=None):
        a = ctypes.c_double()
        i = ctypes.c_int32()
        L.call("tomo_solver_get_state", self._h, ctypes.byref(a), ctypes.byref(i), _stream(stream))
        return float(a.value), int(i.value)

    def set_state(self, alpha_min: float, next_iteration: int, stream=None):
        L.call("tomo_solver_set_state", self._h, float(alpha_min), int(next_iteration), _stream(stream))


def tuning_struct(rs_layout="tex", vi_zc=1, rs_warp_u=0, rs_tile_u=0) -> L.TomoTuning:
    t = L.TomoTuning()
    t.rs_layout = LAYOUTS.get(rs_layout, rs_layout)
    t.vi_zc = int(vi_zc)
    t.rs_warp_u = int(rs_warp_u)
    t.rs_tile_u = int(rs_tile_u)
    return t


class Batch:
    """Many reconstructions advanced together (tomo_batch): every phase of an iteration is
    one launch over all live jobs; one iteration is replayed from a CUDA graph."""

    def __init__(self, params: GradientParams, device: int = 0, graph: bool = True):
        L.load()
        self.params = params
        self.device = device
        h = ctypes.c_void_p()
        L.call("tomo_batch_create", device, ctypes.byref(params.struct()), ctypes.byref(h))
        self._h = h
        self._keep = {}  # job id -> (volume, real sinogram) so the buffers outlive the job
        if not graph:
            L.call("tomo_batch_set_graph", self._h, 0)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.call("tomo_batch_destroy", self._h)
            self._h = ctypes.c_void_p()
            self._keep.clear()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def footprint(cfg: ConfigCT, params: GradientParams, rs_layout="tex", vi_zc=1) -> int:
        n = ctypes.c_size_t()
        L.call("tomo_batch_footprint", ctypes.byref(L.config_struct(cfg)), ctypes.byref(params.struct()),
               ctypes.byref(tuning_struct(rs_layout, vi_zc)), ctypes.byref(n))
        return int(n.value)

    def add(self, cfg: ConfigCT, volume, real_sinogram, rs_layout="tex", vi_zc=1, rs_warp_u=0, rs_tile_u=0) -> int:
        if volume.dtype != torch.float32 or tuple(volume.shape) != cfg.volume_shape:
            raise ValueError("the iterate is an FP32 tensor of the volume shape")
        if tuple(real_sinogram.shape) != cfg.sinogram_shape:
            raise ValueError("real sinogram shape mismatch")
        _check_real(real_sinogram, self.params)
        j = ctypes.c_int32()
        L.call("tomo_batch_add", self._h, ctypes.byref(L.config_struct(cfg)), ctypes.byref(tuning_struct(rs_layout, vi_zc, rs_warp_u, rs_tile_u)),
               _ptr(volume), _ptr(real_sinogram), ctypes.byref(j))
        self._keep[j.value] = (volume, real_sinogram)
        return int(j.value)

    def remove(self, job: int) -> None:
        L.call("tomo_batch_remove", self._h, int(job))
        self._keep.pop(job, None)

    def iterate(self, count: int = 1, stream=None) -> None:
        L.call("tomo_batch_iterate", self._h, int(count), _stream(stream))

    def set_share(self, fraction: float) -> None:
        """Fraction of the persistent CTAs that take work items (takes effect at once)."""
        L.call("tomo_batch_set_share", self._h, float(fraction))

    def host_times(self) -> dict:
        """Host milliseconds spent in iterate: queue rebuilds, captures, graph updates, launches."""
        ms = (ctypes.c_double * 4)()
        L.call("tomo_batch_host_times", self._h, ms)
        return {"rebuild_ms": ms[0], "capture_ms": ms[1], "instantiate_ms": ms[2], "launch_ms": ms[3]}

    def parked_bytes(self) -> int:
        """Device bytes of texture arrays kept from removed jobs for reuse."""
        n = ctypes.c_size_t()
        L.call("tomo_batch_trim", self._h, ctypes.byref(n))
        return int(n.value)

    def trim(self) -> None:
        """Frees the parked texture arrays (synchronises the device)."""
        L.call("tomo_batch_trim", self._h, None)

    def set_priority(self, priority: int) -> None:
        """CUDA stream priority of the batch's kernels (lower = more urgent)."""
        L.call("tomo_batch_set_priority", self._h, int(priority))

    def status(self, job: int, stream=None):
        it = ctypes.c_int32()
        am = ctypes.c_double()
        L.call("tomo_batch_job_status", self._h, int(job), ctypes.byref(it), ctypes.byref(am), _stream(stream))
        return int(it.value), float(am.value)

    def alphas(self, job: int, stream=None) -> np.ndarray:
        n = max(self.params.gradient_iteration_nb, 1)
        out = np.zeros(n, np.float64)
        w = ctypes.c_int32()
        L.call("tomo_batch_job_alphas", self._h, int(job), out.ctypes.data_as(ctypes.c_void_p), n, ctypes.byref(w),
               _stream(stream))
        return out[: w.value]

    def stats(self) -> dict:
        live = ctypes.c_int32()
        items = ctypes.c_int64()
        by = ctypes.c_size_t()
        la = ctypes.c_int64()
        L.call("tomo_batch_stats", self._h, ctypes.byref(live), ctypes.byref(items), ctypes.byref(by), ctypes.byref(la))
        return {"live_jobs": live.value, "work_items": items.value, "bytes": by.value, "kernel_launches": la.value}


# --- element-wise helpers -----------------------------------------------------------
def laplacian(volume, out=None, stream=None):
    out = torch.empty_like(volume) if out is None else out
    nz, ny, nx = volume.shape
    L.call("tomo_laplacian", _ptr(volume), _ptr(out), nx, ny, nz, _stream(stream))
    return out


def sq_norm(x, stream=None) -> float:
    acc = torch.zeros(1, dtype=torch.float64, device=x.device)
    L.call("tomo_sq_norm", _ptr(x), _dtype_code(x), x.numel(), _ptr(acc), _stream(stream))
    return float(acc.item())


def gg_regularization(volume, dJ, lam: float, total_iteration: int, optimal_step_iteration_nb: int, stream=None,
                      beta: float = 2.0):
    """Generalised-Gaussian regularisation criterion on FP32 device volumes, in place:
    dJ += beta*lam * L(g) with g = L volume for beta = 2, sign(volume) |volume|^(beta-1)
    otherwise; returns (jReg = sum |L volume|^beta, normdJProjReg = beta sum |L dJ|^beta), the
    latter None when total_iteration >= optimal_step_iteration_nb
    (GeneralizedGaussianRegularizer_CPU.cu:158-226)."""
    _check_f32_volume(volume, dJ)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=volume.device)
    nz, ny, nx = volume.shape
    L.call("tomo_gg_regularization_beta", _ptr(volume), _ptr(dJ), nx, ny, nz, float(lam), float(beta),
           int(total_iteration), int(optimal_step_iteration_nb), _ptr(out), _stream(stream))
    j, n = out.tolist()
    return j, (n if total_iteration < optimal_step_iteration_nb else None)


def huber_regularization(volume, dJ, lam: float, threshold: float, total_iteration: int,
                         optimal_step_iteration_nb: int, stream=None):
    """Huber regularisation criterion on FP32 device volumes: dJ += lam * L(psi'(L volume)) in
    place; returns (jReg, normdJProjReg), the latter None when total_iteration >=
    optimal_step_iteration_nb (HuberRegularizer_CPU.cu:206-253)."""
    _check_f32_volume(volume, dJ)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=volume.device)
    nz, ny, nx = volume.shape
    L.call("tomo_huber_regularization", _ptr(volume), _ptr(dJ), nx, ny, nz, float(lam), float(threshold),
           int(total_iteration), int(optimal_step_iteration_nb), _ptr(out), _stream(stream))
    j, n = out.tolist()
    return j, (n if total_iteration < optimal_step_iteration_nb else None)


class _CudaArray:
    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2, "strides": None}


def _device_view(ptr: int, shape, typestr: str, device: int):
    """A torch tensor over device memory owned by the library (valid while its owner lives)."""
    return torch.as_tensor(_CudaArray(ptr, shape, typestr), device=f"cuda:{device}")


def _check_f32_volume(*ts):
    for t in ts:
        if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous() or t.dim() != 3:
            raise ValueError("expected contiguous 3-D float32 CUDA volumes")
    if any(t.shape != ts[0].shape for t in ts):
        raise ValueError("volume shapes differ")


def convert(x, dtype, stream=None):
    out = torch.empty(x.shape, dtype=dtype, device=x.device)
    L.call("tomo_convert", _ptr(x), _dtype_code(x), _ptr(out), _dtype_code(out), x.numel(), _stream(stream))
    return out


def phantom(ellipsoids: np.ndarray, nx: int, ny: int, nz: int, device: int = 0, stream=None):
    """Sum-of-ellipsoids phantom (phantom3d.m semantics) rasterised on the GPU, FP32."""
    e = np.ascontiguousarray(ellipsoids, dtype=np.float64).reshape(-1, 10)
    out = torch.empty((nz, ny, nx), dtype=torch.float32, device=f"cuda:{device}")
    L.call("tomo_phantom", e.ctypes.data_as(ctypes.c_void_p), e.shape[0], nx, ny, nz, _ptr(out), _stream(stream))
    return out
