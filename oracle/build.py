"""Build recipe for the oracle (test infrastructure only).

* ``oracle/libtomo_oracle.so``: the CPU restatement in ``tomo_oracle.cpp``.
* ``oracle/_ref/libtomo_ref.so``: the reference's own kernel sources and its Siddon C
  file, compiled for the host in place from the TomoGPI source tree through the shims in
  ``oracle/ref_shim``. Built only where that source tree exists (it is absent on GPU
  machines, which use the prebuilt library). Nothing from it is copied into this
  repository; its output directory is git-ignored.
* ``oracle/_ref/libtomo_ref_reg.so``: the reference's regularisation criteria
  (``src/CPP/GeneralizedGaussianRegularizer_CPU.cu``, ``src/CPP/HuberRegularizer_CPU.cu``
  with their headers in ``inc/``) compiled in place the same way, with the stand-ins of
  ``oracle/ref_shim/reg`` for the volume, convolution and base classes.
* ``oracle/_ref/libtomo_ref_iter.so``: the reference's simple gradient loop
  (``src/CPP/Iter3D_Algo_Gradient.cu``, ``Iter3D::doSimpleGradient``) with its regularisers,
  compiled in place with the stand-ins of ``oracle/ref_shim/iter`` (an Iter3D with the
  members the loop calls, whose projector and backprojector are the reference's kernel
  sources of ``libtomo_ref.so``) and ``oracle/ref_shim/reg``.
* ``oracle/_ref/libtomo_ref_tiff.so``: the reference's detector-file ingest
  (``inc/Config/ConfigTiff.hpp``, ``src/CPP/Config/ConfigTiff.cpp``,
  ``src/CPP/ImageTiff.cu``) compiled in place with the stand-in headers of
  ``oracle/ref_shim/tiff``. Those sources include their headers with quotes, so gcc's
  ``-I-`` (quote includes search only the listed directories, never the including file's
  own) routes ``Config.hpp`` and the image/sinogram headers to the stand-ins instead of
  the reference's GPU class tree.

Both are compiled with ``-ffp-contract=off`` so that no multiply-add is fused and every
FP32 operation rounds exactly as written.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REFERENCE = Path(os.environ.get("TOMOGPI_REFERENCE", "/root/reference"))
# The system g++ carries the OpenMP runtime; prefer it over a CXX override without one.
CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else os.environ.get("CXX", "g++")
FLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-std=c++17", "-shared"]

ORACLE_SO = HERE / "libtomo_oracle.so"
REF_SO = HERE / "_ref" / "libtomo_ref.so"
REF_TIFF_SO = HERE / "_ref" / "libtomo_ref_tiff.so"
REF_REG_SO = HERE / "_ref" / "libtomo_ref_reg.so"
REF_ITER_SO = HERE / "_ref" / "libtomo_ref_iter.so"


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("oracle build failed: " + " ".join(cmd))


def _stale(out: Path, inputs: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.stat().st_mtime > t for p in inputs if p.exists())


def build_oracle(force: bool = False) -> Path:
    src = HERE / "tomo_oracle.cpp"
    if force or _stale(ORACLE_SO, [src, Path(__file__)]):
        _run([CXX, *FLAGS, str(src), "-o", str(ORACLE_SO)])
    return ORACLE_SO


def build_reference(force: bool = False) -> Path | None:
    """Compile the reference's own sources (needs the TomoGPI tree); None if absent."""
    src_root = REFERENCE / "src" / "TomoGPI_lib" / "src"
    if not src_root.is_dir():
        return REF_SO if REF_SO.exists() else None
    shim = HERE / "ref_shim"
    tus = ["shim_common.cpp", "ref_rs_box.cpp", "ref_rs_um.cpp", "ref_vi.cpp", "ref_vi_um.cpp", "ref_fdk.cpp",
           "ref_siddon.cpp"]
    inputs = [shim / t for t in tus] + list(shim.glob("*.h")) + list(shim.glob("*.cuh")) + [Path(__file__)]
    if not (force or _stale(REF_SO, inputs)):
        return REF_SO
    REF_SO.parent.mkdir(parents=True, exist_ok=True)
    incs = [
        f"-I{shim}",
        f"-I{src_root / 'CUDA' / 'Projector'}",
        f"-I{src_root / 'CUDA' / 'BackProjector'}",
        f"-I{src_root / 'CPP'}",
    ]
    _run([CXX, *FLAGS, *incs, *[str(shim / t) for t in tus], "-o", str(REF_SO)])
    return REF_SO


def build_reference_tiff(force: bool = False) -> Path | None:
    """Compile the reference's detector-file ingest (needs the TomoGPI tree); None if absent."""
    lib_root = REFERENCE / "src" / "TomoGPI_lib"
    srcs = [lib_root / "src" / "CPP" / "Config" / "ConfigTiff.cpp", lib_root / "src" / "CPP" / "ImageTiff.cu"]
    if not all(s.exists() for s in srcs):
        return REF_TIFF_SO if REF_TIFF_SO.exists() else None
    shim = HERE / "ref_shim" / "tiff"
    inputs = list(shim.iterdir()) + [Path(__file__)]
    if not (force or _stale(REF_TIFF_SO, inputs)):
        return REF_TIFF_SO
    REF_TIFF_SO.parent.mkdir(parents=True, exist_ok=True)
    _run([CXX, *FLAGS, "-w", f"-I{shim}", "-I-", f"-I{lib_root / 'inc' / 'Config'}", f"-I{lib_root / 'inc'}",
          str(shim / "ref_tiff.cpp"), str(srcs[0]), "-x", "c++", str(srcs[1]), "-o", str(REF_TIFF_SO)])
    return REF_TIFF_SO


def build_reference_reg(force: bool = False) -> Path | None:
    """Compile the reference's regularisation criteria (needs the TomoGPI tree); None if absent."""
    lib_root = REFERENCE / "src" / "TomoGPI_lib"
    srcs = [lib_root / "src" / "CPP" / "GeneralizedGaussianRegularizer_CPU.cu",
            lib_root / "src" / "CPP" / "HuberRegularizer_CPU.cu"]
    if not all(s.exists() for s in srcs):
        return REF_REG_SO if REF_REG_SO.exists() else None
    shim = HERE / "ref_shim" / "reg"
    inputs = list(shim.iterdir()) + [Path(__file__)]
    if not (force or _stale(REF_REG_SO, inputs)):
        return REF_REG_SO
    REF_REG_SO.parent.mkdir(parents=True, exist_ok=True)
    _run([CXX, *FLAGS, "-w", "-DCOMPUTE_J", f"-I{shim}", "-I-", f"-I{lib_root / 'inc'}", str(shim / "ref_reg.cpp"),
          "-x", "c++", *map(str, srcs), "-o", str(REF_REG_SO)])
    return REF_REG_SO


def build_reference_iter(force: bool = False) -> Path | None:
    """Compile the reference's simple gradient loop over its own operator sources (needs the
    TomoGPI tree and libtomo_ref.so); None if absent."""
    lib_root = REFERENCE / "src" / "TomoGPI_lib"
    srcs = [lib_root / "src" / "CPP" / "Iter3D_Algo_Gradient.cu",
            lib_root / "src" / "CPP" / "GeneralizedGaussianRegularizer_CPU.cu",
            lib_root / "src" / "CPP" / "HuberRegularizer_CPU.cu"]
    if not all(s.exists() for s in srcs) or build_reference() is None:
        return REF_ITER_SO if REF_ITER_SO.exists() else None
    ishim, rshim = HERE / "ref_shim" / "iter", HERE / "ref_shim" / "reg"
    inputs = list(ishim.iterdir()) + list(rshim.iterdir()) + [Path(__file__), REF_SO]
    if not (force or _stale(REF_ITER_SO, inputs)):
        return REF_ITER_SO
    _run([CXX, *FLAGS, "-w", f"-I{ishim}", f"-I{rshim}", "-I-", f"-I{lib_root / 'inc'}", str(ishim / "ref_iter.cpp"),
          "-x", "c++", *map(str, srcs), f"-L{REF_SO.parent}", "-ltomo_ref", "-Wl,-rpath,$ORIGIN", "-o",
          str(REF_ITER_SO)])
    return REF_ITER_SO


def main() -> None:
    print(build_oracle(force="--force" in sys.argv))
    print(build_reference(force="--force" in sys.argv))
    print(build_reference_tiff(force="--force" in sys.argv))
    print(build_reference_reg(force="--force" in sys.argv))
    print(build_reference_iter(force="--force" in sys.argv))


if __name__ == "__main__":
    main()
