"""The header-only C++ drop-in (include/tomogpi_b200/TomoGPI.hpp): a program written against
the reference's operator classes compiles and links against libtomogpi_b200 (CPU), and on
a GPU its operators' outputs match the oracle."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "dropin_main.cpp"
LIBDIR = ROOT / "tomogpi_b200"
CUDA_INC = "/usr/local/cuda/include"


def _build(out: Path) -> Path:
    exe = out / "dropin"
    cmd = ["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}", f"-I{CUDA_INC}", str(SRC), "-o", str(exe),
           f"-L{LIBDIR}", "-ltomogpi_b200", f"-Wl,-rpath,{LIBDIR}"]
    cudart = Path("/usr/local/cuda/lib64")
    if (cudart / "libcudart.so").exists():
        cmd += [f"-L{cudart}", "-lcudart", f"-Wl,-rpath,{cudart}"]
    else:
        cmd += ["-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def test_dropin_header_compiles_and_links(tmp_path):
    if not Path(CUDA_INC, "cuda_runtime.h").exists():
        pytest.skip("CUDA headers absent")
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_dropin_operators_match_oracle(tmp_path):
    import oracle
    from conftest import rel_l2
    from tomogpi_b200 import ConfigCT, phantoms

    exe = _build(tmp_path)
    n, P = 32, 24
    cfg = ConfigCT(fod=64.0, fdd=128.0, projection_nb=P, u_detector_size=64.0, v_detector_size=64.0,
                   u_detector_pixel_nb=n, v_detector_pixel_nb=n, x_volume_size=32.0, y_volume_size=32.0,
                   z_volume_size=32.0, x_volume_pixel_nb=n, y_volume_pixel_nb=n, z_volume_pixel_nb=n)
    vol = oracle.phantom(phantoms.config_phantom(0, n), n, n, n)
    vol.tofile(str(tmp_path / "volume.v"))
    res = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ))
    assert res.returncode == 0 and "ok" in res.stdout, res.stdout + res.stderr
    ld = lambda name, shape: np.fromfile(str(tmp_path / name), np.float32).reshape(shape)  # noqa: E731
    rs = ld("rs.s", cfg.sinogram_shape)
    assert rel_l2(rs, oracle.project(cfg, oracle.RS, vol)) <= 1e-5
    assert rel_l2(ld("siddon.s", cfg.sinogram_shape), oracle.project(cfg, oracle.SIDDON_REF, vol)) <= 1e-5
    assert rel_l2(ld("rs_um.s", cfg.sinogram_shape), oracle.project(cfg, oracle.RS_UM, vol)) <= 1e-5
    assert rel_l2(ld("vi.v", cfg.volume_shape), oracle.backproject(cfg, rs)) <= 1e-5
    assert rel_l2(ld("fdk.v", cfg.volume_shape), oracle.fdk_backproject(cfg, rs)) <= 1e-5
    rs_um = ld("rs_um.s", cfg.sinogram_shape)
    assert rel_l2(ld("vi_um.v", cfg.volume_shape), oracle.backproject(cfg, rs_um, um=True)) <= 1e-5
