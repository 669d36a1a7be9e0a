"""Generates the golden fixtures of tests/golden/ by running the REFERENCE's own sources
(projection_ER_kernel.cuh, projection_ER_kernel_UM.cuh, backprojection3D_kernel_16reg*.cuh,
FDK3D_kernel_16reg.cuh, SiddonProjector_compute_C_mem_CPU.cpp), compiled for the host by oracle/build.py from the
TomoGPI source tree. Needs that source tree; run from the repository root:

    python tests/golden/make_golden.py

Each case stores its geometry, a seeded input and the reference outputs (float32).
"""
import json
import sys
import zlib
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle  # noqa: E402
from tomogpi_b200.config import ConfigCT  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = {
    # small cone-beam set-ups in voxel units (FOD = 2N, magnification 2, pitch 2)
    "n16_p8": dict(n=16, views=8, det=16),
    "n32_p16_det48": dict(n=32, views=16, det=48, pitch=1.5),
    "n32_p16_short": dict(n=32, views=16, det=32, fod=40.0),  # strong cone angle, rays leave through z
    "n32_p8_odd_start": dict(n=32, views=8, det=32, start=(1, 3), stop=(7, 3)),
}


def make_cfg(spec):
    c = ConfigCT.cone_beam(spec["n"], spec["views"], det=spec["det"], pitch=spec.get("pitch", 2.0), fod=spec.get("fod"))
    if "start" in spec:
        c = c.replace(num_start_angle=spec["start"][0], den_start_angle=spec["start"][1],
                      num_stop_angle=spec["stop"][0], den_stop_angle=spec["stop"][1])
    return c


def main():
    if oracle.ref_lib() is None:
        raise SystemExit("the reference host build (oracle/_ref) is not available")
    for name, spec in CASES.items():
        c = make_cfg(spec)
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        vol = rng.random(c.volume_shape, dtype=np.float32)
        sino = rng.random(c.sinogram_shape, dtype=np.float32)
        outs = {
            "rs": oracle.ref_project(c, oracle.RS, vol),
            "rs_um": oracle.ref_project(c, oracle.RS_UM, vol),
            "vi": oracle.ref_backproject(c, sino, um=False),
            "vi_um": oracle.ref_backproject(c, sino, um=True),
            "fdk": oracle.ref_fdk_backproject(c, sino),
        }
        if c.u_detector_pixel_nb % 16 == 0 and c.v_detector_pixel_nb % 16 == 0 and c.projection_nb % 8 == 0:
            outs["siddon_ref"] = oracle.ref_project(c, oracle.SIDDON_REF, vol)
        np.savez_compressed(OUT / f"{name}.npz", volume=vol, sinogram=sino, **outs)
        (OUT / f"{name}.json").write_text(json.dumps(c.__dict__, indent=1, sort_keys=True))
        print(name, {k: float(np.abs(v).max()) for k, v in outs.items()})


if __name__ == "__main__":
    main()
