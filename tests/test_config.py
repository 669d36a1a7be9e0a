"""configCT / configIteration readers follow Config::getConfigFileField semantics."""
import pytest

from tomogpi_b200.config import ConfigCT, ConfigError, ConfigIteration, read_field

CONFIG_CT = """[Acquisition]
FOD 98 mm
FDD 230 mm
projectionNb 256
numStartAngle 0
denStartAngle 1
numStopAngle 2
denStopAngle 1
acquisitionScheme Uniform (Uniform, NonUniform)

[Detector]
horizontalDetectorSize 14.2 mm
verticalDetectorSize 14.2 mm
horizontalDetectorPixelNb 256
verticalDetectorPixelNb 256

[Volume]
xVolumeSize 6.05 mm
yVolumeSize 6.05 mm
zVolumeSize 5.86 mm
xVolumePixelNb 256
yVolumePixelNb 256
zVolumePixelNb 256

[Initialization]
initVolumeName none
realVolumeName /data/phantom.v
"""

CONFIG_IT = """[Iteration]
globalIterationNb 1
gradientIterationNb 10
optimalStepIterationNb 10
[PenaltyFunction]
regularizationParameter 0.01
penaltyFunction GGaussian (Huber, GGaussian)
gradient Simple (Simple,Conjugate)
positivity 0
beta 2.0
"""


def test_config_ct_fields(tmp_path):
    p = tmp_path / "configCT"
    p.write_text(CONFIG_CT)
    c = ConfigCT.from_file(str(p))
    assert (c.fod, c.fdd, c.projection_nb) == (98.0, 230.0, 256)
    assert (c.u_detector_size, c.u_detector_pixel_nb) == (14.2, 256)
    assert (c.z_volume_size, c.z_volume_pixel_nb) == (5.86, 256)
    assert c.real_volume_name == "/data/phantom.v"
    assert c.volume_shape == (256, 256, 256) and c.sinogram_shape == (256, 256, 256)
    assert c.voxel_ray_updates == 256 ** 4


def test_first_match_wins_and_missing_field(tmp_path):
    p = tmp_path / "cfg"
    p.write_text("a 1\nfoo 2 foo 3\nfoo 4\n")
    assert read_field(str(p), "foo", int) == 2
    with pytest.raises(ConfigError):
        read_field(str(p), "bar")
    with pytest.raises(ConfigError):
        read_field(str(tmp_path / "nope"), "foo")


def test_config_iteration(tmp_path):
    p = tmp_path / "configIteration"
    p.write_text(CONFIG_IT)
    it = ConfigIteration.from_file(str(p))
    assert it.gradient_iteration_nb == 10 and it.optimal_step_iteration_nb == 10
    assert it.regularization_parameter == 0.01 and it.penalty_function == "GGaussian" and it.beta == 2.0


def test_phi_values():
    import math

    c = ConfigCT.cone_beam(16, 8)
    phi = c.phi()
    assert phi[0] == 0.0 and abs(phi[1] - 2 * math.pi / 8) < 1e-15
