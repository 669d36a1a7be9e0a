"""Host side of the MATLAB-style handle API: the dispatcher's argument checks and the
configCT writer it is tested with (no device needed)."""
import pytest

from tomogpi_b200 import ConfigCT
from tomogpi_b200.iter3d import PRECISION_CODES, STORAGE_CODES, tomogpi_iter_mex


def test_dispatcher_rejects_unknown_handles_and_commands():
    with pytest.raises(ValueError):
        tomogpi_iter_mex("new")
    with pytest.raises(ValueError):
        tomogpi_iter_mex("getLambda", 12345, "./")
    with pytest.raises(ValueError):
        tomogpi_iter_mex("delete")


def test_codes_follow_the_reference_enums():
    assert PRECISION_CODES == {"half": 0, "float": 1, "double": 2}
    assert STORAGE_CODES == {"mem_CPU": 0, "mem_GPU": 1, "mem_MGPU": 2}


def test_config_ct_file_round_trip(tmp_path):
    c = ConfigCT.cone_beam(48, 30, det=40).replace(real_volume_name="a.v", num_stop_angle=1.5)
    c.to_file(str(tmp_path / "configCT"))
    assert ConfigCT.from_file(str(tmp_path / "configCT")) == c
