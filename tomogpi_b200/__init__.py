"""tomogpi_b200 -- B200-native cone-beam projector/backprojector pairs (RSVI, SIDDONVI).

Drop-in for TomoGPI's ``--op=proj`` / ``--op=back`` operators and its simple gradient
loop. The compute path is the hand-written sm_100a CUDA in ``csrc/`` behind the C-ABI
declared in ``include/tomogpi_b200.h``; this package is the host-side mirror of the
reference's operator classes over that C-ABI.
"""
from .config import ConfigCT, ConfigIteration, ConfigComputeArchitecture, ConfigError  # noqa: F401

__all__ = ["ConfigCT", "ConfigIteration", "ConfigComputeArchitecture", "ConfigError"]
