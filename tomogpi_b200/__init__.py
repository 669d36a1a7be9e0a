"""tomogpi_b200 -- B200-native cone-beam projector/backprojector pairs (RSVI, SIDDONVI).

Drop-in for TomoGPI's ``--op=proj`` / ``--op=back`` operators and its simple gradient
loop. The compute path is the hand-written sm_100a CUDA in ``csrc/`` behind the C-ABI
declared in ``include/tomogpi_b200.h``; this package is the host-side mirror of the
reference's operator classes over that C-ABI. There is no CPU fallback: without the
compiled library every operator raises ``LibraryError``.
"""
from .config import ConfigCT, ConfigIteration, ConfigComputeArchitecture, ConfigError  # noqa: F401
from ._lib import LibraryError, TomoError  # noqa: F401
from .operators import (Batch, Context, GradientParams, Solver, convert, gg_regularization,  # noqa: F401
                        huber_regularization, laplacian, phantom, sq_norm)
from . import phantoms  # noqa: F401

# Further modules, imported on use: serve (request loop), autotune, ingest (detector files,
# raw-file sidecars), iter3d (the MATLAB-style handle API), sharded (one job over several
# GPUs), replicas (jobs over several GPUs).

__all__ = ["ConfigCT", "ConfigIteration", "ConfigComputeArchitecture", "ConfigError", "LibraryError", "TomoError",
           "Batch", "Context", "GradientParams", "Solver", "laplacian", "sq_norm", "convert", "phantom", "phantoms",
           "gg_regularization", "huber_regularization"]
