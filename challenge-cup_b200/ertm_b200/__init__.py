"""ertm_b200 — B200-native hot path of the ERTM reverse-time migration.

Drop-in for the reference's ``ertm.propagation`` / ``ertm.imaging`` /
``ertm.solver`` call signatures; the work runs in the sm_100a CUDA library
``libertm_b200.so`` (see ``include/ertm_b200.h``).  Importing the package
needs no GPU; the first propagator created initialises the device and
raises ``SolverError`` if the library or a B200 is missing.
"""

from __future__ import annotations

__version__ = "0.1.0"

from . import segy
from .config import ImagingConfig, QConfig, SolverConfig
from .data import NumpyDataStore
from .exceptions import (ConfigError, DataError, ERTMError, ImagingError, NonFiniteWavefieldError, PipelineError,
                         SolverError)
from .imaging import RTMImager, build_imager
from .preprocess import prepare_shot
from .propagation import (AcousticPropagator, ElasticPropagator, PropagationSpec, QOptions,
                          ViscoacousticPropagator, build_propagator, check_stability, forward_shot, run_forward,
                          source_wavelet)
from .qcomp import QCompensator, attenuate_record, build_compensator
from .solver import FiniteDifferenceSolver, build_solver
from .stacking import stack_images
from .types import ElasticModel, GridSpec, ImageResult, ReceiverSpec, ShotRecord, SourceSpec

__all__ = [
    "AcousticPropagator", "ConfigError", "DataError", "ERTMError", "ElasticModel", "ElasticPropagator",
    "FiniteDifferenceSolver", "GridSpec", "ImageResult", "ImagingConfig", "ImagingError", "PipelineError",
    "PropagationSpec", "QConfig", "QOptions", "RTMImager", "ReceiverSpec", "ShotRecord", "SolverConfig",
    "NonFiniteWavefieldError", "SolverError", "SourceSpec", "ViscoacousticPropagator", "build_imager", "build_propagator", "build_solver",
    "check_stability", "forward_shot", "run_forward", "source_wavelet", "stack_images",
    "NumpyDataStore", "QCompensator", "attenuate_record", "build_compensator", "prepare_shot", "segy",
]
