"""B200-native Debye scattering backend for pripps-style SAXS calculations.

The exact O(N²·Q) Debye pair sum, computed as the six partial profiles of a
cached Debye model, runs in hand-written sm_100a CUDA kernels behind the C ABI
in include/pripps_debye.h (libpripps_debye.so). This package is the host
side: form factors, solvent models, the cached model with its recombination
and fitting, trajectory averaging and the serving client.
"""
from .errors import (DeviceError, InternalError, PrippsError, QOutOfRange, UsageError,
                     ValidationError)
from .formfactor import FormFactorMap, linear_q_values, read_formfactors, sinc
from .solvent import ExcludedVolume, Hydration, SolventConfig
from .structure import Structure
from .debye import DebyeModel, Intensity, Contributions, Pripps, combine

__all__ = [
    "DeviceError", "InternalError", "PrippsError", "QOutOfRange", "UsageError",
    "ValidationError", "FormFactorMap", "linear_q_values", "read_formfactors", "sinc",
    "ExcludedVolume", "Hydration", "SolventConfig", "Structure", "DebyeModel", "Intensity",
    "Contributions", "Pripps", "combine",
]
