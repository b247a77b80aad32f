"""libbi_b200: B200-native bootstrap particle-filter step with LibBi's API.

The product is the CUDA shared library (libbi_b200/_lib/libbi_b200.so, C ABI
in include/libbi_b200.h); this package is its host-side mirror of the
reference's filter/resampler classes.
"""
from ._native import (BpfError, ParticleFilterDegeneratedException, load_library,  # noqa: F401
                      LIB_PATH, EXPORTS)
from .filter import (BootstrapPF, ModelL96, ModelPZ, ExternalModel, Resampler, SystematicResampler,  # noqa: F401
                     MultinomialResampler, MetropolisResampler, gather_rows, StepResult, BatchedBootstrapPF,
                     autotune_resampler)
from .sampler import MarginalMH, Prior, smc2  # noqa: F401
from .proposal import LearnedProposal  # noqa: F401
from .schedule import Observer, Schedule, ScheduleElement  # noqa: F401
from .replicas import sharded_batch_filter  # noqa: F401
from . import configs  # noqa: F401

__all__ = ["BootstrapPF", "ModelL96", "ModelPZ", "ExternalModel", "Resampler", "SystematicResampler", "MultinomialResampler",
           "MetropolisResampler", "BatchedBootstrapPF", "MarginalMH", "Prior", "smc2", "LearnedProposal", "Observer", "Schedule",
           "ScheduleElement", "gather_rows", "autotune_resampler", "BpfError", "ParticleFilterDegeneratedException", "configs"]
