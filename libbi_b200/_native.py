"""ctypes binding of the libbi_b200 C ABI (include/libbi_b200.h).

The shared library is built in-tree (``libbi_b200/_lib/libbi_b200.so``) by
``libbi_b200.build``.  There is no fallback: if the library is missing or a
CUDA device is not available, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_longlong, POINTER, c_double, c_int, c_uint64, c_void_p, c_char_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libbi_b200.so")

BPF_OK = 0
BPF_E_DEGENERATE = 1
BPF_E_INVALID = 2
BPF_E_CUDA = 3
BPF_E_TIMEOUT = 4
BPF_E_NOMEM = 5
BPF_E_TOO_LARGE = 6
BPF_STATIC_MAX_PARTICLES = 65536
BPF_BATCH_MAX_PARTICLES = 32768
BPF_WAIT_LIMIT_DEFAULT = 4000000000

BPF_MODEL_L96 = 1
BPF_MODEL_PZ = 2
BPF_ODE_RK4 = 0
BPF_ODE_RK43 = 1
BPF_F32 = 0
BPF_F64 = 1
BPF_RESAMPLER_SYSTEMATIC = 0
BPF_RESAMPLER_MULTINOMIAL = 1
BPF_RESAMPLER_METROPOLIS = 2
BPF_MAX_THETA = 16

# every symbol include/libbi_b200.h declares
EXPORTS = (
    "bpf_create", "bpf_destroy", "bpf_state_ptrs", "bpf_init", "bpf_step",
    "bpf_step_device", "bpf_filter", "bpf_reduce", "bpf_resample",
    "bpf_resampler_create", "bpf_resampler_destroy", "bpf_ess_reduce",
    "bpf_logsumexp_reduce", "bpf_resampler_ancestors", "bpf_gather_rows",
    "bpf_snapshot_size", "bpf_snapshot", "bpf_restore", "bpf_version",
    "bpf_status_string", "bpf_timing_enable", "bpf_timing_read", "bpf_systematic_ancestors_static",
    "bpf_resampler_timing_enable", "bpf_resampler_timing_read", "bpf_autotune_resampler", "bpf_resampler_set_shape",
    "bpf_batch_create", "bpf_batch_destroy", "bpf_batch_init", "bpf_batch_set_theta", "bpf_batch_step_device",
    "bpf_batch_stats", "bpf_batch_state_ptrs", "bpf_filter_batch", "bpf_batch_timing_enable",
    "bpf_batch_timing_read", "bpf_batch_set_seeds", "bpf_batch_resample_threads",
    "bpf_pmmh_create", "bpf_pmmh_destroy", "bpf_pmmh_run", "bpf_pmmh_state", "bpf_dense_bf16",
    "bpf_proposal_create", "bpf_proposal_destroy", "bpf_proposal_set_data", "bpf_proposal_train",
    "bpf_proposal_loss_grad", "bpf_proposal_params", "bpf_proposal_set_params", "bpf_set_proposal",
    "bpf_batch_set_proposal",
    "bpf_path_cache", "bpf_sample_path", "bpf_step_sparse", "bpf_smc2_run", "bpf_debug_set_wait_limit", "bpf_create_model", "bpf_path_cache_nodes", "bpf_proposal_set_states",
    "bpf_pmmh_set_proposal", "bpf_set_step_form", "bpf_step_form",
)


class ModelDesc(ctypes.Structure):
    _fields_ = [
        ("kind", c_int), ("dim", c_int), ("precision", c_int), ("integrator", c_int),
        ("h", c_double), ("atoler", c_double), ("rtoler", c_double),
        ("theta", c_double * BPF_MAX_THETA),
    ]


class Config(ctypes.Structure):
    _fields_ = [
        ("nparticles", c_int), ("resampler", c_int), ("metropolis_steps", c_int),
        ("ess_rel", c_double), ("seed", c_uint64), ("stream", c_void_p),
    ]


class BatchFilter(ctypes.Structure):
    _fields_ = [
        ("nparticles", c_int), ("resampler", c_int), ("metropolis_steps", c_int), ("seed", c_uint64),
        ("theta", c_double * BPF_MAX_THETA),
    ]


BPF_PRIOR_UNIFORM, BPF_PRIOR_LOG_NORMAL, BPF_PRIOR_GAUSSIAN = 0, 1, 2


class PmmhParam(ctypes.Structure):
    _fields_ = [("index", c_int), ("prior", c_int), ("a", c_double), ("b", c_double), ("step", c_double)]


class PmmhConfig(ctypes.Structure):
    _fields_ = [
        ("nchains", c_int), ("nparticles", c_int), ("resampler", c_int), ("metropolis_steps", c_int),
        ("ess_rel", c_double), ("seed", c_uint64), ("nparams", c_int), ("params", PmmhParam * BPF_MAX_THETA),
        ("chain_nparticles", c_void_p),
    ]


class Smc2Config(ctypes.Structure):
    _fields_ = [
        ("ntheta", c_int), ("nparticles", c_int), ("resampler", c_int), ("metropolis_steps", c_int),
        ("ess_rel", c_double), ("theta_ess_rel", c_double), ("moves", c_int), ("seed", c_uint64),
        ("nparams", c_int), ("params", PmmhParam * BPF_MAX_THETA),
    ]


RESAMPLE_SHAPES = 6  # BPF_RESAMPLE_SHAPES


class TuneResult(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int), ("us", ctypes.c_double * RESAMPLE_SHAPES)]


class ModelOps(ctypes.Structure):
    """bpf_model_ops: the launchers of a model compiled outside the library."""
    _fields_ = [
        ("dim", c_int), ("nobs", c_int), ("nparams", c_int), ("precision", c_int),
        ("init", c_void_p), ("transition", c_void_p),
    ]


class StepOut(ctypes.Structure):
    _fields_ = [
        ("ess", c_double), ("log_weight_sum", c_double), ("log_increment", c_double),
        ("log_likelihood", c_double), ("resampled", c_int), ("status", c_int),
    ]


class BpfError(RuntimeError):
    """A libbi_b200 call returned a non-zero status."""

    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} (status {status})")


class ParticleFilterDegeneratedException(BpfError):
    """All weights zero or not finite when a resample was due; the name and
    meaning of share/src/bi/misc/exception.hpp:47."""


_lib = None


def _declare(L):
    H = c_void_p
    sig = {
        "bpf_create": (c_int, [POINTER(ModelDesc), POINTER(Config), POINTER(H)]),
        "bpf_destroy": (c_int, [H]),
        "bpf_state_ptrs": (c_int, [H, POINTER(c_void_p), POINTER(c_void_p), POINTER(c_void_p), POINTER(c_int)]),
        "bpf_init": (c_int, [H]),
        "bpf_step": (c_int, [H, c_double, c_double, c_void_p, POINTER(StepOut)]),
        "bpf_step_device": (c_int, [H, c_double, c_double, c_void_p, POINTER(StepOut)]),
        "bpf_filter": (c_int, [H, c_int, c_double, c_double, c_void_p, c_void_p, c_void_p, POINTER(c_double)]),
        "bpf_reduce": (c_int, [H, POINTER(c_double), POINTER(c_double)]),
        "bpf_resample": (c_int, [H, c_void_p, c_void_p]),
        "bpf_resampler_create": (c_int, [c_int, c_int, c_int, c_void_p, POINTER(H)]),
        "bpf_resampler_destroy": (c_int, [H]),
        "bpf_ess_reduce": (c_int, [H, c_void_p, c_int, POINTER(c_double), POINTER(c_double)]),
        "bpf_logsumexp_reduce": (c_int, [H, c_void_p, c_int, POINTER(c_double)]),
        "bpf_resampler_ancestors": (c_int, [H, c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p]),
        "bpf_gather_rows": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p]),
        "bpf_snapshot_size": (c_int, [H, POINTER(c_uint64)]),
        "bpf_snapshot": (c_int, [H, c_void_p, c_uint64]),
        "bpf_restore": (c_int, [H, c_void_p, c_uint64]),
        "bpf_timing_enable": (c_int, [H, c_int]),
        "bpf_timing_read": (c_int, [H, c_int, POINTER(c_double), POINTER(c_double), POINTER(c_int)]),
        "bpf_batch_create": (c_int, [POINTER(ModelDesc), c_int, POINTER(BatchFilter), c_double, c_void_p,
                                     POINTER(H)]),
        "bpf_batch_destroy": (c_int, [H]),
        "bpf_batch_init": (c_int, [H]),
        "bpf_batch_set_theta": (c_int, [H, c_void_p]),
        "bpf_batch_step_device": (c_int, [H, c_double, c_double, c_void_p]),
        "bpf_batch_stats": (c_int, [H, c_void_p, c_void_p, c_void_p]),
        "bpf_batch_state_ptrs": (c_int, [H, POINTER(c_void_p), POINTER(c_void_p), POINTER(c_void_p), POINTER(c_int),
                                         c_void_p]),
        "bpf_filter_batch": (c_int, [H, c_int, c_double, c_double, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p]),
        "bpf_batch_timing_enable": (c_int, [H, c_int]),
        "bpf_batch_set_seeds": (c_int, [H, c_void_p]),
        "bpf_batch_resample_threads": (c_int, [H, c_int, POINTER(c_int), c_void_p]),
        "bpf_pmmh_create": (c_int, [POINTER(ModelDesc), POINTER(PmmhConfig), c_int, c_double, c_double, c_void_p,
                                    c_void_p, c_void_p, POINTER(H)]),
        "bpf_pmmh_destroy": (c_int, [H]),
        "bpf_proposal_create": (c_int, [POINTER(ModelDesc), c_double, c_int, c_uint64, c_void_p, POINTER(H)]),
        "bpf_proposal_destroy": (c_int, [H]),
        "bpf_proposal_set_data": (c_int, [H, c_void_p, c_void_p, c_void_p, c_int]),
        "bpf_proposal_set_states": (c_int, [H, c_void_p, c_int]),
        "bpf_pmmh_set_proposal": (c_int, [H, H]),
        "bpf_set_step_form": (c_int, [H, c_int]),
        "bpf_step_form": (c_int, [H, POINTER(c_int)]),
        "bpf_proposal_train": (c_int, [H, c_int, c_int, c_double, c_void_p]),
        "bpf_proposal_loss_grad": (c_int, [H, c_void_p, c_void_p, c_int, POINTER(c_double), c_void_p]),
        "bpf_proposal_params": (c_int, [H, c_void_p, c_void_p, c_void_p, POINTER(c_int)]),
        "bpf_proposal_set_params": (c_int, [H, c_void_p, c_void_p, c_void_p]),
        "bpf_set_proposal": (c_int, [H, H]),
        "bpf_batch_set_proposal": (c_int, [H, H]),
        "bpf_path_cache": (c_int, [H, c_int]),
        "bpf_path_cache_nodes": (c_int, [H, POINTER(c_int), POINTER(c_int)]),
        "bpf_smc2_run": (c_int, [POINTER(ModelDesc), POINTER(Smc2Config), c_int, c_double, c_double, c_void_p,
                                 c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_int), POINTER(c_double)]),
        "bpf_step_sparse": (c_int, [H, c_double, c_double, c_void_p, c_void_p, c_int, POINTER(StepOut)]),
        "bpf_sample_path": (c_int, [H, c_void_p, c_void_p, POINTER(c_int), POINTER(c_int)]),
        "bpf_dense_bf16": (c_int, [c_void_p, c_longlong, c_longlong, c_void_p, c_longlong, c_longlong, c_int, c_int,
                                   c_int, c_void_p, c_int, c_void_p, c_longlong, c_void_p, c_longlong, c_void_p,
                                   c_void_p]),
        "bpf_pmmh_run": (c_int, [H, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
        "bpf_pmmh_state": (c_int, [H, c_void_p, c_void_p, c_void_p, POINTER(c_int)]),
        "bpf_batch_timing_read": (c_int, [H, c_int, POINTER(c_double), POINTER(c_int)]),
        "bpf_resampler_timing_enable": (c_int, [H, c_int]),
        "bpf_resampler_timing_read": (c_int, [H, c_int, POINTER(c_double), POINTER(c_int)]),
        "bpf_autotune_resampler": (c_int, [c_int, c_void_p, POINTER(TuneResult)]),
        "bpf_resampler_set_shape": (c_int, [H, c_int]),
        "bpf_systematic_ancestors_static": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p,
                                                    c_void_p]),
        "bpf_debug_set_wait_limit": (c_int, [c_longlong]),
        "bpf_create_model": (c_int, [POINTER(ModelOps), c_void_p, POINTER(Config), POINTER(H)]),
        "bpf_version": (c_char_p, []),
        "bpf_status_string": (c_char_p, [c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


def load_library(path: str = LIB_PATH):
    """Load the shared library without touching the GPU (CPU-safe)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"libbi_b200 shared library not built: {path} (run libbi_b200.build.build())")
        _lib = _declare(ctypes.CDLL(path))
    return _lib


def lib():
    """The loaded library, for compute calls: requires a CUDA device."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("libbi_b200 needs a CUDA device; there is no CPU fallback")
    return load_library()


def status_string(status: int) -> str:
    try:
        return load_library().bpf_status_string(status).decode()
    except OSError:
        return "library not loaded"


def check(status: int, what: str) -> None:
    if status == BPF_OK:
        return
    if status == BPF_E_DEGENERATE:
        raise ParticleFilterDegeneratedException(status, what)
    raise BpfError(status, what)
