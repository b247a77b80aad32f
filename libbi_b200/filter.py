"""Host-side mirror of LibBi's bootstrap particle filter API, over the C ABI.

Names follow the reference's classes so that calling code reads like it:

    reference (share/src/bi/...)                 here
    Model<L96>, Model<PZ> (generated)            ModelL96, ModelPZ
    Resampler<SystematicResampler> etc.          SystematicResampler, MultinomialResampler,
                                                 MetropolisResampler
    Resampler::reduce / ancestors[Permute]       Resampler.reduce / .ancestors / .ancestors_permute
    logsumexp_reduce, gather_rows                Resampler.logsumexp, gather_rows
    BootstrapPF::step / correct / term           BootstrapPF.step / .filter
    Filter<BootstrapPF>::filter                  BootstrapPF.filter
    BootstrapPFState (lws, as, ess, LL)          BootstrapPF.state(), .ess, .log_likelihood

Device memory is passed as torch CUDA tensors (torch is the plumbing for
device memory and streams); all compute runs in the CUDA kernels of the
shared library.  Errors raise BpfError, and a degenerate resample raises
ParticleFilterDegeneratedException as the reference does.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _native as N


# ---------------------------------------------------------------------------
# device views of raw pointers
# ---------------------------------------------------------------------------
class _DeviceArray:
    def __init__(self, ptr: int, shape, typestr: str, strides=None):
        self.__cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
            "version": 3, "strides": strides,
        }


def _view(ptr: int, shape, dtype: str):
    import torch

    typestr = {"f4": "<f4", "f8": "<f8", "i4": "<i4"}[dtype]
    return torch.as_tensor(_DeviceArray(ptr, shape, typestr), device="cuda")


def _ptr_np(a):
    """Host pointer of a contiguous numpy array (or None)."""
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return t.data_ptr()


# ---------------------------------------------------------------------------
# models
# ---------------------------------------------------------------------------
@dataclass
class ModelL96:
    """Lorenz '96 with additive noise: transition(delta) { eta ~ N(0, sigma_eta);
    ode(RK4, h) { dx[i]/dt = (x[i+1]-x[i-2])*x[i-1] - x[i] + F }; x <- x + eta },
    observation { y[i] ~ N(x[i], sigma_y) }, initial { x[i] ~ N(x0_mean, x0_std) }."""

    dim: int = 40
    F: float = 8.0
    sigma_eta: float = 0.1
    sigma_y: float = 1.0
    h: float = 0.01
    x0_mean: Optional[float] = None
    x0_std: float = 0.01
    precision: str = "f32"

    @property
    def nobs(self) -> int:
        return self.dim

    @property
    def np_dtype(self):
        return np.float32 if self.precision == "f32" else np.float64

    def desc(self) -> N.ModelDesc:
        d = N.ModelDesc()
        d.kind = N.BPF_MODEL_L96
        d.dim = self.dim
        d.precision = N.BPF_F32 if self.precision == "f32" else N.BPF_F64
        d.integrator = N.BPF_ODE_RK4
        d.h = self.h
        th = [self.F, self.sigma_eta, self.sigma_y, self.F if self.x0_mean is None else self.x0_mean, self.x0_std]
        for i, v in enumerate(th):
            d.theta[i] = v
        return d


@dataclass
class ModelPZ:
    """Phytoplankton-zooplankton: transition(delta) { alpha ~ log_normal(mu, sigma);
    ode(RK4(3), h0, atoler, rtoler) { dP/dt = alpha P - c P Z; dZ/dt = e c P Z - m Z - q Z^2 } },
    observation { y ~ N(log P, sigma_y) }, initial { P, Z ~ log_normal }."""

    c: float = 0.25
    e: float = 0.3
    m: float = 0.1
    q: float = 0.1
    mu: float = math.log(0.3)
    sigma: float = 0.2
    sigma_y: float = 0.2
    p0_mu: float = math.log(2.0)
    p0_sigma: float = 0.2
    z0_mu: float = math.log(2.0)
    z0_sigma: float = 0.2
    h: float = 0.1
    atoler: float = 1e-3
    rtoler: float = 1e-3
    precision: str = "f64"
    dim: int = 2

    @property
    def nobs(self) -> int:
        return 1

    @property
    def np_dtype(self):
        return np.float64

    def desc(self) -> N.ModelDesc:
        d = N.ModelDesc()
        d.kind = N.BPF_MODEL_PZ
        d.dim = 2
        d.precision = N.BPF_F64
        d.integrator = N.BPF_ODE_RK43
        d.h, d.atoler, d.rtoler = self.h, self.atoler, self.rtoler
        th = [self.c, self.e, self.m, self.q, self.mu, self.sigma, self.sigma_y,
              self.p0_mu, self.p0_sigma, self.z0_mu, self.z0_sigma]
        for i, v in enumerate(th):
            d.theta[i] = v
        return d


class ExternalModel:
    """A model compiled outside the library: a model class in the shape of
    LibBi's generated Model (share/tt/cpp/model.hpp.tt) built with nvcc
    against include/bpf_model.cuh into a shared library that returns its
    bpf_model_ops table from `symbol` (bpf::model_ops<Model>()).  params:
    the model's parameter (P_VAR) values.  BootstrapPF drives it through
    bpf_create_model exactly as it drives the built-in models."""

    def __init__(self, library: str, symbol: str, params: Sequence[float] = (), name: str = ""):
        self._lib = ctypes.CDLL(library)
        f = getattr(self._lib, symbol)
        f.restype = N.ModelOps
        f.argtypes = []
        self.ops = f()
        self.params = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        if self.params.size != self.ops.nparams:
            raise ValueError(f"the model takes {self.ops.nparams} parameters, got {self.params.size}")
        self.name = name or symbol
        self.dim = int(self.ops.dim)
        self.precision = "f32" if self.ops.precision == N.BPF_F32 else "f64"

    @property
    def nobs(self) -> int:
        return int(self.ops.nobs)

    @property
    def np_dtype(self):
        return np.float32 if self.precision == "f32" else np.float64


# ---------------------------------------------------------------------------
# resamplers
# ---------------------------------------------------------------------------
class Resampler:
    """Resampler<R> (share/src/bi/resampler/Resampler.hpp:33-117) on device
    log-weights (FP64 torch CUDA tensors)."""

    kind = N.BPF_RESAMPLER_SYSTEMATIC

    def __init__(self, ess_rel: float = 0.5, max_n: int = 1 << 20, B: int = 0, stream=None):
        if not (0.0 <= ess_rel <= 1.0):
            raise ValueError("essRel must lie in [0, 1]")
        self.ess_rel = ess_rel
        self.B = B
        self.max_n = max_n
        self._h = ctypes.c_void_p()
        N.check(N.lib().bpf_resampler_create(self.kind, max_n, B, stream, ctypes.byref(self._h)),
                "bpf_resampler_create")

    def close(self):
        if self._h:
            N.load_library().bpf_resampler_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_shape(self, shape: int = -1):
        """Pin the tile shape of the one-launch systematic kernel (0..5; -1:
        the autotuned shape).  Every shape computes the same ancestors."""
        N.check(N.lib().bpf_resampler_set_shape(self._h, int(shape)), "bpf_resampler_set_shape")

    def timing(self, enable: bool = True):
        """Record CUDA events around the kernels of every later call."""
        N.check(N.lib().bpf_resampler_timing_enable(self._h, int(enable)), "bpf_resampler_timing_enable")

    def timing_read(self, reset: bool = True):
        """(summed kernel milliseconds, timed calls) since the last reset."""
        ms, calls = ctypes.c_double(), ctypes.c_int()
        N.check(N.lib().bpf_resampler_timing_read(self._h, int(reset), ctypes.byref(ms), ctypes.byref(calls)),
                "bpf_resampler_timing_read")
        return ms.value, calls.value

    def reduce(self, lws):
        """ESS and lW = log mean exp(lws): Resampler::reduce -> ess_reduce."""
        lW, ess = ctypes.c_double(), ctypes.c_double()
        N.check(N.lib().bpf_ess_reduce(self._h, _ptr(lws), lws.numel(), ctypes.byref(lW), ctypes.byref(ess)),
                "bpf_ess_reduce")
        return ess.value, lW.value

    def logsumexp(self, lws) -> float:
        out = ctypes.c_double()
        N.check(N.lib().bpf_logsumexp_reduce(self._h, _ptr(lws), lws.numel(), ctypes.byref(out)),
                "bpf_logsumexp_reduce")
        return out.value

    def ancestors(self, lws, uniforms=None, permute: bool = False, with_offspring: bool = False):
        import torch

        n = lws.numel()
        a = torch.empty(n, dtype=torch.int32, device=lws.device)
        Os = torch.empty(n, dtype=torch.int32, device=lws.device) if with_offspring else None
        N.check(N.lib().bpf_resampler_ancestors(self._h, _ptr(lws), n, _ptr(uniforms), int(permute), _ptr(a),
                                                _ptr(Os)), "bpf_resampler_ancestors")
        return (a, Os) if with_offspring else a

    def ancestors_permute(self, lws, uniforms=None):
        return self.ancestors(lws, uniforms, permute=True)


class SystematicResampler(Resampler):
    kind = N.BPF_RESAMPLER_SYSTEMATIC


class MultinomialResampler(Resampler):
    kind = N.BPF_RESAMPLER_MULTINOMIAL


class MetropolisResampler(Resampler):
    kind = N.BPF_RESAMPLER_METROPOLIS


RESAMPLERS = {"systematic": N.BPF_RESAMPLER_SYSTEMATIC, "multinomial": N.BPF_RESAMPLER_MULTINOMIAL,
              "metropolis": N.BPF_RESAMPLER_METROPOLIS}


def gather_rows(as_, X, Y, d: int, ld: int, stream=None):
    """Y[j*ld + i] = X[j*ld + as[i]] (gather_rows, out of place)."""
    n = as_.numel()
    N.check(N.lib().bpf_gather_rows(_ptr(as_), _ptr(X), _ptr(Y), n, d, ld, X.element_size(), stream),
            "bpf_gather_rows")


# ---------------------------------------------------------------------------
# filter
# ---------------------------------------------------------------------------
@dataclass
class StepResult:
    ess: float
    log_weight_sum: float
    log_increment: float
    log_likelihood: float
    resampled: bool


# (threads per block, particles per thread) of the one-launch kernel
RESAMPLE_SHAPES = ((256, 2), (128, 4), (512, 1), (512, 2), (256, 4), (1024, 1))


def shape_name(shape) -> str:
    """'256x2' for (256, 2)."""
    return f"{shape[0]}x{shape[1]}"


def autotune_resampler(n: int, stream=None):
    """Time every tile shape (threads per block, particles per thread) of
    the one-launch systematic resampler on n synthetic log-weights and keep
    the fastest for n's size class; returns (shape index, {shape: us})."""
    r = N.TuneResult()
    N.check(N.lib().bpf_autotune_resampler(int(n), stream, ctypes.byref(r)), "bpf_autotune_resampler")
    return r.shape, {RESAMPLE_SHAPES[k]: r.us[k] for k in range(N.RESAMPLE_SHAPES) if r.us[k] > 0}


class BootstrapPF:
    """BootstrapPF<B,F,O,R> + BootstrapPFState for one model on one GPU."""

    def __init__(self, model, nparticles: int, resampler: str = "systematic", ess_rel: float = 0.5,
                 seed: int = 0, metropolis_steps: int = 0, stream=None):
        self.model = model
        self.n = nparticles
        cfg = N.Config()
        cfg.nparticles = nparticles
        cfg.resampler = RESAMPLERS[resampler]
        cfg.metropolis_steps = metropolis_steps
        cfg.ess_rel = ess_rel
        cfg.seed = seed
        cfg.stream = stream
        self._cfg = cfg
        self._h = ctypes.c_void_p()
        if isinstance(model, ExternalModel):
            self._desc = None
            N.check(N.lib().bpf_create_model(ctypes.byref(model.ops), _ptr_np(model.params) if model.params.size
                                             else None, ctypes.byref(cfg), ctypes.byref(self._h)),
                    "bpf_create_model")
        else:
            self._desc = model.desc()
            N.check(N.lib().bpf_create(ctypes.byref(self._desc), ctypes.byref(cfg), ctypes.byref(self._h)),
                    "bpf_create")

    def close(self):
        if self._h:
            N.load_library().bpf_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def init(self):
        N.check(N.lib().bpf_init(self._h), "bpf_init")

    def _y_host(self, y):
        if y is None:
            return None, None
        arr = np.ascontiguousarray(np.asarray(y, dtype=self.model.np_dtype).reshape(-1))
        if arr.size != self.model.nobs:
            raise ValueError(f"expected {self.model.nobs} observations")
        return arr, arr.ctypes.data_as(ctypes.c_void_p)

    def step(self, t1: float, t2: float, y=None) -> StepResult:
        """One BootstrapPF::step to the observation y at t2 (host values)."""
        arr, p = self._y_host(y)
        out = N.StepOut()
        N.check(N.lib().bpf_step(self._h, t1, t2, p, ctypes.byref(out)), "bpf_step")
        return StepResult(out.ess, out.log_weight_sum, out.log_increment, out.log_likelihood, bool(out.resampled))

    def step_sparse(self, t1: float, t2: float, y, idx) -> StepResult:
        """BootstrapPF::step to an observation of the components idx only."""
        vals = np.ascontiguousarray(np.asarray(y, dtype=self.model.np_dtype).reshape(-1))
        ix = np.ascontiguousarray(np.asarray(idx, dtype=np.int32).reshape(-1))
        if vals.size != ix.size:
            raise ValueError("one value per observed component")
        out = N.StepOut()
        N.check(N.lib().bpf_step_sparse(self._h, t1, t2, vals.ctypes.data_as(ctypes.c_void_p),
                                        ix.ctypes.data_as(ctypes.c_void_p), ix.size, ctypes.byref(out)),
                "bpf_step_sparse")
        return StepResult(out.ess, out.log_weight_sum, out.log_increment, out.log_likelihood, bool(out.resampled))

    def step_device(self, t1: float, t2: float, y_dev=None, sync: bool = True) -> Optional[StepResult]:
        """BootstrapPF::step with the observation already on the device."""
        if not sync:
            N.check(N.lib().bpf_step_device(self._h, t1, t2, _ptr(y_dev), None), "bpf_step_device")
            return None
        out = N.StepOut()
        N.check(N.lib().bpf_step_device(self._h, t1, t2, _ptr(y_dev), ctypes.byref(out)), "bpf_step_device")
        return StepResult(out.ess, out.log_weight_sum, out.log_increment, out.log_likelihood, bool(out.resampled))

    def filter(self, y, t0: float = 0.0, dt: float = 1.0):
        """Filter<BootstrapPF>::filter over T observations; returns
        (logLikelihood, logIncrements[T], ess[T])."""
        arr = np.ascontiguousarray(np.asarray(y, dtype=self.model.np_dtype).reshape(-1))
        T = arr.size // self.model.nobs
        inc = np.zeros(T)
        ess = np.zeros(T)
        ll = ctypes.c_double()
        N.check(N.lib().bpf_filter(self._h, T, t0, dt, arr.ctypes.data_as(ctypes.c_void_p),
                                   inc.ctypes.data_as(ctypes.c_void_p), ess.ctypes.data_as(ctypes.c_void_p),
                                   ctypes.byref(ll)), "bpf_filter")
        return ll.value, inc, ess

    def path_cache(self, max_steps: int):
        """Record states and ancestors of up to max_steps steps (0: stop)."""
        N.check(N.lib().bpf_path_cache(self._h, max_steps), "bpf_path_cache")
        self._path_steps = max_steps

    def path_nodes(self):
        """(nodes held, pool capacity) of the pruned path record."""
        nodes, cap = ctypes.c_int(), ctypes.c_int()
        N.check(N.lib().bpf_path_cache_nodes(self._h, ctypes.byref(nodes), ctypes.byref(cap)), "bpf_path_cache_nodes")
        return nodes.value, cap.value

    def sample_path(self, u=None):
        """BootstrapPF::samplePath: (particle, path[len, dim]) with the path of
        a particle drawn from the current weights (u: device tensor with one
        uniform, or None for the handle's own draw)."""
        cap = getattr(self, "_path_steps", 0)
        buf = np.zeros((cap + 1, self.model.dim), dtype=self.model.np_dtype)
        p, n = ctypes.c_int(), ctypes.c_int()
        N.check(N.lib().bpf_sample_path(self._h, _ptr(u), buf.ctypes.data_as(ctypes.c_void_p), ctypes.byref(p),
                                        ctypes.byref(n)), "bpf_sample_path")
        return p.value, buf[:n.value]

    def set_proposal(self, proposal):
        """Attach a LearnedProposal (or None to detach): observed steps then
        propose from it and correct the weights by importance sampling."""
        N.check(N.lib().bpf_set_proposal(self._h, None if proposal is None else proposal.handle), "bpf_set_proposal")
        self._proposal = proposal

    def set_step_form(self, fused: bool):
        """One launch per step with the resampling as the transition's
        prologue (fused), or the resampler and the transition as two
        launches (the default); both give the same numbers bit for bit."""
        N.check(N.lib().bpf_set_step_form(self._h, int(bool(fused))), "bpf_set_step_form")

    @property
    def step_form_fused(self) -> bool:
        v = ctypes.c_int()
        N.check(N.lib().bpf_step_form(self._h, ctypes.byref(v)), "bpf_step_form")
        return bool(v.value)

    def reduce(self):
        lW, ess = ctypes.c_double(), ctypes.c_double()
        N.check(N.lib().bpf_reduce(self._h, ctypes.byref(lW), ctypes.byref(ess)), "bpf_reduce")
        return ess.value, lW.value

    def resample(self, uniforms=None):
        import torch

        out = torch.empty(self.n, dtype=torch.int32, device="cuda")
        N.check(N.lib().bpf_resample(self._h, _ptr(uniforms), _ptr(out)), "bpf_resample")
        return out

    def state(self):
        """Device views (x[dim, ld], lws[n], as[n]) of the particle store."""
        x, lw, as_, ld = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int()
        N.check(N.lib().bpf_state_ptrs(self._h, ctypes.byref(x), ctypes.byref(lw), ctypes.byref(as_),
                                       ctypes.byref(ld)), "bpf_state_ptrs")
        dt = "f4" if self.model.precision == "f32" else "f8"
        return (_view(x.value, (self.model.dim, ld.value), dt), _view(lw.value, (self.n,), "f8"),
                _view(as_.value, (self.n,), "i4"))

    def timing(self, enable: bool = True):
        N.check(N.lib().bpf_timing_enable(self._h, int(enable)), "bpf_timing_enable")

    def timing_read(self, reset: bool = True):
        """(resample_ms, transition_ms, steps) summed since the last reset."""
        r, t, k = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        N.check(N.lib().bpf_timing_read(self._h, int(reset), ctypes.byref(r), ctypes.byref(t), ctypes.byref(k)),
                "bpf_timing_read")
        return r.value, t.value, k.value

    def snapshot(self) -> bytes:
        size = ctypes.c_uint64()
        N.check(N.lib().bpf_snapshot_size(self._h, ctypes.byref(size)), "bpf_snapshot_size")
        buf = ctypes.create_string_buffer(size.value)
        N.check(N.lib().bpf_snapshot(self._h, buf, size.value), "bpf_snapshot")
        return buf.raw

    def restore(self, blob: bytes):
        buf = ctypes.create_string_buffer(blob, len(blob))
        N.check(N.lib().bpf_restore(self._h, buf, len(blob)), "bpf_restore")


# ---------------------------------------------------------------------------
# batched filters
# ---------------------------------------------------------------------------
class BatchedBootstrapPF:
    """Many independent BootstrapPF filters of one model kind advanced together
    (bpf_batch_*).  models[f] gives filter f's constants (all of one kind,
    dimension, precision and integrator settings); nparticles, resamplers,
    seeds and metropolis_steps are per filter (scalars broadcast)."""

    def __init__(self, models, nparticles, resamplers="systematic", seeds=0, ess_rel: float = 0.5,
                 metropolis_steps=0, stream=None):
        models = list(models)
        F = len(models)
        bc = lambda v: list(v) if isinstance(v, (list, tuple, np.ndarray)) else [v] * F  # noqa: E731
        nparticles, resamplers, seeds, msteps = bc(nparticles), bc(resamplers), bc(seeds), bc(metropolis_steps)
        if not (len(nparticles) == len(resamplers) == len(seeds) == len(msteps) == F):
            raise ValueError("per-filter settings must have one entry per model")
        self.model = models[0]
        self.models = models
        self.nf = F
        self.n = [int(v) for v in nparticles]
        self._desc = self.model.desc()
        arr = (N.BatchFilter * F)()
        for f, m in enumerate(models):
            d = m.desc()
            if (d.kind, d.dim, d.precision, d.integrator) != (self._desc.kind, self._desc.dim, self._desc.precision,
                                                              self._desc.integrator):
                raise ValueError("all filters of a batch share the model kind, dimension and precision")
            arr[f].nparticles = int(nparticles[f])
            arr[f].resampler = RESAMPLERS[resamplers[f]] if isinstance(resamplers[f], str) else int(resamplers[f])
            arr[f].metropolis_steps = int(msteps[f])
            arr[f].seed = int(seeds[f])
            for i in range(N.BPF_MAX_THETA):
                arr[f].theta[i] = d.theta[i]
        self._filters = arr
        self._h = ctypes.c_void_p()
        N.check(N.lib().bpf_batch_create(ctypes.byref(self._desc), F, arr, ess_rel, stream, ctypes.byref(self._h)),
                "bpf_batch_create")

    def close(self):
        if self._h:
            N.load_library().bpf_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self):
        N.check(N.lib().bpf_batch_init(self._h), "bpf_batch_init")

    def set_theta(self, theta):
        """theta: (nfilters, k <= BPF_MAX_THETA) model constants per filter."""
        t = np.zeros((self.nf, N.BPF_MAX_THETA))
        th = np.asarray(theta, dtype=np.float64)
        t[:, :th.shape[1]] = th
        N.check(N.lib().bpf_batch_set_theta(self._h, t.ctypes.data_as(ctypes.c_void_p)), "bpf_batch_set_theta")

    def step_device(self, t1: float, t2: float, y_dev=None):
        """One step of every filter; y_dev: (nfilters, nobs) device tensor or None."""
        N.check(N.lib().bpf_batch_step_device(self._h, t1, t2, _ptr(y_dev)), "bpf_batch_step_device")

    def timing(self, enable: bool = True):
        N.check(N.lib().bpf_batch_timing_enable(self._h, int(enable)), "bpf_batch_timing_enable")

    def timing_read(self, reset: bool = True):
        """(device milliseconds, steps) timed since the last reset."""
        ms, k = ctypes.c_double(), ctypes.c_int()
        N.check(N.lib().bpf_batch_timing_read(self._h, int(reset), ctypes.byref(ms), ctypes.byref(k)),
                "bpf_batch_timing_read")
        return ms.value, k.value

    def stats(self):
        """(logLikelihood[F], ess[F], status[F]) on the host; no exception for
        degenerate filters (their logLikelihood is -inf)."""
        ll, ess, st = np.zeros(self.nf), np.zeros(self.nf), np.zeros(self.nf, np.int32)
        N.lib().bpf_batch_stats(self._h, ll.ctypes.data_as(ctypes.c_void_p), ess.ctypes.data_as(ctypes.c_void_p),
                                st.ctypes.data_as(ctypes.c_void_p))
        return ll, ess, st

    def resample_threads(self, threads: int = 0):
        """Threads per filter CTA of the resampler: pin 256, 512 or 1024, or
        0 to keep the autotuned count; returns (current, {count: tuning us})."""
        cur = ctypes.c_int()
        us = np.zeros(3)
        N.check(N.lib().bpf_batch_resample_threads(self._h, int(threads), ctypes.byref(cur),
                                                   us.ctypes.data_as(ctypes.c_void_p)), "bpf_batch_resample_threads")
        return cur.value, {256: us[0], 512: us[1], 1024: us[2]}

    def set_proposal(self, proposal):
        """Attach a LearnedProposal to every filter (or None to detach):
        observed steps then run the guided step for the whole batch."""
        N.check(N.lib().bpf_batch_set_proposal(self._h, None if proposal is None else proposal.handle),
                "bpf_batch_set_proposal")
        self._proposal = proposal

    def filter(self, y, t0: float = 0.0, dt: float = 1.0):
        """Filter<BootstrapPF>::filter for every filter; y: (T, nfilters,
        nobs) host observations.  Returns (logLikelihood[F],
        logIncrements[T, F], ess[T, F], status[F])."""
        arr = np.ascontiguousarray(np.asarray(y, dtype=self.model.np_dtype))
        T = arr.size // (self.nf * self.model.nobs)
        if arr.size != T * self.nf * self.model.nobs:
            raise ValueError("y must hold T x nfilters x nobs values")
        ll, st = np.zeros(self.nf), np.zeros(self.nf, np.int32)
        inc, ess = np.zeros((T, self.nf)), np.zeros((T, self.nf))
        rc = N.lib().bpf_filter_batch(self._h, T, t0, dt, arr.ctypes.data_as(ctypes.c_void_p),
                                      ll.ctypes.data_as(ctypes.c_void_p), inc.ctypes.data_as(ctypes.c_void_p),
                                      ess.ctypes.data_as(ctypes.c_void_p), st.ctypes.data_as(ctypes.c_void_p))
        if rc not in (N.BPF_OK, N.BPF_E_DEGENERATE):
            N.check(rc, "bpf_filter_batch")
        return ll, inc, ess, st

    def state(self):
        """Device views (x[dim, ld], lws[ld], as[ld]) and per-filter offsets."""
        x, lw, as_, ld = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int()
        offs = np.zeros(self.nf, np.int32)
        N.check(N.lib().bpf_batch_state_ptrs(self._h, ctypes.byref(x), ctypes.byref(lw), ctypes.byref(as_),
                                             ctypes.byref(ld), offs.ctypes.data_as(ctypes.c_void_p)),
                "bpf_batch_state_ptrs")
        dt = "f4" if self.model.precision == "f32" else "f8"
        return (_view(x.value, (self.model.dim, ld.value), dt), _view(lw.value, (ld.value,), "f8"),
                _view(as_.value, (ld.value,), "i4"), offs)
