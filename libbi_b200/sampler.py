"""Samplers over the batched filter: MarginalMH (particle-marginal
Metropolis-Hastings, share/src/bi/sampler/MarginalMH.hpp) for many chains
at once.  Host-side mirror of bpf_pmmh_* (include/libbi_b200.h)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .filter import RESAMPLERS, _ptr_np


@dataclass
class Prior:
    """Prior of one sampled parameter: kind "uniform" (a, b = bounds),
    "log_normal" or "gaussian" (a, b = mu, sigma); step is the standard
    deviation of its random-walk proposal; index its position in theta."""

    index: int
    kind: str
    a: float
    b: float
    step: float


_KINDS = {"uniform": N.BPF_PRIOR_UNIFORM, "log_normal": N.BPF_PRIOR_LOG_NORMAL, "gaussian": N.BPF_PRIOR_GAUSSIAN}


class MarginalMH:
    """C chains of particle-marginal Metropolis-Hastings, each iteration one
    batched filter run over all chains' proposals."""

    def __init__(self, model, priors, y, t0: float = 0.0, dt: float = 1.0, nchains: int = 128,
                 nparticles: int = 1024, resampler: str = "systematic", ess_rel: float = 1.0, seed: int = 0,
                 theta0=None, metropolis_steps: int = 0, stream=None):
        self.model = model
        self.priors = list(priors)
        self.nchains = nchains
        self.nparams = len(self.priors)
        cfg = N.PmmhConfig()
        # nparticles: one count for every chain, or one per chain
        counts = np.atleast_1d(np.asarray(nparticles, dtype=np.int32))
        if counts.size not in (1, nchains):
            raise ValueError("nparticles: one value, or one per chain")
        self.nparticles = counts if counts.size == nchains else np.full(nchains, int(counts[0]), np.int32)
        self._counts = np.ascontiguousarray(self.nparticles, dtype=np.int32)
        cfg.nchains, cfg.nparticles = nchains, int(self.nparticles.max())
        cfg.chain_nparticles = self._counts.ctypes.data_as(ctypes.c_void_p).value
        cfg.resampler, cfg.metropolis_steps = RESAMPLERS[resampler], metropolis_steps
        cfg.ess_rel, cfg.seed, cfg.nparams = ess_rel, seed, self.nparams
        for j, q in enumerate(self.priors):
            cfg.params[j].index, cfg.params[j].prior = q.index, _KINDS[q.kind]
            cfg.params[j].a, cfg.params[j].b, cfg.params[j].step = q.a, q.b, q.step
        self._cfg = cfg
        self._desc = model.desc()
        yy = np.ascontiguousarray(np.asarray(y, dtype=model.np_dtype))
        self.T = yy.size // model.nobs
        th0 = None if theta0 is None else np.ascontiguousarray(np.asarray(theta0, np.float64).reshape(nchains, -1))
        self._h = ctypes.c_void_p()
        N.check(N.lib().bpf_pmmh_create(ctypes.byref(self._desc), ctypes.byref(cfg), self.T, t0, dt, _ptr_np(yy),
                                        _ptr_np(th0), stream, ctypes.byref(self._h)), "bpf_pmmh_create")

    def close(self):
        if self._h:
            N.load_library().bpf_pmmh_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_proposal(self, proposal):
        """Filter later iterations with the learned proposal (a
        LearnedProposal of the same model; None: the bootstrap filter)."""
        N.check(N.lib().bpf_pmmh_set_proposal(self._h, None if proposal is None else proposal.handle),
                "bpf_pmmh_set_proposal")
        self._proposal = proposal

    def run(self, iterations: int):
        """Returns dict(samples[it, C, P], loglik[it, C], logprior[it, C],
        proposal_loglik[it, C], accepted[C])."""
        C, P = self.nchains, self.nparams
        smp = np.zeros((iterations, C, P))
        ll, lp, pll = np.zeros((iterations, C)), np.zeros((iterations, C)), np.zeros((iterations, C))
        acc = np.zeros(C, np.int32)
        N.check(N.lib().bpf_pmmh_run(self._h, iterations, _ptr_np(smp), _ptr_np(ll), _ptr_np(lp), _ptr_np(pll),
                                     _ptr_np(acc)), "bpf_pmmh_run")
        return dict(samples=smp, loglik=ll, logprior=lp, proposal_loglik=pll, accepted=acc)

    def state(self):
        """(theta[C, P], loglik[C], logprior[C], filter runs so far)."""
        C, P = self.nchains, self.nparams
        th, ll, lp = np.zeros((C, P)), np.zeros(C), np.zeros(C)
        runs = ctypes.c_int()
        N.check(N.lib().bpf_pmmh_state(self._h, _ptr_np(th), _ptr_np(ll), _ptr_np(lp), ctypes.byref(runs)),
                "bpf_pmmh_state")
        return th, ll, lp, runs.value


def smc2(model, priors, y, t0: float = 0.0, dt: float = 1.0, ntheta: int = 64, nparticles: int = 1024,
         resampler: str = "systematic", ess_rel: float = 1.0, theta_ess_rel: float = 0.5, moves: int = 1,
         seed: int = 0, metropolis_steps: int = 0, stream=None):
    """SMC^2 (MarginalSIR) over the batched filter: returns dict(theta[P, k],
    log_weights[P], log_evidence_increments[T], resample_steps, acceptance)."""
    cfg = N.Smc2Config()
    cfg.ntheta, cfg.nparticles = ntheta, nparticles
    cfg.resampler, cfg.metropolis_steps = RESAMPLERS[resampler], metropolis_steps
    cfg.ess_rel, cfg.theta_ess_rel, cfg.moves, cfg.seed = ess_rel, theta_ess_rel, moves, seed
    cfg.nparams = len(priors)
    for j, q in enumerate(priors):
        cfg.params[j].index, cfg.params[j].prior = q.index, _KINDS[q.kind]
        cfg.params[j].a, cfg.params[j].b, cfg.params[j].step = q.a, q.b, q.step
    desc = model.desc()
    yy = np.ascontiguousarray(np.asarray(y, dtype=model.np_dtype))
    T = yy.size // model.nobs
    th, lw, ev = np.zeros((ntheta, len(priors))), np.zeros(ntheta), np.zeros(T)
    nres, acc = ctypes.c_int(), ctypes.c_double()
    N.check(N.lib().bpf_smc2_run(ctypes.byref(desc), ctypes.byref(cfg), T, t0, dt, _ptr_np(yy), stream, _ptr_np(th),
                                 _ptr_np(lw), _ptr_np(ev), ctypes.byref(nres), ctypes.byref(acc)), "bpf_smc2_run")
    return dict(theta=th, log_weights=lw, log_evidence_increments=ev, resample_steps=nres.value,
                acceptance=acc.value)
