"""Host-side mirror of the learned proposal (bpf_proposal_*,
include/libbi_b200.h): create, train on simulated triples, attach to a
filter (BootstrapPF.set_proposal)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N


class LearnedProposal:
    """Lorenz '96: q(x_{t+1} | x_t, y_{t+1}) = N(m(x_t) + delta,
    diag(exp(2 s))) with (delta, s) from a 80-128-128-80 network on the
    tensor cores.  Plankton (PZ): q(log alpha | P, Z, y_{t+1}) =
    N(mu + delta, exp(2 s)) over the transition's log-noise, from a
    3-128-128-2 network."""

    def __init__(self, model, dt: float, max_batch: int = 8192, seed: int = 0, stream=None):
        self.model = model
        self.dt = dt
        self._desc = model.desc()
        self._h = ctypes.c_void_p()
        N.check(N.lib().bpf_proposal_create(ctypes.byref(self._desc), dt, max_batch, seed, stream,
                                            ctypes.byref(self._h)), "bpf_proposal_create")
        self._data = None
        self.din = 3 if self._desc.kind == N.BPF_MODEL_PZ else 2 * self._desc.dim

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            N.load_library().bpf_proposal_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_data(self, x_t, x_t1, y_t1):
        """Training triples: CUDA float32 tensors (n, 40), kept alive here."""
        for t in (x_t, x_t1, y_t1):
            if not (t.is_cuda and t.is_contiguous()):
                raise ValueError("expected contiguous CUDA tensors")
        self._data = (x_t, x_t1, y_t1)
        N.check(N.lib().bpf_proposal_set_data(self._h, x_t.data_ptr(), x_t1.data_ptr(), y_t1.data_ptr(),
                                              x_t.shape[0]), "bpf_proposal_set_data")

    def set_states(self, x_t):
        """PZ: training rows simulated by the model from the states x_t (a
        CUDA float64 tensor (n, 2)), kept alive here."""
        if not (x_t.is_cuda and x_t.is_contiguous()):
            raise ValueError("expected a contiguous CUDA tensor")
        self._data = (x_t,)
        N.check(N.lib().bpf_proposal_set_states(self._h, x_t.data_ptr(), x_t.shape[0]), "bpf_proposal_set_states")

    def train(self, steps: int, batch: int = 4096, lr: float = 1e-3, trace: bool = True):
        out = np.zeros(steps, np.float32) if trace else None
        N.check(N.lib().bpf_proposal_train(self._h, steps, batch, lr,
                                           None if out is None else out.ctypes.data_as(ctypes.c_void_p)),
                "bpf_proposal_train")
        return out

    def params(self):
        """(flat FP32 parameters, input shift, input scale)."""
        n = ctypes.c_int()
        N.lib().bpf_proposal_params(self._h, None, None, None, ctypes.byref(n))
        P = np.zeros(n.value, np.float32)
        sh, sc = np.zeros(self.din, np.float32), np.zeros(self.din, np.float32)
        N.check(N.lib().bpf_proposal_params(self._h, P.ctypes.data_as(ctypes.c_void_p),
                                            sh.ctypes.data_as(ctypes.c_void_p), sc.ctypes.data_as(ctypes.c_void_p),
                                            None), "bpf_proposal_params")
        return P, sh, sc

    def set_params(self, params=None, shift=None, scale=None):
        def p(a):
            return None if a is None else np.ascontiguousarray(a, np.float32).ctypes.data_as(ctypes.c_void_p)

        keep = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (params, shift, scale)]
        N.check(N.lib().bpf_proposal_set_params(self._h, *(None if a is None else a.ctypes.data_as(ctypes.c_void_p)
                                                           for a in keep)), "bpf_proposal_set_params")
