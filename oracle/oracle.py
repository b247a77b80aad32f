"""ORACLE — test infrastructure only (tests/, the smoke check and the bench's
CPU-baseline leg).  ctypes binding of the C restatement (bpf_oracle.c ->
_build/liboracle.so) and of the reference's own code compiled from its
sources, when built: the resampler code (ref/ref_resampler.cpp) and the host
updaters on hand-rendered model classes (ref/model_l96.cpp, ref/model_pz.cpp)
-> _ref/libbiref.so, and the L96 model with real = float -> _ref/libbiref_f32.so."""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbiref.so")
REF_F32_SO = os.path.join(HERE, "_ref", "libbiref_f32.so")
REF_TREE = "/root/reference/share/src"


def build(ref: bool = True) -> None:
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref and os.path.isdir(REF_TREE):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_TREE}"], check=True)


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        L = ctypes.CDLL(path)
        L.orc_ess_reduce.restype = c_double
        L.orc_ess_reduce.argtypes = [c_void_p, c_int, POINTER(c_double)]
        L.orc_logsumexp.restype = c_double
        L.orc_logsumexp.argtypes = [c_void_p, c_int]
        L.orc_systematic.argtypes = [c_void_p, c_int, c_double, c_int, c_void_p, c_void_p, c_void_p]
        L.orc_multinomial.argtypes = [c_void_p, c_int, c_void_p, c_int, c_void_p]
        L.orc_metropolis.argtypes = [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p]
        L.orc_cumsum_exact.argtypes = [c_void_p, c_int, c_void_p]
        L.orc_ref_permute.argtypes = [c_void_p, c_int]
        L.orc_permute_rule.argtypes = [c_void_p, c_int, c_void_p]
        L.orc_gather.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int]
        L.orc_resample_uniforms.argtypes = [c_int, c_int, c_int, c_uint64, c_int, c_void_p]
        L.orc_init.argtypes = [c_void_p, c_void_p, c_int, c_int, c_void_p, c_uint64]
        L.orc_transition.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_void_p,
                                     c_void_p, c_double, c_double, c_uint64, c_int, c_double]
        L.orc_filter.argtypes = [c_void_p, c_void_p, c_int, c_double, c_double, c_void_p, c_void_p, c_void_p,
                                 c_void_p, POINTER(c_double), c_void_p, c_void_p]
        L.orc_transition_mask.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_void_p,
                                          c_void_p, c_double, c_double, c_uint64, c_int, c_double, c_uint64]
        L.orc_noise_normals.argtypes = [c_uint64, ctypes.c_uint32, c_int, c_int, c_int, c_void_p]
        L.orc_pmmh_draws.argtypes = [c_uint64, c_int, c_int, c_int, c_void_p, POINTER(c_double)]
        L.orc_simulate.argtypes = [c_void_p, c_uint64, c_int, c_double, c_double, c_void_p, c_void_p]
        L.orc_pz_guided_step.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_void_p,
                                         c_double, c_double, c_double, c_uint64, c_int, c_double, c_void_p, c_void_p]
        self.L = L

    # reductions
    def ess_reduce(self, lw):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        lW = c_double()
        ess = self.L.orc_ess_reduce(_p(lw), lw.size, ctypes.byref(lW))
        return ess, lW.value

    def logsumexp(self, lw):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        return self.L.orc_logsumexp(_p(lw), lw.size)

    # resamplers
    def systematic(self, lw, a, permute=True):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        n = lw.size
        Ws, Os, as_ = np.zeros(n), np.zeros(n, np.int32), np.zeros(n, np.int32)
        rc = self.L.orc_systematic(_p(lw), n, float(a), int(permute), _p(Ws), _p(Os), _p(as_))
        return rc, Ws, Os, as_

    def multinomial(self, lw, u, permute=0):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        as_ = np.zeros(lw.size, np.int32)
        rc = self.L.orc_multinomial(_p(lw), lw.size, _p(u), int(permute), _p(as_))
        return rc, as_

    def metropolis(self, lw, B, u, permute=0):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        as_ = np.zeros(lw.size, np.int32)
        rc = self.L.orc_metropolis(_p(lw), lw.size, int(B), _p(u), int(permute), _p(as_))
        return rc, as_

    def cumsum_exact(self, lw):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        Ws = np.zeros(lw.size)
        self.L.orc_cumsum_exact(_p(lw), lw.size, _p(Ws))
        return Ws

    def ref_permute(self, as_):
        a = np.ascontiguousarray(as_, dtype=np.int32).copy()
        self.L.orc_ref_permute(_p(a), a.size)
        return a

    def permute_rule(self, as_):
        a = np.ascontiguousarray(as_, dtype=np.int32)
        out = np.zeros_like(a)
        self.L.orc_permute_rule(_p(a), a.size, _p(out))
        return out

    def resample_uniforms(self, kind, n, B, seed, step):
        size = 1 if kind == 0 else (n if kind == 1 else 2 * n * max(B, 1))
        u = np.zeros(size)
        self.L.orc_resample_uniforms(kind, n, B, seed, step, _p(u))
        return u

    # models / filter
    def init(self, desc, n, seed):
        ld = (n + 31) // 32 * 32
        dt = np.float32 if desc.precision == 0 else np.float64
        x = np.zeros((desc.dim, ld), dt)
        lw = np.zeros(n)
        self.L.orc_init(ctypes.byref(desc), _p(x), ld, n, _p(lw), seed)
        return x, lw

    def transition(self, desc, x_in, n, as_, resampled, lw, y, t1, t2, seed, step, ll):
        x_out = np.zeros_like(x_in)
        lw = lw.copy()
        as_ = None if as_ is None else np.ascontiguousarray(as_, np.int32)
        y = None if y is None else np.ascontiguousarray(y, x_in.dtype)
        self.L.orc_transition(ctypes.byref(desc), _p(x_in), _p(x_out), x_in.shape[1], n, _p(as_), int(resampled),
                              _p(lw), _p(y), t1, t2, seed, step, ll)
        return x_out, lw

    def transition_mask(self, desc, x_in, n, as_, resampled, lw, y, t1, t2, seed, step, ll, mask):
        """transition with only the components of bitmask `mask` observed"""
        x_out = np.zeros_like(x_in)
        lw = lw.copy()
        as_ = None if as_ is None else np.ascontiguousarray(as_, np.int32)
        y = None if y is None else np.ascontiguousarray(y, x_in.dtype)
        self.L.orc_transition_mask(ctypes.byref(desc), _p(x_in), _p(x_out), x_in.shape[1], n, _p(as_),
                                   int(resampled), _p(lw), _p(y), t1, t2, seed, step, ll, mask)
        return x_out, lw

    def filter(self, desc, cfg, y, T, t0, dt):
        n = cfg.nparticles
        ld = (n + 31) // 32 * 32
        dtp = np.float32 if desc.precision == 0 else np.float64
        y = np.ascontiguousarray(y, dtp)
        inc, ess, res = np.zeros(T), np.zeros(T), np.zeros(T, np.int32)
        ll = c_double()
        x = np.zeros((desc.dim, ld), dtp)
        lw = np.zeros(n)
        rc = self.L.orc_filter(ctypes.byref(desc), ctypes.byref(cfg), T, t0, dt, _p(y), _p(inc), _p(ess), _p(res),
                               ctypes.byref(ll), _p(x), _p(lw))
        return dict(rc=rc, ll=ll.value, inc=inc, ess=ess, resampled=res, x=x, lw=lw)

    def pz_guided_step(self, desc, x_in, n, as_, resampled, lw, y, t1, t2, seed, step, ll, delta, s):
        """The PZ guided step given the proposal's outputs (delta[n], s[n],
        s clamped): returns (x_out, lw_out)."""
        x_in = np.ascontiguousarray(x_in, np.float64)
        x_out = np.zeros_like(x_in)
        lw = np.ascontiguousarray(lw, np.float64).copy()
        as_ = None if as_ is None else np.ascontiguousarray(as_, np.int32)
        d = np.ascontiguousarray(delta, np.float64)
        s = np.ascontiguousarray(s, np.float64)
        self.L.orc_pz_guided_step(ctypes.byref(desc), _p(x_in), _p(x_out), x_in.shape[1], n, _p(as_), int(resampled),
                                  _p(lw), float(y), t1, t2, seed, step, ll, _p(d), _p(s))
        return x_out, lw

    def noise_normals(self, seed, p, step, n, f32):
        """The n standard normals of particle p's process noise at step, in
        the order the transition consumes them (include/bpf_philox.h)."""
        z = np.zeros(n)
        self.L.orc_noise_normals(c_uint64(seed), int(p), int(step), int(n), 0 if f32 else 1, _p(z))
        return z

    def pmmh_draws(self, seed, c, r, nparams):
        """(proposal normals[nparams], acceptance uniform) of PMMH chain c at
        filter run r."""
        z = np.zeros(nparams)
        u = c_double()
        self.L.orc_pmmh_draws(c_uint64(seed), int(c), int(r), int(nparams), _p(z), ctypes.byref(u))
        return z, u.value

    def simulate(self, desc, seed, T, t0, dt):
        dtp = np.float32 if desc.precision == 0 else np.float64
        nobs = desc.dim if desc.kind == 1 else 1
        y = np.zeros(T * nobs, dtp)
        xt = np.zeros(T * desc.dim, dtp)
        self.L.orc_simulate(ctypes.byref(desc), seed, T, t0, dt, _p(y), _p(xt))
        return y.reshape(T, nobs), xt.reshape(T, desc.dim)


class RefResampler:
    """The reference's own host resampler code (share/src/bi/...), compiled
    from its sources with a tape of uniforms (oracle/ref/ref_resampler.cpp)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise OSError(f"reference build missing: {path}")
        L = ctypes.CDLL(path)
        L.ref_ess_reduce.restype = c_double
        L.ref_ess_reduce.argtypes = [c_void_p, c_int, POINTER(c_double)]
        L.ref_logsumexp_reduce.restype = c_double
        L.ref_logsumexp_reduce.argtypes = [c_void_p, c_int]
        L.ref_systematic.argtypes = [c_void_p, c_int, c_double, c_int, c_void_p, c_void_p, c_void_p]
        L.ref_multinomial.argtypes = [c_void_p, c_int, c_void_p, c_int, c_void_p]
        L.ref_metropolis.argtypes = [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p]
        L.ref_permute.argtypes = [c_void_p, c_int]
        L.ref_gather_rows.argtypes = [c_void_p, c_void_p, c_int, c_int]
        self.L = L

    def ess_reduce(self, lw):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        lW = c_double()
        return self.L.ref_ess_reduce(_p(lw), lw.size, ctypes.byref(lW)), lW.value

    def logsumexp(self, lw):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        return self.L.ref_logsumexp_reduce(_p(lw), lw.size)

    def systematic(self, lw, a, permute=True):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        n = lw.size
        Ws, Os, as_ = np.zeros(n), np.zeros(n, np.int32), np.zeros(n, np.int32)
        rc = self.L.ref_systematic(_p(lw), n, float(a), int(permute), _p(Ws), _p(Os), _p(as_))
        return rc, Ws, Os, as_

    def multinomial(self, lw, u, permute=0):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        as_ = np.zeros(lw.size, np.int32)
        rc = self.L.ref_multinomial(_p(lw), lw.size, _p(u), int(permute), _p(as_))
        return rc, as_

    def metropolis(self, lw, B, u, permute=0):
        lw = np.ascontiguousarray(lw, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        as_ = np.zeros(lw.size, np.int32)
        rc = self.L.ref_metropolis(_p(lw), lw.size, int(B), _p(u), int(permute), _p(as_))
        return rc, as_

    def permute(self, as_):
        a = np.ascontiguousarray(as_, dtype=np.int32).copy()
        self.L.ref_permute(_p(a), a.size)
        return a

    def gather_rows(self, as_, X):
        X = np.ascontiguousarray(X, dtype=np.float64).copy()
        d, n = X.shape
        a = np.ascontiguousarray(as_, dtype=np.int32)
        self.L.ref_gather_rows(_p(a), _p(X), n, d)
        return X


class RefModels:
    """The reference's own host updaters (RK4IntegratorHost,
    RK43IntegratorHost, StaticSamplerHost, StaticUpdaterHost,
    SparseStaticLogDensityHost) on hand-rendered L96 (d = 40) and PZ model
    classes (oracle/ref/model_l96.cpp, model_pz.cpp), draws from a tape of
    standard normals.  f32 selects the L96 build with real = float."""

    L96_DIM = 40

    def __init__(self, f32: bool = False):
        path = REF_F32_SO if f32 else REF_SO
        if not os.path.exists(path):
            raise OSError(f"reference build missing: {path}")
        L = ctypes.CDLL(path)
        sig = [c_void_p, c_int, c_void_p, c_double, c_double, c_void_p, c_void_p]
        L.ref_l96_transition.argtypes = sig
        if not f32:
            L.ref_pz_transition.argtypes = sig
        self.L = L
        self.f32 = f32

    def l96_transition(self, x, z, t1, t2, y=None, lp=None):
        """x: (P, 40) particle-major state; z: (P, 40) standard normals in the
        sampler's draw order; returns (x_out, lp_out)."""
        x = np.ascontiguousarray(x, np.float64).copy()
        P = x.shape[0]
        z = np.ascontiguousarray(z, np.float64)
        lp = np.zeros(P) if lp is None else np.ascontiguousarray(lp, np.float64).copy()
        y = None if y is None else np.ascontiguousarray(y, np.float64)
        rc = self.L.ref_l96_transition(_p(x), P, _p(z), float(t1), float(t2), _p(y), _p(lp))
        if rc:
            raise RuntimeError("reference L96 transition did not consume its draws exactly")
        return x, lp

    def pz_transition(self, x, z, t1, t2, y=None, lp=None):
        """x: (P, 2) state (P, Z); z: P standard normals (the alpha draws)."""
        x = np.ascontiguousarray(x, np.float64).copy()
        P = x.shape[0]
        z = np.ascontiguousarray(z, np.float64)
        lp = np.zeros(P) if lp is None else np.ascontiguousarray(lp, np.float64).copy()
        y = None if y is None else np.ascontiguousarray(np.atleast_1d(y), np.float64)
        rc = self.L.ref_pz_transition(_p(x), P, _p(z), float(t1), float(t2), _p(y), _p(lp))
        if rc:
            raise RuntimeError("reference PZ transition did not consume its draws exactly")
        return x, lp
