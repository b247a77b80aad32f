"""FP32 against FP64 on the same seeds (identical Philox draws, so the two
filters differ by rounding only): one step from the same state and
log-weights agrees to 1e-4 relative, and over many seeds the two
log-likelihood estimators have the same mean within sampling error."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _obs(oracle, model, T, dt, seed):
    y, _ = oracle.simulate(model.desc(), seed, T, 0.0, dt)
    return y


def test_every_step_same_input_within_1e_4(cuda, oracle):
    """At every step of an FP64 run, its state and log-weights before the
    step are written into an FP32 and an FP64 filter, each takes the step:
    the increments agree to 1e-4 relative (to the step's own increment)."""
    import torch
    from libbi_b200 import BootstrapPF, ModelL96

    m32, m64 = ModelL96(dim=40), ModelL96(dim=40, precision="f64")
    n, dt, T = 4096, 0.05, 30
    y64 = np.asarray(_obs(oracle, m64, T, dt, 12), np.float64)
    y32 = y64.astype(np.float32)
    ref = BootstrapPF(m64, n, ess_rel=0.5, seed=5)
    probes = [BootstrapPF(m, n, ess_rel=0.5, seed=77) for m in (m32, m64)]
    errs = []
    for k in range(T):
        x, lw, _ = ref.state()
        lw_inj = float(torch.logsumexp(lw, 0)) - np.log(n)
        incs = []
        for pf, y in zip(probes, (y32, y64)):
            pf.init()
            xv, lwv, _ = pf.state()
            xv[:, :n].copy_(x[:, :n].to(xv.dtype))
            lwv.copy_(lw)
            incs.append(pf.step(k * dt, (k + 1) * dt, y[k]).log_increment)
        errs.append(abs(incs[0] - incs[1]) / max(abs(incs[1] - lw_inj), 1.0))
        ref.step(k * dt, (k + 1) * dt, y64[k])
    for pf in probes + [ref]:
        pf.close()
    assert max(errs) <= 1e-4, errs


def test_batched_fp32_against_fp64(cuda, oracle):
    """The batched filters in FP32 against the same batch in FP64 (same
    seeds, observations and settings): the first step's increments agree to
    1e-4, and the paired difference of the log-likelihood estimates has mean
    within three standard errors of zero."""
    from dataclasses import replace

    from libbi_b200 import BatchedBootstrapPF, ModelL96

    nf, T, dt = 24, 20, 0.05
    rng = np.random.default_rng(8)
    Fs = rng.uniform(6.0, 10.0, nf)
    ns = [int(v) for v in rng.integers(512, 4096, nf)]
    res = ["systematic" if f % 2 == 0 else "multinomial" for f in range(nf)]
    models = [ModelL96(dim=40, F=float(F)) for F in Fs]
    y = np.stack([oracle.simulate(m.desc(), 70 + f, T, 0.0, dt)[0] for f, m in enumerate(models)], axis=1)
    out = {}
    for prec in ("f32", "f64"):
        b = BatchedBootstrapPF([replace(m, precision=prec) for m in models], ns, res, list(range(300, 300 + nf)),
                               ess_rel=0.5)
        ll, inc, _, st = b.filter(y if prec == "f32" else y.astype(np.float64), 0.0, dt)
        assert (st == 0).all()
        out[prec] = (ll, inc)
        b.close()
    (l32, i32), (l64, i64) = out["f32"], out["f64"]
    first = np.abs(i32[0] - i64[0]) / np.maximum(np.abs(i64[0]), 1.0)
    assert first.max() <= 1e-4, first.max()
    d = l32 - l64
    assert abs(d.mean()) <= 3 * d.std(ddof=1) / np.sqrt(nf) + 1e-9 * np.abs(l64).mean(), (d.mean(), d.std())


def test_guided_every_step_against_fp64(cuda, oracle):
    """The guided filter (FP32 arithmetic, BF16 network operands with FP32
    accumulation) at every step of a run, from the same input, against the
    oracle's FP64 guided step (FP64 RK4 mean, the network in FP64 on the same
    BF16 weights and BF16-rounded inputs and activations, FP64 normals of the
    same draws): the step's log-likelihood increments agree to 1e-4
    relative at every step (measured on B200: median 1.4e-7, max 5.2e-7)."""
    from libbi_b200 import BootstrapPF, LearnedProposal, ModelL96
    from oracle.mlp_oracle import forward, guided_step

    model = ModelL96(dim=40, sigma_eta=0.5, sigma_y=0.1)
    n, dt, seed, T = 2048, 0.05, 21, 12
    prop = LearnedProposal(model, dt, max_batch=1024, seed=4)
    P, sh, sc = prop.params()
    rng = np.random.default_rng(0)
    P = (P + 0.05 * rng.standard_normal(P.size)).astype(np.float32)
    sh = (0.3 * rng.standard_normal(80)).astype(np.float32)
    sc = (1.0 + 0.1 * rng.standard_normal(80)).astype(np.float32)
    prop.set_params(P, sh, sc)
    y = _obs(oracle, model, T, dt, 8)
    pf = BootstrapPF(model, n, ess_rel=0.5, seed=seed)
    pf.set_proposal(prop)
    mdesc = ModelL96(dim=40, sigma_eta=0.0, sigma_y=0.1, precision="f64").desc()
    ll_prev, errs = 0.0, []
    for k in range(T):
        x_in, lw_in, _ = pf.state()
        x_in = x_in.cpu().numpy()[:, :n].astype(np.float64)
        lw_in = lw_in.cpu().numpy().copy()
        r = pf.step(k * dt, (k + 1) * dt, y[k])
        _, _, as_ = pf.state()
        if r.resampled:
            src = as_.cpu().numpy()
            x_src, base = np.ascontiguousarray(x_in[:, src]), np.full(n, ll_prev)
        else:
            x_src, base = x_in, lw_in
        ld = (n + 31) // 32 * 32
        xs = np.zeros((40, ld))
        xs[:, :n] = x_src
        m, _ = oracle.transition(mdesc, xs, n, None, False, np.zeros(n), None, k * dt, (k + 1) * dt, seed, k + 1,
                                 0.0)
        m = m[:, :n].T
        delta, s = forward(P, sh, sc, x_src.T, (np.asarray(y[k], np.float64)[None, :] - m))
        z = np.stack([oracle.noise_normals(seed, p, k + 1, 40, False) for p in range(n)])
        _, lw = guided_step(delta.astype(np.float64), s.astype(np.float64), m, z, np.asarray(y[k], np.float64),
                            0.5, 0.1, base)
        mx = lw.max()
        inc64 = mx + np.log(np.mean(np.exp(lw - mx))) - ll_prev
        errs.append(abs(r.log_increment - inc64) / max(abs(inc64), 1.0))
        ll_prev = r.log_likelihood
    pf.close()
    prop.close()
    errs = np.array(errs)
    print("guided FP32/BF16 vs FP64, per-step increment relative error: median %.3g max %.3g"
          % (np.median(errs), errs.max()))
    assert errs.max() <= 1e-4, errs


def test_estimator_means_agree(cuda, oracle):
    from libbi_b200 import BootstrapPF, ModelL96

    m32, m64 = ModelL96(dim=8), ModelL96(dim=8, precision="f64")
    n, dt, T, seeds = 1024, 0.05, 20, 24
    y64 = np.asarray(_obs(oracle, m64, T, dt, 3), np.float64)
    lls = {}
    for m, y in ((m32, y64.astype(np.float32)), (m64, y64)):
        out = []
        for s in range(seeds):
            pf = BootstrapPF(m, n, ess_rel=0.5, seed=900 + s)
            out.append(pf.filter(y, 0.0, dt)[0])
            pf.close()
        lls[m.precision] = np.array(out)
    a, b = lls["f32"], lls["f64"]
    se = np.sqrt(a.var(ddof=1) / seeds + b.var(ddof=1) / seeds)
    assert abs(a.mean() - b.mean()) <= 3 * se + 1e-9 * abs(b.mean()), (a.mean(), b.mean(), se)
