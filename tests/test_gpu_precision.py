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


def test_one_step_same_input_within_1e_4(cuda, oracle):
    import torch
    from libbi_b200 import BootstrapPF, ModelL96

    m32, m64 = ModelL96(dim=40), ModelL96(dim=40, precision="f64")
    n, dt, T = 4096, 0.05, 30
    y64 = np.asarray(_obs(oracle, m64, T, dt, 12), np.float64)
    y32 = y64.astype(np.float32)
    ref = BootstrapPF(m64, n, ess_rel=0.5, seed=5)
    errs = []
    for k in range(T):
        if k in (0, 3, 12, 29):
            x, lw, _ = ref.state()
            x, lw = x[:, :n].clone(), lw.clone()
            lw_inj = float(torch.logsumexp(lw, 0)) - np.log(n)
            incs = []
            for m, y in ((m32, y32), (m64, y64)):
                pf = BootstrapPF(m, n, ess_rel=0.5, seed=77)
                xv, lwv, _ = pf.state()
                xv[:, :n].copy_(x.to(xv.dtype))
                lwv.copy_(lw)
                incs.append(pf.step(k * dt, (k + 1) * dt, y[k]).log_increment)
                pf.close()
            errs.append(abs(incs[0] - incs[1]) / max(abs(incs[1] - lw_inj), 1.0))
        ref.step(k * dt, (k + 1) * dt, y64[k])
    ref.close()
    assert max(errs) <= 1e-4, errs


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
