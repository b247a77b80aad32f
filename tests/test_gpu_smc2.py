"""SMC^2 over the batched filter (bpf_smc2_run, MarginalSIR): without
parameter resampling it is importance sampling from the priors, each
parameter particle's final log-weight equal to a single filter's
log-likelihood with its parameters and seed; with resample-move rounds the
run is deterministic, moves are accepted at a proper rate and the internal
replays reproduce every log-likelihood (checked by the run itself)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _priors():
    from libbi_b200 import Prior

    return [Prior(0, "uniform", 0.1, 0.5, 0.02), Prior(3, "log_normal", math.log(0.1), 0.5, 0.02)]


def test_smc2_without_resampling_is_importance_sampling(cuda, oracle):
    from libbi_b200 import BootstrapPF, ModelPZ, smc2

    T, dt, P, N, seed = 15, 1.0, 6, 512, 21
    model = ModelPZ()
    y, _ = oracle.simulate(model.desc(), 4, T, 0.0, dt)
    out = smc2(model, _priors(), y[:, 0], 0.0, dt, ntheta=P, nparticles=N, ess_rel=1.0, theta_ess_rel=0.0,
               moves=0, seed=seed)
    assert out["resample_steps"] == 0
    for i in range(P):
        c, q = out["theta"][i]
        pf = BootstrapPF(ModelPZ(c=c, q=q), N, ess_rel=1.0, seed=seed + 1 + i)
        ll, _, _ = pf.filter(y[:, 0], 0.0, dt)
        np.testing.assert_allclose(out["log_weights"][i], ll, rtol=1e-12)
        pf.close()
    # the evidence increments telescope to log mean exp of the final weights
    lw = out["log_weights"]
    m = lw.max()
    np.testing.assert_allclose(out["log_evidence_increments"].sum(), m + np.log(np.mean(np.exp(lw - m))),
                               rtol=1e-10)


def test_smc2_resample_move_is_deterministic(cuda, oracle):
    from libbi_b200 import ModelPZ, smc2

    T, dt = 30, 1.0
    model = ModelPZ()
    y, _ = oracle.simulate(model.desc(), 4, T, 0.0, dt)
    kw = dict(ntheta=32, nparticles=256, ess_rel=1.0, theta_ess_rel=0.5, moves=2, seed=3)
    a = smc2(model, _priors(), y[:, 0], 0.0, dt, **kw)
    b = smc2(model, _priors(), y[:, 0], 0.0, dt, **kw)
    assert a["resample_steps"] >= 1
    assert 0.0 < a["acceptance"] < 1.0
    assert np.isfinite(a["log_evidence_increments"]).all()
    np.testing.assert_array_equal(a["theta"], b["theta"])
    np.testing.assert_array_equal(a["log_evidence_increments"], b["log_evidence_increments"])
