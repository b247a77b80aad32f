"""Particle-marginal Metropolis-Hastings over many chains (bpf_pmmh_*):
every chain's proposals and acceptance draws replayed from the oracle's
restatement of the draw scheme, the Metropolis-Hastings rule of
MarginalMH::acceptReject (share/src/bi/sampler/MarginalMH.hpp:250-271)
replayed on the host, and a share of the proposals' filter log-likelihoods
checked against the oracle's FP64 filter with the same seeds."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _log_prior(priors, th):
    lp = 0.0
    for q in priors:
        x = th[q.index] if len(th) > q.index else th[priors.index(q)]
        if q.kind == "uniform":
            lp += -math.log(q.b - q.a) if q.a <= x <= q.b else -math.inf
        elif q.kind == "log_normal":
            if x <= 0:
                return -math.inf
            z = (math.log(x) - q.a) / q.b
            lp += -0.5 * z * z - 0.91893853320467274178032973640562 - math.log(q.b * x)
    return lp


def test_pmmh_chains_follow_the_mh_rule_and_oracle_filters(cuda, oracle):
    from libbi_b200 import MarginalMH, ModelPZ, Prior
    from libbi_b200 import _native as N

    T, dt = 20, 1.0
    truth = ModelPZ()
    y, _ = oracle.simulate(truth.desc(), 4, T, 0.0, dt)
    priors = [Prior(0, "uniform", 0.0, 1.0, 0.02), Prior(1, "uniform", 0.0, 1.0, 0.02),
              Prior(2, "log_normal", math.log(0.1), 0.5, 0.02), Prior(3, "log_normal", math.log(0.1), 0.5, 0.02)]
    C, Np, seed, iters = 8, 256, 11, 12
    rng = np.random.default_rng(0)
    th0 = np.array([[0.25, 0.3, 0.1, 0.1]] * C) * (1.0 + 0.05 * rng.standard_normal((C, 4)))
    th0[0, 1] = 0.999  # near the edge of its uniform prior: some proposals fall outside
    mh = MarginalMH(truth, priors, y[:, 0], 0.0, dt, nchains=C, nparticles=Np, resampler="systematic",
                    ess_rel=1.0, seed=seed, theta0=th0)
    cur, cll, clp, runs = mh.state()
    assert runs == 1
    np.testing.assert_array_equal(cur, th0)

    def oracle_ll(theta, fseed):
        m = ModelPZ(c=theta[0], e=theta[1], m=theta[2], q=theta[3])
        cfg = N.Config()
        cfg.nparticles, cfg.resampler, cfg.ess_rel, cfg.seed = Np, 0, 1.0, fseed
        out = oracle.filter(m.desc(), cfg, y, T, 0.0, dt)
        return out["ll"] if out["rc"] == 0 else -math.inf

    for c in (0, 5):
        np.testing.assert_allclose(cll[c], oracle_ll(cur[c], seed + 1 + c), rtol=1e-10)

    out = mh.run(iters)
    steps = np.array([q.step for q in priors])
    checked = outside = 0
    for i in range(iters):
        r = i + 1
        for c in range(C):
            z, u = oracle.pmmh_draws(seed, c, r, 4)
            prop = cur[c] + steps * z
            lp2 = _log_prior(priors, prop)
            ll2 = out["proposal_loglik"][i, c]
            if not math.isfinite(lp2):
                assert ll2 == -math.inf
                outside += 1
            elif (i * C + c) % 10 == 0:
                np.testing.assert_allclose(ll2, oracle_ll(prop, seed + 1 + r * C + c), rtol=1e-10)
                checked += 1
            if not math.isfinite(ll2):
                acc = False
            elif not math.isfinite(cll[c]):
                acc = True
            else:
                acc = math.log(u) < (ll2 - cll[c]) + (lp2 - clp[c])
            if acc:
                cur[c], cll[c], clp[c] = prop, ll2, lp2
            np.testing.assert_array_equal(out["samples"][i, c], cur[c])
            assert out["loglik"][i, c] == cll[c]
            np.testing.assert_allclose(out["logprior"][i, c], clp[c], rtol=1e-14)
    assert checked >= 5 and outside >= 1
    acc_rate = (out["accepted"] - 1) / iters
    assert (acc_rate > 0).any() and (acc_rate < 1).any()
    mh.close()


def test_pmmh_chains_with_their_own_particle_counts(cuda, oracle):
    """Chains with different filter sizes (N log-uniform in [1024, 8192]):
    each chain's initial log-likelihood and its accepted proposals'
    log-likelihoods equal the oracle's FP64 filter with that chain's N and
    seed."""
    from libbi_b200 import MarginalMH, ModelPZ, Prior
    from libbi_b200 import _native as N

    T, dt = 15, 1.0
    truth = ModelPZ()
    y, _ = oracle.simulate(truth.desc(), 4, T, 0.0, dt)
    priors = [Prior(0, "uniform", 0.0, 1.0, 0.02), Prior(1, "uniform", 0.0, 1.0, 0.02),
              Prior(2, "log_normal", math.log(0.1), 0.5, 0.02), Prior(3, "log_normal", math.log(0.1), 0.5, 0.02)]
    C, seed, iters = 6, 21, 4
    ns = [1024, 8192, 2048, 4000, 1500, 6144]
    th0 = np.array([[0.25, 0.3, 0.1, 0.1]] * C)
    mh = MarginalMH(truth, priors, y[:, 0], 0.0, dt, nchains=C, nparticles=ns, resampler="systematic",
                    ess_rel=1.0, seed=seed, theta0=th0)

    def oracle_ll(theta, n, fseed):
        m = ModelPZ(c=theta[0], e=theta[1], m=theta[2], q=theta[3])
        cfg = N.Config()
        cfg.nparticles, cfg.resampler, cfg.ess_rel, cfg.seed = n, 0, 1.0, fseed
        out = oracle.filter(m.desc(), cfg, y, T, 0.0, dt)
        return out["ll"] if out["rc"] == 0 else -math.inf

    _, cll, _, _ = mh.state()
    for c in range(C):
        np.testing.assert_allclose(cll[c], oracle_ll(th0[c], ns[c], seed + 1 + c), rtol=1e-10)
    out = mh.run(iters)
    checked = 0
    prev = th0
    for i in range(iters):
        r = i + 1
        for c in range(C):
            if not np.array_equal(out["samples"][i, c], prev[c]):
                np.testing.assert_allclose(out["proposal_loglik"][i, c],
                                           oracle_ll(out["samples"][i, c], ns[c], seed + 1 + r * C + c), rtol=1e-10)
                checked += 1
        prev = out["samples"][i]
    assert checked >= 2
    mh.close()
