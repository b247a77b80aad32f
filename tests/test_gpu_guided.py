"""The guided filter step (learned proposal + importance weights): one step
against the CPU oracle's restatement (RK4 mean from the oracle's model with
no noise, the network from oracle/mlp_oracle.py with the same BF16
roundings, the same standard normals), and filter-level behaviour: an
untrained proposal (close to the transition) gives the bootstrap filter's
likelihood, a trained one on an informative observation cuts its variance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _truth(oracle, model, T, dt, seed):
    y, _ = oracle.simulate(model.desc(), seed, T, 0.0, dt)
    return y


def test_guided_step_matches_oracle(cuda, oracle):
    from libbi_b200 import BootstrapPF, LearnedProposal, ModelL96
    from oracle.mlp_oracle import forward, guided_step

    model = ModelL96(dim=40, sigma_eta=0.5, sigma_y=0.1)
    n, dt, seed = 1000, 0.05, 21
    prop = LearnedProposal(model, dt, max_batch=1024, seed=4)
    P, sh, sc = prop.params()
    rng = np.random.default_rng(0)
    P = (P + 0.05 * rng.standard_normal(P.size)).astype(np.float32)
    sh = (0.3 * rng.standard_normal(80)).astype(np.float32)
    sc = (1.0 + 0.1 * rng.standard_normal(80)).astype(np.float32)
    prop.set_params(P, sh, sc)
    pf = BootstrapPF(model, n, ess_rel=0.0, seed=seed)
    pf.set_proposal(prop)
    x0, lw0, _ = pf.state()
    x0 = x0.cpu().numpy()[:, :n].copy()
    y = _truth(oracle, model, 1, dt, 8)[0]
    pf.step(0.0, dt, y)
    x1, lw1, _ = pf.state()
    x1, lw1 = x1.cpu().numpy()[:, :n], lw1.cpu().numpy()
    # oracle: RK4 mean (sigma_eta = 0), network, normals of step 1
    mdesc = ModelL96(dim=40, sigma_eta=0.0, sigma_y=0.1).desc()
    m, _ = oracle.transition(mdesc, x0, n, None, False, np.zeros(n), None, 0.0, dt, seed, 1, 0.0)
    m = m[:, :n].T.astype(np.float32)
    delta, s = forward(P, sh, sc, x0.T.astype(np.float32), (y[None, :] - m).astype(np.float32))
    z = np.stack([oracle.noise_normals(seed, p, 1, 40, True) for p in range(n)]).astype(np.float32)
    xw, lww = guided_step(delta.astype(np.float64), s.astype(np.float64), m.astype(np.float64), z, y, 0.5, 0.1,
                          np.zeros(n))
    dx = np.abs(x1.T - xw)
    assert np.median(dx) < 1e-5 and dx.max() < 5e-3, (np.median(dx), dx.max())
    dl = np.abs(lw1 - lww) / np.maximum(1.0, np.abs(lww))
    assert np.median(dl) < 1e-5 and dl.max() < 5e-3, (np.median(dl), dl.max())
    pf.close()
    prop.close()


def _lls(model, prop, y, n, seeds, dt):
    from libbi_b200 import BootstrapPF

    out = []
    for s in seeds:
        pf = BootstrapPF(model, n, ess_rel=0.5, seed=s)
        if prop is not None:
            pf.set_proposal(prop)
        ll, _, _ = pf.filter(y, 0.0, dt)
        out.append(ll)
        pf.close()
    return np.array(out)


def test_untrained_proposal_gives_the_bootstrap_likelihood(cuda, oracle):
    from libbi_b200 import LearnedProposal, ModelL96

    model = ModelL96(dim=40)
    dt, T, n = 0.05, 10, 2048
    y = _truth(oracle, model, T, dt, 31)
    prop = LearnedProposal(model, dt, seed=2)
    seeds = list(range(100, 116))
    a = _lls(model, None, y, n, seeds, dt)
    b = _lls(model, prop, y, n, seeds, dt)
    # the untrained proposal is the transition (delta = 0, s = log sigma_eta):
    # the same draws, weights equal to rounding
    assert np.median(np.abs(a - b)) < 1e-2, (a, b)
    se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
    assert abs(a.mean() - b.mean()) < 4 * se + 1e-6, (a.mean(), b.mean(), se)
    prop.close()


def test_trained_proposal_cuts_variance_on_informative_observations(cuda, oracle):
    import torch
    from libbi_b200 import BootstrapPF, LearnedProposal, ModelL96

    model = ModelL96(dim=40, sigma_eta=0.5, sigma_y=0.1)
    dt, n_data = 0.05, 1 << 16
    sim = BootstrapPF(model, n_data, seed=9)
    for k in range(40):
        sim.step(k * dt, (k + 1) * dt, None)
    x, _, _ = sim.state()
    xt = x[:, :n_data].T.contiguous().clone()
    sim.step(40 * dt, 41 * dt, None)
    x, _, _ = sim.state()
    xt1 = x[:, :n_data].T.contiguous().clone()
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    yt1 = (xt1 + model.sigma_y * torch.randn(xt1.shape, generator=g, device="cuda")).contiguous()
    sim.close()
    prop = LearnedProposal(model, dt, max_batch=4096, seed=5)
    prop.set_data(xt, xt1, yt1)
    trace = prop.train(1500, 4096, 2e-3)
    assert trace[-50:].mean() / 40 < trace[:10].mean() / 40 - 0.5
    y = _truth(oracle, model, 8, dt, 77)
    seeds = list(range(200, 212))
    boot = _lls(model, None, y, 1024, seeds, dt)
    guid = _lls(model, prop, y, 1024, seeds, dt)
    assert np.isfinite(guid).all()
    assert guid.std() < 0.5 * boot.std(), (guid.std(), boot.std())
    # log-likelihood estimates are biased low by their variance: the guided
    # (lower-variance) estimate is not below the bootstrap's
    assert guid.mean() > boot.mean() - 2 * boot.std() / np.sqrt(len(boot))
    prop.close()


def test_batched_guided_matches_single_guided_filters(cuda, oracle):
    """The guided step of a batch (one launch over every filter's 128-particle
    tiles) against single guided filters with the same N, resampler, seed and
    constants: increments, ESS, states and log-weights bit for bit."""
    from libbi_b200 import BatchedBootstrapPF, BootstrapPF, LearnedProposal, ModelL96

    dt, T = 0.05, 8
    Fs = [8.0, 7.5, 8.5, 9.0, 6.5]
    models = [ModelL96(dim=40, F=F, sigma_eta=0.5, sigma_y=0.1) for F in Fs]
    ns = [100, 128, 1000, 4096, 300]
    res = ["systematic", "multinomial", "systematic", "metropolis", "systematic"]
    seeds = [31 + f for f in range(len(ns))]
    prop = LearnedProposal(models[0], dt, max_batch=1024, seed=4)
    P, sh, sc = prop.params()
    rng = np.random.default_rng(2)
    prop.set_params((P + 0.03 * rng.standard_normal(P.size)).astype(np.float32), sh, sc)
    y = np.stack([oracle.simulate(m.desc(), 60 + f, T, 0.0, dt)[0] for f, m in enumerate(models)], axis=1)
    singles = []
    for f, m in enumerate(models):
        pf = BootstrapPF(m, ns[f], resampler=res[f], ess_rel=0.5, seed=seeds[f], metropolis_steps=4)
        pf.set_proposal(prop)
        ll, inc, ess = pf.filter(y[:, f], 0.0, dt)
        x, lw, _ = pf.state()
        singles.append((ll, inc, ess, x.cpu().numpy()[:, :ns[f]].copy(), lw.cpu().numpy().copy()))
        pf.close()
    batch = BatchedBootstrapPF(models, ns, res, seeds, ess_rel=0.5, metropolis_steps=4)
    batch.set_proposal(prop)
    for _ in range(2):  # the capturing run and a graph replay
        ll, inc, ess, st = batch.filter(y, 0.0, dt)
        assert (st == 0).all()
        x, lw, _, offs = batch.state()
        x, lw = x.cpu().numpy(), lw.cpu().numpy()
        for f, (sll, sinc, sess, sx, slw) in enumerate(singles):
            np.testing.assert_array_equal(inc[:, f], sinc)
            np.testing.assert_array_equal(ess[:, f], sess)
            np.testing.assert_array_equal(x[:, offs[f]:offs[f] + ns[f]], sx)
            np.testing.assert_array_equal(lw[offs[f]:offs[f] + ns[f]], slw)
            np.testing.assert_allclose(ll[f], sll, rtol=1e-12)
    # detached again: the plain batched transition
    batch.set_proposal(None)
    _, inc0, _, _ = batch.filter(y, 0.0, dt)
    assert not np.array_equal(inc0, inc)
    batch.close()
    prop.close()
