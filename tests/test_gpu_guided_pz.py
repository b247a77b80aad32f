"""The plankton (PZ) model's learned proposal over the transition's
log-noise: training on rows the model simulates from given states, the
batched guided step against the oracle's FP64 restatement
(orc_pz_guided_step, the network from oracle/mlp_oracle.py with the same
BF16 roundings), filter-level behaviour (an untrained proposal is the prior,
so the guided filter gives the bootstrap filter's likelihood; a trained one
cuts the estimator's spread on informative observations), and PMMH chains
whose filters run guided, replayed one filter at a time."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _states(model, n, steps=20, seed=9):
    """Particle states (n x 2, FP64, row-major) after `steps` unobserved days
    of the library's own PZ transition."""
    from libbi_b200 import BootstrapPF

    pf = BootstrapPF(model, n, seed=seed)
    for k in range(steps):
        pf.step(float(k), float(k + 1), None)
    x, _, _ = pf.state()
    xt = x[:, :n].T.contiguous().clone()
    pf.close()
    return xt


def test_pz_loss_and_gradient_match_oracle(cuda):
    import ctypes

    import torch
    from libbi_b200 import LearnedProposal, ModelPZ
    from libbi_b200 import _native as N
    from oracle.mlp_oracle import bf16, loss_grad

    prop = LearnedProposal(ModelPZ(), 1.0, max_batch=1024, seed=3)
    P, _, _ = prop.params()
    assert P.size == 128 * 3 + 128 + 128 * 128 + 128 + 2 * 128 + 2
    rng = np.random.default_rng(5)
    P = (P + 0.05 * rng.standard_normal(P.size)).astype(np.float32)
    prop.set_params(P)
    B = 777
    U = bf16(rng.standard_normal((B, 3)).astype(np.float32))
    r0 = (0.2 * rng.standard_normal((B, 1))).astype(np.float32)
    Ud = torch.as_tensor(U).to(torch.bfloat16).cuda()
    r0d = torch.as_tensor(r0).cuda()
    g = torch.zeros(P.size, dtype=torch.float32, device="cuda")
    loss = ctypes.c_double()
    N.check(N.lib().bpf_proposal_loss_grad(prop.handle, Ud.data_ptr(), r0d.data_ptr(), B, ctypes.byref(loss),
                                           g.data_ptr()), "bpf_proposal_loss_grad")
    want_loss, want_g = loss_grad(P, U, r0, d=1)
    np.testing.assert_allclose(loss.value, want_loss, rtol=1e-4)
    got = g.cpu().numpy().astype(np.float64)
    o = 0
    for n in (128 * 3, 128, 128 * 128, 128, 2 * 128, 2):
        a, b = got[o:o + n], want_g[o:o + n]
        assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b) + 1e-9, (o, np.linalg.norm(a - b), np.linalg.norm(b))
        o += n
    prop.close()


def test_pz_guided_step_matches_oracle(cuda, oracle):
    """One batched guided step of three filters from their initial states
    (no resampling at the first step) against orc_pz_guided_step fed the
    oracle network's outputs for the same inputs."""
    import torch
    from libbi_b200 import BatchedBootstrapPF, LearnedProposal, ModelPZ
    from oracle.mlp_oracle import forward_rows

    models = [ModelPZ(), ModelPZ(c=0.3, mu=math.log(0.25)), ModelPZ(sigma=0.3, sigma_y=0.1)]
    ns, seeds, dt = [300, 1024, 77], [41, 42, 43], 1.0
    prop = LearnedProposal(models[0], dt, max_batch=1024, seed=4)
    P, sh, sc = prop.params()
    rng = np.random.default_rng(7)
    P = (P + 0.05 * rng.standard_normal(P.size)).astype(np.float32)
    sh = np.array([0.7, 0.6, -0.1], np.float32)
    sc = np.array([4.0, 5.0, 3.0], np.float32)
    prop.set_params(P, sh, sc)
    b = BatchedBootstrapPF(models, ns, "systematic", seeds, ess_rel=0.5)
    b.set_proposal(prop)
    b.init()
    x0, lw0, _, offs = b.state()
    x0, lw0 = x0.cpu().numpy().copy(), lw0.cpu().numpy().copy()
    y = np.array([[0.9], [0.4], [0.6]])
    b.step_device(0.0, dt, torch.as_tensor(y).cuda())
    x1, lw1, _, _ = b.state()
    x1, lw1 = x1.cpu().numpy(), lw1.cpu().numpy()
    _, _, st = b.stats()
    assert (st == 0).all()
    for f, m in enumerate(models):
        n, o = ns[f], offs[f]
        xi = np.ascontiguousarray(x0[:, o:o + n])
        lp = np.log(xi[0])
        feats = np.stack([lp, np.log(xi[1]), y[f, 0] - lp], axis=1).astype(np.float32)
        delta, s = forward_rows(P, sh, sc, feats, d=1)
        xw, lww = oracle.pz_guided_step(m.desc(), xi, n, None, False, lw0[o:o + n], y[f, 0], 0.0, dt, seeds[f], 1,
                                        0.0, delta[:, 0].astype(np.float64), s[:, 0].astype(np.float64))
        dx = np.abs(x1[:, o:o + n] - xw) / np.abs(xw)
        assert np.median(dx) < 1e-5 and dx.max() < 1e-3, (f, np.median(dx), dx.max())
        dl = np.abs(lw1[o:o + n] - lww) / np.maximum(1.0, np.abs(lww))
        assert np.median(dl) < 1e-5 and dl.max() < 1e-3, (f, np.median(dl), dl.max())
    b.close()
    prop.close()


def _batch_lls(model, prop, y, n, seeds, dt):
    from libbi_b200 import BatchedBootstrapPF

    nf = len(seeds)
    b = BatchedBootstrapPF([model] * nf, [n] * nf, "systematic", seeds, ess_rel=0.5)
    if prop is not None:
        b.set_proposal(prop)
    yy = np.repeat(np.asarray(y, np.float64).reshape(-1, 1, 1), nf, axis=1)
    ll, _, _, st = b.filter(yy, 0.0, dt)
    b.close()
    assert (st == 0).all()
    return ll


def test_untrained_pz_proposal_gives_the_bootstrap_likelihood(cuda, oracle):
    """The untrained proposal is the prior N(mu, sigma) (zero output layer,
    s = log sigma): the same log-noise up to FP32 rounding of log sigma and
    a weight correction of rounding size."""
    from libbi_b200 import LearnedProposal, ModelPZ

    model = ModelPZ()
    T, dt, n = 20, 1.0, 512
    y, _ = oracle.simulate(model.desc(), 5, T, 0.0, dt)
    prop = LearnedProposal(model, dt, max_batch=1024, seed=2)
    seeds = list(range(500, 516))
    a = _batch_lls(model, None, y, n, seeds, dt)
    g = _batch_lls(model, prop, y, n, seeds, dt)
    assert np.median(np.abs(a - g)) < 1e-4, (a, g)
    prop.close()


def test_trained_pz_proposal_cuts_spread_on_informative_observations(cuda, oracle):
    """Observation noise sigma_y = 0.05 against a log-noise deviation of 0.5:
    y pins down each day's growth rate.  After training on simulated rows
    the loss falls well below the prior's, and the guided filter's
    log-likelihood spread over seeds is below the bootstrap filter's."""
    from libbi_b200 import LearnedProposal, ModelPZ

    model = ModelPZ(sigma=0.5, sigma_y=0.05)
    dt = 1.0
    prop = LearnedProposal(model, dt, max_batch=4096, seed=6)
    prop.set_states(_states(model, 1 << 16))
    trace = prop.train(1500, 4096, 2e-3)
    # prior loss: log 0.5 + 1/2 = -0.19; the posterior of log alpha given y
    # is several times narrower
    assert trace[:5].mean() > -0.3 and trace[-50:].mean() < trace[:5].mean() - 0.5, (trace[:5], trace[-50:])
    T, n = 12, 1024
    y, _ = oracle.simulate(model.desc(), 17, T, 0.0, dt)
    seeds = list(range(700, 724))
    boot = _batch_lls(model, None, y, n, seeds, dt)
    guid = _batch_lls(model, prop, y, n, seeds, dt)
    print("PZ ll spread over %d seeds: bootstrap %.4f, guided %.4f" % (len(seeds), boot.std(), guid.std()))
    assert np.isfinite(guid).all()
    assert guid.std() < 0.7 * boot.std(), (guid.std(), boot.std())
    # estimates are biased low by their variance: the guided mean is not below
    assert guid.mean() > boot.mean() - 2 * boot.std() / np.sqrt(len(boot))
    prop.close()


def test_pmmh_chains_with_guided_filters_replay(cuda, oracle):
    """PMMH with the proposal attached and per-chain particle counts: the
    chains' proposal log-likelihoods equal one-filter guided batches run
    with each proposal's parameters, seed and particle count."""
    from libbi_b200 import BatchedBootstrapPF, LearnedProposal, MarginalMH, ModelPZ, Prior

    T, dt = 15, 1.0
    truth = ModelPZ()
    y, _ = oracle.simulate(truth.desc(), 4, T, 0.0, dt)
    priors = [Prior(0, "uniform", 0.0, 1.0, 0.02), Prior(1, "uniform", 0.0, 1.0, 0.02),
              Prior(2, "log_normal", math.log(0.1), 0.5, 0.02), Prior(3, "log_normal", math.log(0.1), 0.5, 0.02)]
    C, seed, iters = 6, 13, 4
    ns = [1024, 1500, 2048, 3000, 4096, 8192]
    th0 = np.array([[0.25, 0.3, 0.1, 0.1]] * C)
    prop = LearnedProposal(truth, dt, max_batch=1024, seed=8)
    P, sh, sc = prop.params()
    rng = np.random.default_rng(3)
    prop.set_params((P + 0.03 * rng.standard_normal(P.size)).astype(np.float32), np.array([0.7, 0.6, 0.0],
                    np.float32), np.array([4.0, 5.0, 3.0], np.float32))
    mh = MarginalMH(truth, priors, y[:, 0], 0.0, dt, nchains=C, nparticles=ns, resampler="systematic",
                    ess_rel=0.5, seed=seed, theta0=th0)
    mh.set_proposal(prop)
    out = mh.run(iters)
    checked = 0
    for i in range(iters):
        r = i + 1
        for c in range(C):
            ll2 = out["proposal_loglik"][i, c]
            if not math.isfinite(ll2) or (i * C + c) % 3:
                continue
            z, _ = oracle.pmmh_draws(seed, c, r, 4)
            cur = out["samples"][i - 1, c] if i > 0 else th0[c]
            th = cur + np.array([q.step for q in priors]) * z
            m = ModelPZ(c=th[0], e=th[1], m=th[2], q=th[3])
            b = BatchedBootstrapPF([m], [ns[c]], "systematic", [seed + 1 + r * C + c], ess_rel=0.5)
            b.set_proposal(prop)
            ll, _, _, st = b.filter(np.asarray(y, np.float64).reshape(T, 1, 1), 0.0, dt)
            b.close()
            assert st[0] == 0
            np.testing.assert_allclose(ll2, ll[0], rtol=1e-12, atol=1e-12)
            checked += 1
    assert checked >= 4
    mh.set_proposal(None)
    mh.close()
    prop.close()
