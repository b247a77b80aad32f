"""Batched filters (bpf_batch_*, bpf_filter_batch) against single filters
(bpf_create / bpf_filter) with the same particle counts, resamplers, seeds
and constants: filter f of a batch draws what the single filter draws, so
log-likelihood increments, ESS and final states are bit-identical; the final
log-likelihood (BootstrapPF::term) agrees to reduction rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _singles(models, ns, res, seeds, ess_rel, B, y, dt):
    from libbi_b200 import BootstrapPF

    out = []
    for f, m in enumerate(models):
        pf = BootstrapPF(m, ns[f], resampler=res[f], ess_rel=ess_rel, seed=seeds[f], metropolis_steps=B)
        ll, inc, ess = pf.filter(y[:, f], 0.0, dt)
        x, lw, _ = pf.state()
        out.append((ll, inc, ess, x.cpu().numpy()[:, :ns[f]].copy(), lw.cpu().numpy().copy()))
        pf.close()
    return out


def _check(batch, singles, y, dt, ns):
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
    return ll, inc


def test_l96_batch_matches_single_filters(cuda, oracle):
    from libbi_b200 import BatchedBootstrapPF, ModelL96

    ns = [512, 700, 1024, 1, 3000, 4096, 2048]
    res = ["systematic", "multinomial", "metropolis", "systematic", "multinomial", "systematic", "metropolis"]
    seeds = [1000 + f for f in range(len(ns))]
    Fs = [6.0, 7.5, 8.0, 9.0, 10.0, 6.5, 8.5]
    models = [ModelL96(dim=40, F=F) for F in Fs]
    T, dt = 10, 0.05
    y = np.stack([oracle.simulate(m.desc(), 40 + f, T, 0.0, dt)[0] for f, m in enumerate(models)], axis=1)
    singles = _singles(models, ns, res, seeds, 0.5, 6, y, dt)
    batch = BatchedBootstrapPF(models, ns, res, seeds, ess_rel=0.5, metropolis_steps=6)
    ll1, inc1 = _check(batch, singles, y, dt, ns)
    # the captured graph replays to the same numbers
    ll2, inc2, _, _ = batch.filter(y, 0.0, dt)
    np.testing.assert_array_equal(inc1, inc2)
    np.testing.assert_array_equal(ll1, ll2)
    batch.close()


def test_pz_batch_matches_single_filters_and_theta_update(cuda, oracle):
    from libbi_b200 import BatchedBootstrapPF, ModelPZ

    ns = [1024, 2048, 777, 4096]
    res = ["systematic", "multinomial", "systematic", "metropolis"]
    seeds = [7, 8, 9, 10]
    models = [ModelPZ(c=0.25 + 0.02 * f, q=0.1 + 0.01 * f) for f in range(4)]
    T, dt = 12, 1.0
    y = np.stack([oracle.simulate(m.desc(), 90 + f, T, 0.0, dt)[0] for f, m in enumerate(models)], axis=1)
    singles = _singles(models, ns, res, seeds, 1.0, 5, y, dt)
    batch = BatchedBootstrapPF(models, ns, res, seeds, ess_rel=1.0, metropolis_steps=5)
    _check(batch, singles, y, dt, ns)
    # new constants through bpf_batch_set_theta, replayed graph
    models2 = [ModelPZ(c=0.3, e=0.25 + 0.01 * f, m=0.12) for f in range(4)]
    batch.set_theta([list(m.desc().theta) for m in models2])
    singles2 = _singles(models2, ns, res, seeds, 1.0, 5, y, dt)
    _check(batch, singles2, y, dt, ns)
    batch.close()


def test_batch_step_api_matches_filter(cuda, oracle):
    import torch
    from libbi_b200 import BatchedBootstrapPF, ModelL96

    ns = [600, 1500, 32768]
    models = [ModelL96(dim=40, F=8.0 + f) for f in range(3)]
    T, dt = 4, 0.05
    y = np.stack([oracle.simulate(m.desc(), 5 + f, T, 0.0, dt)[0] for f, m in enumerate(models)], axis=1)
    batch = BatchedBootstrapPF(models, ns, ["systematic", "multinomial", "systematic"], [1, 2, 3])
    ll, inc, _, _ = batch.filter(y, 0.0, dt)
    batch.init()
    yd = torch.as_tensor(y, device="cuda")
    for k in range(T):
        batch.step_device(k * dt, (k + 1) * dt, yd[k])
    ll2, _, st = batch.stats()
    assert (st == 0).all()
    np.testing.assert_array_equal(ll, ll2)
    batch.close()


def test_batch_rejects_bad_sizes(cuda):
    from libbi_b200 import BatchedBootstrapPF, BpfError, ModelL96

    with pytest.raises(BpfError):
        BatchedBootstrapPF([ModelL96(dim=40)], [32769])
    with pytest.raises(BpfError):
        BatchedBootstrapPF([ModelL96(dim=40)], [0])


def test_c3_shape_batch_matches_sampled_single_filters(cuda, oracle):
    """The batched configuration at its full shape: 256 Lorenz-96 filters,
    N log-uniform in [512, 32768] rounded to 32 (about 1.9 M particles),
    F_i ~ U(6, 10), systematic and multinomial alternating; a spread of the
    filters (smallest, largest and others) against single filters with the
    same settings, bit for bit over a short run."""
    from libbi_b200 import BatchedBootstrapPF, ModelL96

    rng = np.random.default_rng(3)
    nf = 256
    Fs = rng.uniform(6.0, 10.0, nf)
    ns = np.floor(np.exp(rng.uniform(np.log(512), np.log(32768), nf))).astype(int)
    ns = [int(v) for v in np.clip((ns + 31) // 32 * 32, 512, 32768)]
    models = [ModelL96(dim=40, F=float(F)) for F in Fs]
    res = ["systematic" if f % 2 == 0 else "multinomial" for f in range(nf)]
    seeds = [1000 + f for f in range(nf)]
    T, dt = 6, 0.05
    y = np.stack([oracle.simulate(m.desc(), 300 + f, T, 0.0, dt)[0] for f, m in enumerate(models)], axis=1)
    batch = BatchedBootstrapPF(models, ns, res, seeds, ess_rel=0.5)
    ll, inc, ess, st = batch.filter(y, 0.0, dt)
    assert (st == 0).all()
    x, lw, _, offs = batch.state()
    pick = sorted({int(np.argmin(ns)), int(np.argmax(ns)), 0, 1, 127, 255})
    models_p = [models[f] for f in pick]
    singles = _singles(models_p, [ns[f] for f in pick], [res[f] for f in pick], [seeds[f] for f in pick], 0.5, 0,
                       y[:, pick], dt)
    x, lw = x.cpu().numpy(), lw.cpu().numpy()
    for j, f in enumerate(pick):
        sll, sinc, sess, sx, slw = singles[j]
        np.testing.assert_array_equal(inc[:, f], sinc)
        np.testing.assert_array_equal(ess[:, f], sess)
        np.testing.assert_array_equal(x[:, offs[f]:offs[f] + ns[f]], sx)
        np.testing.assert_array_equal(lw[offs[f]:offs[f] + ns[f]], slw)
    batch.close()


def test_every_resampler_thread_count_gives_the_single_filters(cuda, oracle):
    """The batched resampler's CTA size is autotuned at create (256, 512 or
    1024 threads per filter); each count must give the single filters'
    numbers bit for bit."""
    from libbi_b200 import BatchedBootstrapPF, ModelL96

    ns = [512, 700, 4096, 32768, 1, 3000]
    res = ["systematic", "multinomial", "metropolis", "systematic", "multinomial", "metropolis"]
    seeds = [2000 + f for f in range(len(ns))]
    models = [ModelL96(dim=40, F=F) for F in (6.0, 7.0, 8.0, 9.0, 10.0, 8.5)]
    T, dt = 8, 0.05
    y = np.stack([oracle.simulate(m.desc(), 80 + f, T, 0.0, dt)[0] for f, m in enumerate(models)], axis=1)
    singles = _singles(models, ns, res, seeds, 0.5, 5, y, dt)
    batch = BatchedBootstrapPF(models, ns, res, seeds, ess_rel=0.5, metropolis_steps=5)
    tuned, us = batch.resample_threads()
    assert tuned in (256, 512, 1024) and all(v > 0 for v in us.values())
    for threads in (256, 512, 1024):
        assert batch.resample_threads(threads)[0] == threads
        _check(batch, singles, y, dt, ns)
    batch.close()



def test_c3_largest_filters_match_oracle(cuda, oracle):
    """The batched configuration's largest filters (32768 particles, one
    systematic and one multinomial, F = 6.5 and 9.5) over its T = 100,
    inside a batch with small filters, each directly against the oracle's
    filter with the same settings: increments, ESS and final states."""
    from libbi_b200 import BatchedBootstrapPF, ModelL96
    from libbi_b200 import _native as N

    ns = [32768, 512, 32768, 1000]
    res = ["systematic", "multinomial", "multinomial", "systematic"]
    seeds = [1000, 1001, 1002, 1003]
    models = [ModelL96(dim=40, F=F) for F in (6.5, 8.0, 9.5, 7.0)]
    T, dt = 100, 0.05
    y = np.stack([oracle.simulate(m.desc(), 500 + f, T, 0.0, dt)[0] for f, m in enumerate(models)], axis=1)
    batch = BatchedBootstrapPF(models, ns, res, seeds, ess_rel=0.5)
    ll, inc, ess, st = batch.filter(y, 0.0, dt)
    assert (st == 0).all()
    x, lw, _, offs = batch.state()
    x, lw = x.cpu().numpy(), lw.cpu().numpy()
    for f in (0, 2):
        cfg = N.Config()
        cfg.nparticles = ns[f]
        cfg.resampler = N.BPF_RESAMPLER_SYSTEMATIC if res[f] == "systematic" else N.BPF_RESAMPLER_MULTINOMIAL
        cfg.ess_rel = 0.5
        cfg.seed = seeds[f]
        want = oracle.filter(models[f].desc(), cfg, np.ascontiguousarray(y[:, f]), T, 0.0, dt)
        assert want["rc"] == 0 and want["resampled"].sum() > 0
        np.testing.assert_allclose(inc[:, f], want["inc"], rtol=1e-10, atol=1e-9)
        np.testing.assert_allclose(ess[:, f], want["ess"], rtol=1e-9)
        np.testing.assert_allclose(ll[f], want["ll"], rtol=1e-10)
        np.testing.assert_array_equal(x[:, offs[f]:offs[f] + ns[f]], want["x"][:, :ns[f]])
        np.testing.assert_allclose(lw[offs[f]:offs[f] + ns[f]], want["lw"], rtol=1e-12)
    batch.close()
