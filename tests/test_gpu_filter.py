"""The fused CUDA transition and the whole filter against the oracle, on the
same draws: states and log-weights bit-identical, log-likelihoods equal to
reduction rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mk(model, n, resampler="systematic", ess_rel=0.5, seed=3, B=0):
    from libbi_b200 import BootstrapPF

    return BootstrapPF(model, n, resampler=resampler, ess_rel=ess_rel, seed=seed, metropolis_steps=B)


def _cfg(pf):
    return pf._cfg


@pytest.mark.parametrize("which", ["l96_f32", "l96_f64", "pz"])
def test_first_step_bit_identical(cuda, oracle, which):
    from libbi_b200 import ModelL96, ModelPZ

    model = {"l96_f32": ModelL96(dim=40), "l96_f64": ModelL96(dim=40, precision="f64"), "pz": ModelPZ()}[which]
    n = 3000
    pf = _mk(model, n)
    desc = model.desc()
    x0, lw0 = oracle.init(desc, n, pf._cfg.seed)
    x, lw, _ = pf.state()
    np.testing.assert_array_equal(x.cpu().numpy()[:, :n], x0[:, :n])
    np.testing.assert_array_equal(lw.cpu().numpy(), lw0)
    dt = 0.05 if model.dim == 40 else 1.0
    y, _ = oracle.simulate(desc, 11, 3, 0.0, dt)
    res = pf.step(0.0, dt, y[0])
    x1, lw1 = oracle.transition(desc, x0, n, None, False, lw0, y[0], 0.0, dt, pf._cfg.seed, 1, 0.0)
    x, lw, _ = pf.state()
    np.testing.assert_array_equal(x.cpu().numpy()[:, :n], x1[:, :n])
    np.testing.assert_array_equal(lw.cpu().numpy(), lw1)
    ess, lW = oracle.ess_reduce(lw1)
    np.testing.assert_allclose(res.ess, ess, rtol=1e-12)
    np.testing.assert_allclose(res.log_likelihood, lW, rtol=1e-12)


@pytest.mark.parametrize("resampler,B", [("systematic", 0), ("multinomial", 0), ("metropolis", 8)])
@pytest.mark.parametrize("which", ["l96", "l96_grid", "pz"])
def test_filter_matches_oracle(cuda, oracle, resampler, B, which):
    """Filters of up to 4096 particles resample in one CTA; l96_grid (8192
    particles) takes the grid-wide resamplers."""
    from libbi_b200 import ModelL96, ModelPZ

    if which == "l96":
        model, n, T, dt, ess_rel = ModelL96(dim=40), 2048, 12, 0.05, 0.5
    elif which == "l96_grid":
        model, n, T, dt, ess_rel = ModelL96(dim=40), 8192, 8, 0.05, 0.5
    else:
        model, n, T, dt, ess_rel = ModelPZ(), 1024, 15, 1.0, 1.0
    desc = model.desc()
    y, _ = oracle.simulate(desc, 21, T, 0.0, dt)
    pf = _mk(model, n, resampler, ess_rel, seed=9, B=B)
    ll, inc, ess = pf.filter(y, 0.0, dt)
    want = oracle.filter(desc, pf._cfg, y, T, 0.0, dt)
    assert want["rc"] == 0
    assert want["resampled"].sum() > 0
    np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(ess, want["ess"], rtol=1e-9)
    np.testing.assert_allclose(ll, want["ll"], rtol=1e-10)
    x, lw, _ = pf.state()
    np.testing.assert_array_equal(x.cpu().numpy()[:, :n], want["x"][:, :n])
    np.testing.assert_allclose(lw.cpu().numpy(), want["lw"], rtol=1e-12)


def test_pz_config_c1_matches_oracle(cuda, oracle):
    """The PZ configuration at its own sizes: N = 4096, FP64, RK4(3),
    systematic resampling at every step (essRel = 1), T = 100 daily
    observations from a seeded model run; every increment, the ESS, the
    log-likelihood and the final state against the oracle's FP64 filter."""
    from libbi_b200 import ModelPZ

    model, n, T, dt = ModelPZ(), 4096, 100, 1.0
    desc = model.desc()
    y, _ = oracle.simulate(desc, 1, T, 0.0, dt)
    pf = _mk(model, n, "systematic", 1.0, seed=2)
    ll, inc, ess = pf.filter(y, 0.0, dt)
    want = oracle.filter(desc, pf._cfg, y, T, 0.0, dt)
    assert want["rc"] == 0
    assert want["resampled"].sum() >= T - 1
    np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(ess, want["ess"], rtol=1e-9)
    np.testing.assert_allclose(ll, want["ll"], rtol=1e-10)
    x, _, _ = pf.state()
    np.testing.assert_array_equal(x.cpu().numpy()[:, :n], want["x"][:, :n])
    pf.close()


def test_l96_config_c2_matches_oracle(cuda, oracle):
    """The benchmarked Lorenz-96 configuration at its own size: d = 40,
    N = 65536 FP32 particles, RK4 h = 0.01, observations of all 40
    components with N(0, 1) noise every 0.05, systematic resampling at
    ESS < 0.5 N, T = 200, on the bench's synthetic observations (one model
    run from the data seed, observed with N(0, 1) noise from a numpy
    generator on the same seed); every increment, the ESS, the
    log-likelihood and the final state against the oracle's filter."""
    from libbi_b200 import ModelL96

    model, n, T, dt = ModelL96(dim=40), 65536, 200, 0.05
    desc = model.desc()
    _, xs = oracle.simulate(desc, 102, T, 0.0, dt)
    y = (xs + model.sigma_y * np.random.default_rng(102).standard_normal(xs.shape)).astype(np.float32)
    pf = _mk(model, n, "systematic", 0.5, seed=2)
    ll, inc, ess = pf.filter(y, 0.0, dt)
    want = oracle.filter(desc, pf._cfg, y, T, 0.0, dt)
    assert want["rc"] == 0
    assert want["resampled"].sum() >= T // 2
    np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(ess, want["ess"], rtol=1e-9)
    np.testing.assert_allclose(ll, want["ll"], rtol=1e-10)
    x, lw, _ = pf.state()
    np.testing.assert_array_equal(x.cpu().numpy()[:, :n], want["x"][:, :n])
    np.testing.assert_allclose(lw.cpu().numpy(), want["lw"], rtol=1e-12)
    pf.close()


def test_handle_reused_across_runs_and_restores(cuda, oracle):
    """One handle, several filter runs on different observations, with a
    snapshot restored in between: every run equals the oracle's filter.  The
    one-launch resampler (N = 65536: several blocks handing over through
    published words) reuses its scratch from run to run; the words of earlier
    launches must never be taken for the current one's."""
    from libbi_b200 import ModelL96

    model, n, T, dt = ModelL96(dim=40), 65536, 12, 0.05
    desc = model.desc()
    pf = _mk(model, n, "systematic", 1.0, seed=8)
    snap = None
    for r, dseed in enumerate((31, 32, 33)):
        y, _ = oracle.simulate(desc, dseed, T, 0.0, dt)
        ll, inc, _ = pf.filter(y, 0.0, dt)
        want = oracle.filter(desc, pf._cfg, y, T, 0.0, dt)
        assert want["rc"] == 0 and want["resampled"].sum() >= T - 1
        np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
        x, _, _ = pf.state()
        np.testing.assert_array_equal(x.cpu().numpy()[:, :n], want["x"][:, :n])
        if r == 0:
            snap = pf.snapshot()
        elif r == 1:
            pf.restore(snap)
    pf.close()


def test_step_api_and_snapshot(cuda, oracle):
    from libbi_b200 import ModelL96

    model = ModelL96(dim=40)
    n, dt = 4096, 0.05
    y, _ = oracle.simulate(model.desc(), 5, 8, 0.0, dt)
    pf = _mk(model, n, seed=4)
    steps = [pf.step(k * dt, (k + 1) * dt, y[k]) for k in range(4)]
    blob = pf.snapshot()
    rest = [pf.step(k * dt, (k + 1) * dt, y[k]) for k in range(4, 8)]
    pf.restore(blob)
    again = [pf.step(k * dt, (k + 1) * dt, y[k]) for k in range(4, 8)]
    for a, b in zip(rest, again):
        assert a == b
    # step-by-step equals the whole-filter call
    pf2 = _mk(model, n, seed=4)
    ll, inc, ess = pf2.filter(y, 0.0, dt)
    np.testing.assert_array_equal(inc, np.array([s.log_increment for s in steps + rest]))
    assert sum(s.resampled for s in steps + rest) >= 1


def test_unobserved_steps(cuda, oracle):
    from libbi_b200 import ModelL96

    model = ModelL96(dim=8)
    pf = _mk(model, 1000, seed=2)
    r = pf.step(0.0, 0.05, None)
    assert r.log_likelihood == 0.0 and not r.resampled
    _, lw, _ = pf.state()
    assert float(lw.abs().max()) == 0.0


@pytest.mark.parametrize("which", ["pz", "pz_metropolis", "l96_multinomial", "l96_one_launch", "l96_large"])
def test_repeated_filter_calls_replay_the_same_steps(cuda, oracle, which):
    """bpf_filter runs a repeated schedule as a CUDA graph from the second
    call on (captured then, replayed after): every call equals the oracle's
    filter of its observations, and a call with another schedule in between
    runs directly and leaves the captured steps in place."""
    from libbi_b200 import ModelL96, ModelPZ

    if which == "pz":
        model, n, T, dt, res, ess_rel = ModelPZ(), 1024, 15, 1.0, "systematic", 1.0
    elif which == "pz_metropolis":
        model, n, T, dt, res, ess_rel = ModelPZ(), 2048, 12, 1.0, "metropolis", 1.0
    elif which == "l96_multinomial":
        model, n, T, dt, res, ess_rel = ModelL96(dim=40), 8192, 8, 0.05, "multinomial", 0.5
    elif which == "l96_one_launch":
        model, n, T, dt, res, ess_rel = ModelL96(dim=40), 4096, 8, 0.05, "systematic", 1.0
    else:
        model, n, T, dt, res, ess_rel = ModelL96(dim=40), 65536, 6, 0.05, "systematic", 1.0
    desc = model.desc()
    pf = _mk(model, n, res, ess_rel, seed=14, B=8 if res == "metropolis" else 0)
    if which == "l96_one_launch":
        pf.set_step_form(True)
    runs = [oracle.simulate(desc, dseed, T, 0.0, dt)[0] for dseed in (81, 82, 83, 84)]
    short, _ = oracle.simulate(desc, 85, T - 2, 0.0, dt)
    for r, y in enumerate(runs):
        if r == 3:
            pf.filter(short, 0.0, dt)  # another schedule: run directly
        ll, inc, ess = pf.filter(y, 0.0, dt)
        want = oracle.filter(desc, pf._cfg, y, T, 0.0, dt)
        assert want["rc"] == 0
        np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
        np.testing.assert_allclose(ess, want["ess"], rtol=1e-9)
        np.testing.assert_allclose(ll, want["ll"], rtol=1e-10)
        x, _, _ = pf.state()
        np.testing.assert_array_equal(x.cpu().numpy()[:, :n], want["x"][:, :n])
    pf.close()


@pytest.mark.parametrize("one_launch", [True, False])
def test_filter_graph_after_a_timed_out_run(cuda, oracle, one_launch):
    """Whole-filter calls under a wait limit that makes every hand-over give
    up report BPF_E_TIMEOUT (the second such call captures its steps as a
    graph); with the default limit back, the next calls of the same
    schedule run again correctly: the limit a capture was made under is
    part of what a replay must match."""
    from libbi_b200 import BpfError, ModelL96
    from libbi_b200 import _native as N

    model = ModelL96(dim=40)
    desc = model.desc()
    n, T, dt = 65536, 5, 0.05
    y, _ = oracle.simulate(desc, 91, T, 0.0, dt)
    pf = _mk(model, n, "systematic", 1.0, seed=19)
    pf.set_step_form(one_launch)
    try:
        assert N.lib().bpf_debug_set_wait_limit(-1) == N.BPF_OK
        for _ in range(2):
            with pytest.raises(BpfError) as e:
                pf.filter(y, 0.0, dt)
            assert e.value.status == N.BPF_E_TIMEOUT
    finally:
        N.lib().bpf_debug_set_wait_limit(N.BPF_WAIT_LIMIT_DEFAULT)
    want = oracle.filter(desc, pf._cfg, y, T, 0.0, dt)
    assert want["rc"] == 0
    for _ in range(3):
        ll, inc, ess = pf.filter(y, 0.0, dt)
        np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
        x, _, _ = pf.state()
        np.testing.assert_array_equal(x.cpu().numpy()[:, :n], want["x"][:, :n])
    pf.close()
