"""Sparse observations (bpf_step_sparse, the observation Mask) and the
Schedule/Observer driver: the masked transition bit-identical to the
oracle's, a dense regular schedule identical to bpf_filter, and an irregular
sparse schedule against a filter loop written over the oracle's
primitives (transition with mask, systematic resampling, ESS reduction)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["l96_f32", "pz"])
def test_masked_step_bit_identical_to_oracle(cuda, oracle, which):
    from libbi_b200 import BootstrapPF, ModelL96, ModelPZ

    model = ModelL96(dim=40) if which == "l96_f32" else ModelPZ()
    n, seed = 1500, 12
    dt = 0.05 if which == "l96_f32" else 1.0
    desc = model.desc()
    y, _ = oracle.simulate(desc, 3, 1, 0.0, dt)
    idx = np.array([3, 17, 0, 39, 22, 8] if which == "l96_f32" else [0], dtype=np.int32)
    mask = 0
    for i in idx:
        mask |= 1 << int(i)
    pf = BootstrapPF(model, n, seed=seed)
    x0, lw0, _ = pf.state()
    x0, lw0 = x0.cpu().numpy().copy(), lw0.cpu().numpy().copy()
    pf.step_sparse(0.0, dt, y[0][idx], idx)
    x1, lw1, _ = pf.state()
    ydense = np.zeros(model.nobs, dtype=model.np_dtype)
    ydense[idx] = y[0][idx]
    wx, wlw = oracle.transition_mask(desc, x0, n, None, False, lw0, ydense, 0.0, dt, seed, 1, 0.0, mask)
    np.testing.assert_array_equal(x1.cpu().numpy()[:, :n], wx[:, :n])
    np.testing.assert_array_equal(lw1.cpu().numpy(), wlw)
    pf.close()


def test_dense_schedule_equals_filter(cuda, oracle):
    from libbi_b200 import BootstrapPF, ModelL96
    from libbi_b200.schedule import Observer, Schedule

    model = ModelL96(dim=40)
    T, dt, n = 8, 0.05, 2048
    y, _ = oracle.simulate(model.desc(), 4, T, 0.0, dt)
    times = np.repeat(dt * np.arange(1, T + 1), 40)
    coords = np.tile(np.arange(40), T)
    obs = Observer(times, coords, y.reshape(-1))
    pf = BootstrapPF(model, n, seed=5)
    ll, inc, ess = pf.filter(y, 0.0, dt)
    out = Schedule(0.0, dt, obs).run(pf)
    np.testing.assert_array_equal(out["log_increments"], inc)
    np.testing.assert_array_equal(out["ess"], ess)
    np.testing.assert_allclose(out["loglik"], ll, rtol=1e-12)
    pf.close()


def test_sparse_schedule_against_oracle_loop(cuda, oracle):
    from libbi_b200 import BootstrapPF, ModelL96
    from libbi_b200.schedule import Observer, Schedule

    model = ModelL96(dim=40)
    desc = model.desc()
    dt, n, seed, ess_rel = 0.05, 1024, 6, 0.5
    ytrue, _ = oracle.simulate(desc, 8, 14, 0.0, dt)
    rng = np.random.default_rng(2)
    times, coords, vals = [], [], []
    for k in (1, 2, 4, 5, 6, 9, 10, 11, 14):  # irregular observation times
        comps = np.sort(rng.choice(40, size=int(rng.integers(5, 41)), replace=False))
        times += [k * dt] * comps.size
        coords += list(comps)
        vals += list(ytrue[k - 1][comps])
    obs = Observer(times, coords, vals)
    sched = Schedule(0.0, dt, obs, output_times=[16 * dt])
    pf = BootstrapPF(model, n, ess_rel=ess_rel, seed=seed)
    out = sched.run(pf)
    x_gpu, lw_gpu, _ = pf.state()

    # the same run on the oracle's primitives
    x, lw = oracle.init(desc, n, seed)
    ll, resample_next, incs, step = 0.0, False, [], 0
    for prev, el in zip(sched.elements[:-1], sched.elements[1:]):
        step += 1
        as_, resampled = None, False
        if resample_next:
            a = oracle.resample_uniforms(0, n, 0, seed, step)[0]
            rc, _, _, as_ = oracle.systematic(lw, a, permute=True)
            assert rc == 0
            resampled = True
        ydense, mask = None, 0
        if el.observed:
            idx, v = obs.get(el.index_obs)
            ydense = np.zeros(40, np.float32)
            ydense[idx] = v
            for i in idx:
                mask |= 1 << int(i)
        x, lw = oracle.transition_mask(desc, x, n, as_, resampled, lw, ydense, prev.time, el.time, seed, step, ll,
                                       mask)
        if el.observed:
            ess, lW = oracle.ess_reduce(lw)
            incs.append(lW - ll)
            ll = lW
            resample_next = ess < ess_rel * n
        else:
            resample_next = False
    np.testing.assert_allclose(out["log_increments"], incs, rtol=1e-10, atol=1e-9)
    np.testing.assert_array_equal(x_gpu.cpu().numpy()[:, :n], x[:, :n])
    assert out["resampled"].any()
    pf.close()
