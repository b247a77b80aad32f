"""CUDA resamplers and reductions against the oracle (and the reference's
golden vectors): ancestors bit-exact on the same log-weights and uniforms."""
import numpy as np
import pytest

from tests.golden.make_golden import UNIFORM_SEED

pytestmark = pytest.mark.gpu


def _t(a, dtype=None):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a), device="cuda", dtype=dtype)


def _resamplers(maxn=1 << 16, B=0):
    from libbi_b200 import SystematicResampler, MultinomialResampler, MetropolisResampler

    return SystematicResampler(max_n=maxn), MultinomialResampler(max_n=maxn), MetropolisResampler(max_n=maxn, B=B)


def _uniforms(oracle, kind, n, B, step):
    return oracle.resample_uniforms(kind, n, B, UNIFORM_SEED, step)


def _near_tie_ok(oracle, lw, a, got_Os, want_Os):
    """Mismatches of cumulative offspring are allowed only where the oracle's
    Ws/W*n + a lies within 1e-9 of an integer (a rounding tie)."""
    bad = np.nonzero(got_Os != want_Os)[0]
    if bad.size == 0:
        return True
    _, Ws, _, _ = oracle.systematic(lw, a)
    r = Ws[bad] / Ws[-1] * lw.size + a
    return bool(np.all(np.abs(r - np.round(r)) < 1e-9))


def test_golden_all_resamplers(cuda, oracle, golden):
    import torch

    sysr, mult, _ = _resamplers()
    from libbi_b200 import MetropolisResampler

    for name, c in golden.items():
        lw = c["lw"]
        n = lw.size
        lw_d = _t(lw, torch.float64)
        step = int(c["step"][0])
        # systematic: cumulative offspring, permuted and sorted ancestors
        a = _uniforms(oracle, 0, n, 0, step)
        perm, Os = sysr.ancestors(lw_d, _t(a, torch.float64), permute=True, with_offspring=True)
        Os = Os.cpu().numpy()
        assert _near_tie_ok(oracle, lw, a[0], Os, c["Os"].astype(np.int32)), name
        np.testing.assert_array_equal(Os, c["Os"], err_msg=name)
        np.testing.assert_array_equal(perm.cpu().numpy(), c["sys_perm"], err_msg=name)
        srt = sysr.ancestors(lw_d, _t(a, torch.float64), permute=False)
        np.testing.assert_array_equal(srt.cpu().numpy(), c["sys_sorted"], err_msg=name)
        # multinomial: sorted draws bit-exact; permuted form by the path's rule
        u = _uniforms(oracle, 1, n, 0, step)
        m = mult.ancestors(lw_d, _t(u, torch.float64), permute=False).cpu().numpy()
        np.testing.assert_array_equal(m, c["mult"], err_msg=name)
        mp = mult.ancestors(lw_d, _t(u, torch.float64), permute=True).cpu().numpy()
        np.testing.assert_array_equal(mp, oracle.permute_rule(c["mult"]), err_msg=name)
        # Metropolis with the harness's B
        B = int(c["B"][0])
        mh = MetropolisResampler(max_n=1 << 16, B=B)
        u = _uniforms(oracle, 2, n, B, step)
        g = mh.ancestors(lw_d, _t(u, torch.float64), permute=False).cpu().numpy()
        np.testing.assert_array_equal(g, c["metro"], err_msg=name)
        gp = mh.ancestors(lw_d, _t(u, torch.float64), permute=True).cpu().numpy()
        np.testing.assert_array_equal(gp, oracle.permute_rule(c["metro"]), err_msg=name)
        mh.close()


def test_golden_reductions(cuda, golden):
    import torch

    sysr, _, _ = _resamplers()
    for name, c in golden.items():
        ess, lW = sysr.reduce(_t(c["lw"], torch.float64))
        if np.isnan(c["ess"][0]):
            assert np.isnan(ess), name
        else:
            np.testing.assert_allclose(ess, c["ess"][0], rtol=1e-12, err_msg=name)
        np.testing.assert_allclose(lW, c["lW"][0], rtol=1e-12, atol=1e-12, err_msg=name)
        lse = sysr.logsumexp(_t(c["lw"], torch.float64))
        np.testing.assert_allclose(lse, c["lse"][0], rtol=1e-12, atol=1e-12, err_msg=name)


@pytest.mark.parametrize("n", [1, 2, 31, 2047, 2048, 2049, 6144, 65536, 100003])
def test_random_sizes_systematic_and_multinomial(cuda, oracle, n):
    import torch

    sysr, mult, _ = _resamplers(maxn=1 << 17)
    rng = np.random.default_rng(n)
    for scale in (0.1, 3.0, 40.0):
        lw = rng.standard_normal(n) * scale
        lw_d = _t(lw, torch.float64)
        a = rng.random(1)
        perm, Os = sysr.ancestors(lw_d, _t(a, torch.float64), permute=True, with_offspring=True)
        rc, _, Os_o, perm_o = oracle.systematic(lw, a[0], permute=True)
        assert _near_tie_ok(oracle, lw, a[0], Os.cpu().numpy(), Os_o)
        np.testing.assert_array_equal(perm.cpu().numpy(), perm_o)
        u = rng.random(n)
        m = mult.ancestors(lw_d, _t(u, torch.float64), permute=False).cpu().numpy()
        np.testing.assert_array_equal(m, oracle.multinomial(lw, u, 0)[1])


def test_degenerate_raises(cuda):
    import torch
    from libbi_b200 import ParticleFilterDegeneratedException

    sysr, mult, _ = _resamplers()
    lw = torch.full((1000,), float("-inf"), dtype=torch.float64, device="cuda")
    with pytest.raises(ParticleFilterDegeneratedException):
        sysr.ancestors(lw, _t(np.array([0.5]), torch.float64))
    with pytest.raises(ParticleFilterDegeneratedException):
        mult.ancestors(lw, _t(np.full(1000, 0.5), torch.float64))
    lw = torch.full((1000,), float("nan"), dtype=torch.float64, device="cuda")
    with pytest.raises(ParticleFilterDegeneratedException):
        sysr.ancestors(lw, _t(np.array([0.5]), torch.float64))
    # the resampler recovers for the next call
    ok = torch.zeros(1000, dtype=torch.float64, device="cuda")
    a = sysr.ancestors(ok, _t(np.array([0.5]), torch.float64), permute=True)
    np.testing.assert_array_equal(a.cpu().numpy(), np.arange(1000))


def test_large_n_properties(cuda):
    """At 2^22 particles (beyond L2): offspring sum to n, survivors in place,
    unpermuted ancestors sorted, cumulative offspring monotone ending at n."""
    import torch

    n = 1 << 22
    from libbi_b200 import SystematicResampler, MultinomialResampler

    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    lw = torch.randn(n, dtype=torch.float64, device="cuda", generator=g) * 2
    for R in (SystematicResampler(max_n=n), MultinomialResampler(max_n=n)):
        u = torch.rand(n, dtype=torch.float64, device="cuda", generator=g).clamp_(1e-12, 1 - 1e-12)
        srt = R.ancestors(lw, u[:1] if isinstance(R, SystematicResampler) else u, permute=False)
        assert bool((srt[1:] >= srt[:-1]).all())
        assert int(srt.min()) >= 0 and int(srt.max()) < n
        perm, Os = R.ancestors(lw, u[:1] if isinstance(R, SystematicResampler) else u, permute=True,
                               with_offspring=True)
        o = torch.bincount(perm.long(), minlength=n)
        assert int(o.sum()) == n
        assert bool((Os[1:] >= Os[:-1]).all()) and int(Os[-1]) == n
        surv = o > 0
        idx = torch.arange(n, device="cuda")
        assert bool((perm.long()[surv] == idx[surv]).all())
        np.testing.assert_array_equal(torch.bincount(srt.long(), minlength=n).cpu().numpy(), o.cpu().numpy())
        R.close()


def test_gather_rows(cuda, oracle):
    import torch
    from libbi_b200 import gather_rows

    rng = np.random.default_rng(5)
    for n, d, dt in ((1, 1, np.float32), (1000, 40, np.float32), (4099, 3, np.float64)):
        ld = (n + 31) // 32 * 32
        X = rng.standard_normal((d, ld)).astype(dt)
        as_ = rng.integers(0, n, n).astype(np.int32)
        Y = torch.zeros((d, ld), dtype=torch.float32 if dt == np.float32 else torch.float64, device="cuda")
        gather_rows(_t(as_), _t(X), Y, d, ld)
        want = np.zeros_like(X)
        oracle.L.orc_gather(as_.ctypes.data, X.ctypes.data, want.ctypes.data, n, d, ld, X.itemsize)
        np.testing.assert_array_equal(Y.cpu().numpy()[:, :n], want[:, :n])


@pytest.mark.parametrize("n", [700001, 1300000])
def test_systematic_multi_tile_matches_oracle(cuda, oracle, n):
    """Sizes beyond one 512-tile per resident block take the multi-tile
    cooperative kernel; ancestors must still equal the oracle's."""
    import torch
    from libbi_b200 import SystematicResampler

    rng = np.random.default_rng(n)
    lw = rng.standard_normal(n) * 3.0
    a = rng.random(1)
    R = SystematicResampler(max_n=n)
    perm, Os = R.ancestors(_t(lw, torch.float64), _t(a, torch.float64), permute=True, with_offspring=True)
    rc, _, Os_o, perm_o = oracle.systematic(lw, a[0], permute=True)
    assert rc == 0
    assert _near_tie_ok(oracle, lw, a[0], Os.cpu().numpy(), Os_o)
    np.testing.assert_array_equal(perm.cpu().numpy(), perm_o)
    ess, lW = R.reduce(_t(lw, torch.float64))
    ess_o, lW_o = oracle.ess_reduce(lw)
    np.testing.assert_allclose([ess, lW], [ess_o, lW_o], rtol=1e-11)
    R.close()


@pytest.mark.parametrize("n", [700, 2049, 65536, 100003])
def test_every_tile_shape_gives_the_oracles_ancestors(cuda, oracle, n):
    """The one-launch systematic kernel in each of its tile shapes (threads
    per block x particles per thread) computes the same integers: the
    autotuner may pick any of them."""
    import torch
    from libbi_b200 import SystematicResampler
    from libbi_b200._native import RESAMPLE_SHAPES

    rng = np.random.default_rng(7 * n)
    lw = rng.standard_normal(n) * 3.0
    a = rng.random(1)
    rc, _, Os_o, perm_o = oracle.systematic(lw, a[0], permute=True)
    assert rc == 0
    R = SystematicResampler(max_n=n)
    for k in range(RESAMPLE_SHAPES):
        R.set_shape(k)
        perm, Os = R.ancestors(_t(lw, torch.float64), _t(a, torch.float64), permute=True, with_offspring=True)
        assert _near_tie_ok(oracle, lw, a[0], Os.cpu().numpy(), Os_o), k
        np.testing.assert_array_equal(perm.cpu().numpy(), perm_o, err_msg=f"shape {k}")
    R.close()


def test_autotune_picks_a_timed_shape(cuda):
    from libbi_b200 import autotune_resampler
    from libbi_b200._native import RESAMPLE_SHAPES
    from libbi_b200.filter import RESAMPLE_SHAPES as SHAPES

    best, us = autotune_resampler(65536)
    assert 0 <= best < RESAMPLE_SHAPES
    assert SHAPES[best] in us and us[SHAPES[best]] == min(us.values())
    assert len(us) >= 2 and all(v > 0 for v in us.values())


def _harness_lw(z, P, x):
    """The reference harness's log-weights (test_resampler_cpu.cpp.tt:120-136):
    log N(x; 0, 1) of standard normals x shifted by 0.5 per Z step."""
    xs = x[:P] + 0.5 * z
    return -0.5 * xs * xs - 0.91893853320467274178


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_resampler_harness_metrics(cuda, oracle, kind):
    """The metrics of the reference's resampler harness
    (test_resampler_cpu.cpp.tt:199-245): over REPS resamplings, bias^2 =
    sum_i (mean offspring_i - P w_i)^2 and the trace of the offspring
    variance, per Z and P.  With the same uniforms the GPU and the oracle give
    the same offspring, so the same metrics; and the statistics behave: bias^2
    is Monte Carlo noise of the unbiased resamplers (about tr_var / REPS),
    systematic has the smallest variance."""
    import torch
    from libbi_b200 import MetropolisResampler, MultinomialResampler, SystematicResampler

    reps = 120
    x = np.random.default_rng(11).standard_normal(4096)
    out = {}
    for z in (0, 2, 4):
        for P in (16, 256, 4096):
            lw = _harness_lw(z, P, x)
            w = np.exp(lw - lw.max())
            ws = P * w / w.sum()
            if kind == 2:
                # the harness's B for a 1% bias bound at this Z
                Z = 0.5 * z
                EW = np.exp(-0.25 * Z * Z) / (2.0 * np.sqrt(np.pi))
                beta = EW / (1.0 / np.sqrt(np.pi))
                B = int(np.ceil(np.log(1e-2) / np.log(1.0 - beta)))
            else:
                B = 0
            R = (SystematicResampler, MultinomialResampler, lambda max_n: MetropolisResampler(max_n=max_n, B=B))[kind](
                max_n=P)
            lw_d = _t(lw, torch.float64)
            O_gpu = np.zeros((reps, P))
            O_orc = np.zeros((reps, P))
            for r in range(reps):
                u = _uniforms(oracle, kind, P, B, 1000 + r)
                a = R.ancestors(lw_d, _t(u, torch.float64), permute=False).cpu().numpy()
                O_gpu[r] = np.bincount(a, minlength=P)
                if kind == 0:
                    want = oracle.systematic(lw, u[0], permute=False)[3]
                elif kind == 1:
                    want = oracle.multinomial(lw, u, 0)[1]
                else:
                    want = oracle.metropolis(lw, B, u, 0)[1]
                O_orc[r] = np.bincount(want, minlength=P)
            R.close()
            metrics = []
            for O in (O_gpu, O_orc):
                mu, var = O.mean(0), O.var(0, ddof=1)
                metrics.append((float(((mu - ws) ** 2).sum()), float(var.sum())))
            assert metrics[0] == metrics[1], (z, P, metrics)
            bias2, tr_var = metrics[0]
            out[(z, P)] = (bias2, tr_var)
            if kind in (0, 1):  # unbiased: E[bias^2] = tr_var / reps
                assert bias2 <= 3.0 * tr_var / reps + 1e-9, (z, P, bias2, tr_var)
    if kind == 0:
        # systematic resampling's trace variance stays below multinomial's (P (1 - sum w^2) at most)
        for (z, P), (_, tv) in out.items():
            lw = _harness_lw(z, P, x)
            w = np.exp(lw - lw.max())
            w /= w.sum()
            assert tv <= P * (1.0 - (w * w).sum()) + 1e-9, (z, P, tv)
