"""The oracle restatement against the reference's own code: golden vectors
made by the reference's compiled resampler (tests/golden/make_golden.py), and,
where the reference build is present, random cases run through it live."""
import numpy as np
import pytest

from tests.golden.make_golden import UNIFORM_SEED


def _uniforms(oracle, case, kind):
    n = case["lw"].size
    return oracle.resample_uniforms(kind, n, int(case["B"][0]), UNIFORM_SEED, int(case["step"][0]))


def test_golden_systematic(oracle, golden):
    for name, c in golden.items():
        a = _uniforms(oracle, c, 0)[0]
        rc, Ws, Os, perm = oracle.systematic(c["lw"], a, permute=True)
        assert rc == 0
        np.testing.assert_array_equal(Os, c["Os"], err_msg=name)
        np.testing.assert_array_equal(perm, c["sys_perm"], err_msg=name)
        _, _, _, srt = oracle.systematic(c["lw"], a, permute=False)
        np.testing.assert_array_equal(srt, c["sys_sorted"], err_msg=name)


def test_golden_multinomial(oracle, golden):
    for name, c in golden.items():
        u = _uniforms(oracle, c, 1)
        np.testing.assert_array_equal(oracle.multinomial(c["lw"], u, 0)[1], c["mult"], err_msg=name)
        np.testing.assert_array_equal(oracle.multinomial(c["lw"], u, 2)[1], c["mult_refperm"], err_msg=name)


def test_golden_metropolis(oracle, golden):
    for name, c in golden.items():
        u = _uniforms(oracle, c, 2)
        B = int(c["B"][0])
        np.testing.assert_array_equal(oracle.metropolis(c["lw"], B, u, 0)[1], c["metro"], err_msg=name)
        np.testing.assert_array_equal(oracle.metropolis(c["lw"], B, u, 2)[1], c["metro_refperm"], err_msg=name)


def test_golden_reductions(oracle, golden):
    for name, c in golden.items():
        ess, lW = oracle.ess_reduce(c["lw"])
        assert ess == c["ess"][0] or (np.isnan(ess) and np.isnan(c["ess"][0])), name
        assert lW == c["lW"][0], name
        assert oracle.logsumexp(c["lw"]) == c["lse"][0], name


@pytest.mark.parametrize("seed", range(4))
def test_live_reference(oracle, ref, seed):
    rng = np.random.default_rng(seed)
    for n in (1, 3, 31, 1000, 3001):
        lw = rng.standard_normal(n) * (1 + 5 * seed)
        a = rng.random()
        r1, r2 = oracle.systematic(lw, a), ref.systematic(lw, a)
        for x, y in zip(r1[1:], r2[1:]):
            np.testing.assert_array_equal(x, y)
        u = rng.random(n)
        np.testing.assert_array_equal(oracle.multinomial(lw, u, 2)[1], ref.multinomial(lw, u, 1)[1])
        B = 3
        u = rng.random(2 * B * n)
        np.testing.assert_array_equal(oracle.metropolis(lw, B, u, 2)[1], ref.metropolis(lw, B, u, 1)[1])
        assert oracle.ess_reduce(lw) == ref.ess_reduce(lw)
        X = rng.standard_normal((5, n))
        as_ = ref.systematic(lw, a)[3]
        Y = np.zeros_like(X)
        ld = n
        oracle.L.orc_gather(as_.ctypes.data, X.ctypes.data, Y.ctypes.data, n, 5, ld, 8)
        np.testing.assert_array_equal(Y, ref.gather_rows(as_, X))


def test_degenerate(oracle, ref):
    lw = np.full(100, -np.inf)
    assert oracle.systematic(lw, 0.5)[0] == 1
    assert ref.systematic(lw, 0.5)[0] == 1
    assert oracle.multinomial(lw, np.full(100, 0.5))[0] == 1
