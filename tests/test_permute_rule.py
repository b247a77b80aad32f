"""The CUDA path's parallel formulation of the permutation and of the
fixed-point prefix sum, checked on the CPU against the oracle's sequential
restatement of the reference (ResamplerHost::cumulativeOffspringToAncestorsPermute,
share/src/bi/host/resampler/ResamplerHost.hpp:134-168)."""
import numpy as np


def parallel_permute(Os):
    """survivors in place; childless slot of rank r gets the ancestor a with
    E_a <= r < E_{a+1}, E_i = Os_{i-1} - i + Z_i, Z_i = #childless before i."""
    n = Os.size
    prev = np.concatenate([[0], Os[:-1]])
    o = Os - prev
    zero = (o == 0).astype(np.int64)
    Z = np.concatenate([[0], np.cumsum(zero)[:-1]])
    E = prev - np.arange(n) + Z
    as_ = np.where(o > 0, np.arange(n), -1)
    free = np.nonzero(o == 0)[0]
    as_[free] = np.searchsorted(E, Z[free], side="right") - 1
    return as_


def test_parallel_rule_matches_sequential(oracle):
    rng = np.random.default_rng(0)
    for trial in range(300):
        n = int(rng.integers(1, 3000))
        lw = rng.standard_normal(n) * rng.uniform(0, 8)
        rc, _, Os, seq = oracle.systematic(lw, rng.random(), permute=True)
        assert rc == 0
        np.testing.assert_array_equal(parallel_permute(Os), seq)


def test_permute_rule_invariants(oracle):
    rng = np.random.default_rng(1)
    for n in (1, 5, 100, 5000):
        as_in = np.sort(rng.integers(0, n, n)).astype(np.int32)
        out = oracle.permute_rule(as_in)
        counts_in = np.bincount(as_in, minlength=n)
        counts_out = np.bincount(out, minlength=n)
        np.testing.assert_array_equal(counts_in, counts_out)
        survivors = counts_in > 0
        np.testing.assert_array_equal(out[survivors], np.nonzero(survivors)[0])
        # the swap-based ResamplerHost::permute yields the same multiset with
        # the same survivors in place
        refp = oracle.ref_permute(as_in)
        np.testing.assert_array_equal(np.bincount(refp, minlength=n), counts_in)
        np.testing.assert_array_equal(refp[survivors], np.nonzero(survivors)[0])


def test_fixed_point_cumsum_close_to_sequential(oracle):
    rng = np.random.default_rng(2)
    for n in (1, 10, 4096, 100000):
        lw = rng.standard_normal(n) * 5
        ex = oracle.cumsum_exact(lw)
        _, Ws, _, _ = oracle.systematic(lw, 0.5)
        # what decides ancestors is Ws/W: both sums agree to within the
        # sequential FP64 sum's own rounding, a few n ulps of the total
        W = Ws[-1]
        assert np.max(np.abs(ex - Ws)) / W <= max(n, 16) * 2.0 ** -53
        assert np.all(np.diff(ex) >= 0)
