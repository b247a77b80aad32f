"""Failure detection without a GPU fault: the bounded waits of the
cooperative resampler.  Every grid-wide barrier of the one-launch systematic
resampler waits for the other blocks at most a limit of SM clock cycles and
then records BPF_E_TIMEOUT and returns.  A limit below zero makes a block
that finds a barrier still closed give up at once, so these tests take the
timeout path with every block of the kernel running normally: nothing waits
for a flag that is never set, and the context stays usable.  After the
default limit is back, the next call on the same scratch (where the
abandoned launch left a barrier counter above zero) must again return the
oracle's ancestors bit for bit.  The one-tile kernel hands its phases over
through published words rather than barriers; under a negative limit every
one of its polls gives up, and the next status reset moves its epoch on.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _set_limit(cycles):
    from libbi_b200 import _native as N

    assert N.lib().bpf_debug_set_wait_limit(int(cycles)) == N.BPF_OK


@pytest.mark.parametrize("n", [65536, 1 << 20])
def test_barrier_timeout_reported_then_next_call_exact(cuda, oracle, n):
    """n = 65536: one tile per block (k_systematic_coop1); 2^20: several
    tiles per block (k_systematic_coop)."""
    import torch
    from libbi_b200 import BpfError, SystematicResampler
    from libbi_b200 import _native as N

    rng = np.random.default_rng(n + 7)
    lw = rng.standard_normal(n) * 2.0
    a = rng.random(1)
    lw_d = torch.as_tensor(lw, device="cuda", dtype=torch.float64)
    a_d = torch.as_tensor(a, device="cuda", dtype=torch.float64)
    # the abandoned launch runs on other log-weights, so that anything it
    # left behind and a later launch took for its own would show
    lw_other = torch.as_tensor(rng.standard_normal(n) * 3.0, device="cuda", dtype=torch.float64)
    R = SystematicResampler(max_n=n)
    try:
        _set_limit(-1)
        with pytest.raises(BpfError) as e:
            R.ancestors(lw_other, a_d, permute=True)
        assert e.value.status == N.BPF_E_TIMEOUT
    finally:
        _set_limit(N.BPF_WAIT_LIMIT_DEFAULT)
    _, _, Os_o, perm_o = oracle.systematic(lw, a[0], permute=True)
    for _ in range(2):
        perm, Os = R.ancestors(lw_d, a_d, permute=True, with_offspring=True)
        np.testing.assert_array_equal(Os.cpu().numpy(), Os_o)
        np.testing.assert_array_equal(perm.cpu().numpy(), perm_o)
    R.close()


@pytest.mark.parametrize("one_launch", [True, False])
def test_filter_step_timeout_is_sticky_until_init(cuda, oracle, one_launch):
    """A filter whose resampling gave up reports BPF_E_TIMEOUT on that step
    and every later one (the status is sticky, so no later launch starts on
    the abandoned barrier state); bpf_init clears it, and the next whole
    filter equals the oracle's.  one_launch: the resampling is the step
    kernel's prologue (its polls give up); otherwise the one-launch
    resampler's."""
    from libbi_b200 import BootstrapPF, BpfError, ModelL96
    from libbi_b200 import _native as N

    model = ModelL96(dim=40)
    desc = model.desc()
    n, T, dt = 65536, 6, 0.05
    y, _ = oracle.simulate(desc, 31, T, 0.0, dt)
    pf = BootstrapPF(model, n, resampler="systematic", ess_rel=1.0, seed=12)
    pf.set_step_form(one_launch)
    pf.step(0.0, dt, y[0])  # observed: the next step resamples (essRel = 1)
    try:
        _set_limit(-1)
        with pytest.raises(BpfError) as e:
            pf.step(dt, 2 * dt, y[1])
        assert e.value.status == N.BPF_E_TIMEOUT
    finally:
        _set_limit(N.BPF_WAIT_LIMIT_DEFAULT)
    with pytest.raises(BpfError) as e:
        pf.step(2 * dt, 3 * dt, y[2])
    assert e.value.status == N.BPF_E_TIMEOUT
    ll, inc, ess = pf.filter(y, 0.0, dt)  # bpf_init first
    want = oracle.filter(desc, pf._cfg, y, T, 0.0, dt)
    assert want["rc"] == 0 and want["resampled"].sum() >= T - 1
    np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
    x, _, _ = pf.state()
    np.testing.assert_array_equal(x.cpu().numpy()[:, :n], want["x"][:, :n])
    pf.close()
