"""The Lorenz-96 step in one launch (systematic resampling as the
transition's prologue) against the two-launch form (the one-launch
resampler, then the transition) and the oracle: ancestors, states,
log-weights and every step's statistics bit for bit, at one block, a few
blocks, many blocks and a ragged last block, in both precisions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(model, n, ess_rel, seed):
    from libbi_b200 import BootstrapPF

    one = BootstrapPF(model, n, resampler="systematic", ess_rel=ess_rel, seed=seed)
    two = BootstrapPF(model, n, resampler="systematic", ess_rel=ess_rel, seed=seed)
    assert not one.step_form_fused  # the two-launch form is the default
    one.set_step_form(True)
    return one, two


@pytest.mark.parametrize(
    "dim,prec,n,ess_rel,T",
    [
        (40, "f32", 65536, 1.0, 10),
        (40, "f32", 1000, 0.5, 12),
        (40, "f32", 8192 + 77, 0.5, 10),
        (8, "f64", 4096, 1.0, 10),
        (40, "f64", 128, 1.0, 8),
    ],
)
def test_one_launch_step_equals_two_launch_and_oracle(cuda, oracle, dim, prec, n, ess_rel, T):
    from libbi_b200 import ModelL96

    model = ModelL96(dim=dim, precision=prec)
    desc = model.desc()
    dt = 0.05
    y, _ = oracle.simulate(desc, 40 + dim, T, 0.0, dt)
    one, two = _pair(model, n, ess_rel, seed=21)
    assert one.step_form_fused and not two.step_form_fused
    ra = [one.step(k * dt, (k + 1) * dt, y[k]) for k in range(T)]
    rb = [two.step(k * dt, (k + 1) * dt, y[k]) for k in range(T)]
    assert sum(r.resampled for r in ra) >= 2
    for a, b in zip(ra, rb):
        assert a == b
    xa, lwa, asa = one.state()
    xb, lwb, asb = two.state()
    np.testing.assert_array_equal(xa.cpu().numpy()[:, :n], xb.cpu().numpy()[:, :n])
    np.testing.assert_array_equal(lwa.cpu().numpy(), lwb.cpu().numpy())
    np.testing.assert_array_equal(asa.cpu().numpy(), asb.cpu().numpy())
    if n <= 8192 + 77:
        want = oracle.filter(desc, one._cfg, y, T, 0.0, dt)
        assert want["rc"] == 0
        np.testing.assert_array_equal(xa.cpu().numpy()[:, :n], want["x"][:, :n])
        np.testing.assert_allclose(lwa.cpu().numpy(), want["lw"], rtol=1e-12)
        np.testing.assert_allclose([r.log_increment for r in ra], want["inc"], rtol=1e-10, atol=1e-9)
    one.close()
    two.close()


def test_whole_filter_and_graph_replay_in_one_launch_form(cuda, oracle):
    """bpf_filter (the whole observation sequence, steps captured once as a
    CUDA graph and replayed) in the one-launch form, three runs on one
    handle: each equals the oracle's filter."""
    from libbi_b200 import BootstrapPF, ModelL96

    model = ModelL96(dim=40)
    desc = model.desc()
    n, T, dt = 65536, 12, 0.05
    pf = BootstrapPF(model, n, resampler="systematic", ess_rel=1.0, seed=5)
    pf.set_step_form(True)
    assert pf.step_form_fused
    for dseed in (51, 52, 53):
        y, _ = oracle.simulate(desc, dseed, T, 0.0, dt)
        ll, inc, ess = pf.filter(y, 0.0, dt)
        want = oracle.filter(desc, pf._cfg, y, T, 0.0, dt)
        assert want["rc"] == 0 and want["resampled"].sum() >= T - 1
        np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
        np.testing.assert_allclose(ess, want["ess"], rtol=1e-9)
        x, _, _ = pf.state()
        np.testing.assert_array_equal(x.cpu().numpy()[:, :n], want["x"][:, :n])
    pf.close()


def test_step_form_only_for_systematic(cuda):
    from libbi_b200 import BootstrapPF, BpfError, ModelL96, ModelPZ

    pf = BootstrapPF(ModelL96(dim=40), 4096, resampler="multinomial", seed=1)
    assert not pf.step_form_fused
    with pytest.raises(BpfError):
        pf.set_step_form(True)
    pf.set_step_form(False)
    pf.close()
    pz = BootstrapPF(ModelPZ(), 1024, resampler="systematic", seed=1)
    assert not pz.step_form_fused
    with pytest.raises(BpfError):
        pz.set_step_form(True)
    pz.close()
