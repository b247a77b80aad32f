"""Path output (bpf_path_cache / bpf_sample_path, BootstrapPF::samplePath):
the drawn particle against the multinomial draw restated on the oracle's
exact cumulative weights, and the path against the states and ancestors
read back after every step."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["l96", "pz"])
def test_sample_path_follows_recorded_ancestry(cuda, oracle, which):
    import torch
    from libbi_b200 import BootstrapPF, ModelL96, ModelPZ

    if which == "l96":
        model, n, T, dt, ess_rel = ModelL96(dim=40), 1024, 15, 0.05, 0.5
    else:
        model, n, T, dt, ess_rel = ModelPZ(), 777, 12, 1.0, 1.0
    y, _ = oracle.simulate(model.desc(), 5, T, 0.0, dt)
    pf = BootstrapPF(model, n, ess_rel=ess_rel, seed=3)
    pf.path_cache(T)
    x, _, _ = pf.state()
    xs = [x.cpu().numpy()[:, :n].copy()]
    anc = []
    resampled = 0
    for k in range(T):
        res = pf.step(k * dt, (k + 1) * dt, y[k])
        x, lw, as_ = pf.state()
        xs.append(x.cpu().numpy()[:, :n].copy())
        anc.append(as_.cpu().numpy().copy() if res.resampled else np.arange(n))
        resampled += res.resampled
    assert resampled > 0
    lw = lw.cpu().numpy().copy()
    for uval in (0.0, 0.3719, 0.999999):
        u = torch.tensor([uval], dtype=torch.float64, device="cuda")
        p, path = pf.sample_path(u)
        Ws = oracle.cumsum_exact(lw)
        want_p = int(np.argmax(Ws >= Ws[-1] * uval))
        assert p == want_p
        assert path.shape == (T + 1, model.dim)
        a = p
        for t in range(T, -1, -1):
            np.testing.assert_array_equal(path[t], xs[t][:, a])
            if t > 0:
                a = int(anc[t - 1][a])
    # the handle's own draw gives a valid particle and path
    p, path = pf.sample_path()
    assert 0 <= p < n and np.isfinite(path).all()
    # a restarted record (bpf_init) holds the initial state only
    pf.init()
    _, path = pf.sample_path()
    assert path.shape == (1, model.dim)
    pf.close()
