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


def test_path_record_is_pruned_to_the_genealogy(cuda, oracle):
    """The record keeps a node only for particles with a line to the current
    generation (AncestryCache's prune): after every step its node count
    equals the size of the current particles' genealogy computed on the host
    from the recorded ancestors, far below (T + 1) x N, and a sampled path
    still follows the recorded states."""
    from libbi_b200 import BootstrapPF, ModelL96

    model, n, T, dt = ModelL96(dim=40), 4096, 40, 0.05
    y, _ = oracle.simulate(model.desc(), 9, T, 0.0, dt)
    pf = BootstrapPF(model, n, ess_rel=1.0, seed=6)
    pf.path_cache(T)
    x, _, _ = pf.state()
    xs = [x.cpu().numpy()[:, :n].copy()]
    anc = []
    for k in range(T):
        res = pf.step(k * dt, (k + 1) * dt, y[k])
        x, _, as_ = pf.state()
        xs.append(x.cpu().numpy()[:, :n].copy())
        anc.append(as_.cpu().numpy().copy() if res.resampled else np.arange(n))
        # the genealogy of the current particles: distinct ancestors per generation
        live, want = np.arange(n), n
        for a in reversed(anc):
            live = np.unique(a[live])
            want += live.size
        nodes, cap = pf.path_nodes()
        assert nodes == want, (k, nodes, want)
    assert nodes < (T + 1) * n // 4 and cap < (T + 1) * n // 2
    p, path = pf.sample_path()
    a = p
    for t in range(T, -1, -1):
        np.testing.assert_array_equal(path[t], xs[t][:, a])
        if t > 0:
            a = int(anc[t - 1][a])
    pf.close()
