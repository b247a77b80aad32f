"""The learned proposal: the tensor-core forward/backward against the CPU
oracle's restatement (oracle/mlp_oracle.py) on the same minibatch, and
training on triples simulated by the library's own model."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _make(model, seed=3, max_batch=4096):
    from libbi_b200 import _native as N

    h = ctypes.c_void_p()
    d = model.desc()
    N.check(N.lib().bpf_proposal_create(ctypes.byref(d), 0.05, max_batch, seed, None, ctypes.byref(h)),
            "bpf_proposal_create")
    return h


def _params(h):
    from libbi_b200 import _native as N

    n = ctypes.c_int()
    N.lib().bpf_proposal_params(h, None, None, None, ctypes.byref(n))
    P = np.zeros(n.value, np.float32)
    N.check(N.lib().bpf_proposal_params(h, P.ctypes.data, None, None, None), "bpf_proposal_params")
    return P


@pytest.mark.parametrize("B", [128, 333, 2048])
def test_loss_and_gradient_match_oracle(cuda, B):
    import torch
    from libbi_b200 import ModelL96
    from libbi_b200 import _native as N
    from oracle.mlp_oracle import bf16, loss_grad

    h = _make(ModelL96(dim=40))
    P = _params(h)
    # a trained-looking output layer, so that both heads carry gradient
    rng = np.random.default_rng(B)
    P = (P + 0.05 * rng.standard_normal(P.size)).astype(np.float32)
    N.check(N.lib().bpf_proposal_set_params(h, P.ctypes.data, None, None), "bpf_proposal_set_params")
    U = bf16(rng.standard_normal((B, 80)).astype(np.float32))
    r0 = (0.1 * rng.standard_normal((B, 40))).astype(np.float32)
    Ud = torch.as_tensor(U).to(torch.bfloat16).cuda()
    r0d = torch.as_tensor(r0).cuda()
    g = torch.zeros(P.size, dtype=torch.float32, device="cuda")
    loss = ctypes.c_double()
    N.check(N.lib().bpf_proposal_loss_grad(h, Ud.data_ptr(), r0d.data_ptr(), B, ctypes.byref(loss), g.data_ptr()),
            "bpf_proposal_loss_grad")
    want_loss, want_g = loss_grad(P, U, r0)
    np.testing.assert_allclose(loss.value, want_loss, rtol=1e-4)
    got = g.cpu().numpy().astype(np.float64)
    # blocks W1, b1, W2, b2, W3, b3: relative L2 error of each
    sizes = [128 * 80, 128, 128 * 128, 128, 80 * 128, 80]
    o = 0
    for n in sizes:
        a, b = got[o:o + n], want_g[o:o + n]
        assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b) + 1e-9, (o, np.linalg.norm(a - b), np.linalg.norm(b))
        o += n
    N.lib().bpf_proposal_destroy(h)


def _triples(model, n, dt):
    """(x_t, x_{t+1}, y_{t+1}) simulated by the library's own model."""
    import torch
    from libbi_b200 import BootstrapPF

    pf = BootstrapPF(model, n, seed=9)
    for k in range(40):  # onto the attractor
        pf.step(k * dt, (k + 1) * dt, None)
    x, _, _ = pf.state()
    xt = x[:, :n].T.contiguous().clone()
    pf.step(40 * dt, 41 * dt, None)
    x, _, _ = pf.state()
    xt1 = x[:, :n].T.contiguous().clone()
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    y = (xt1 + model.sigma_y * torch.randn(xt1.shape, generator=g, device="cuda")).contiguous()
    pf.close()
    return xt, xt1, y


def test_training_is_reproducible(cuda):
    """The same seed, data and schedule give the same loss trace and the same
    parameters, bit for bit (no atomics in the gradient sums)."""
    from libbi_b200 import ModelL96
    from libbi_b200 import _native as N

    model = ModelL96(dim=40, sigma_eta=0.5, sigma_y=0.1)
    n = 1 << 14
    xt, xt1, y = _triples(model, n, 0.05)
    out = []
    for _ in range(2):
        h = _make(model, max_batch=2048)
        N.check(N.lib().bpf_proposal_set_data(h, xt.data_ptr(), xt1.data_ptr(), y.data_ptr(), n),
                "bpf_proposal_set_data")
        trace = np.zeros(200, np.float32)
        N.check(N.lib().bpf_proposal_train(h, 200, 2048, 2e-3, trace.ctypes.data), "bpf_proposal_train")
        out.append((trace, _params(h)))
        N.lib().bpf_proposal_destroy(h)
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][0][-20:].mean() < out[0][0][:5].mean()


def test_training_learns_the_observation_update(cuda):
    """With an informative observation (sigma_y = 0.1 against sigma_eta = 0.5)
    the optimal proposal moves most of the way to y; training from the
    transition-like start must find most of that gain."""
    import torch
    from libbi_b200 import BootstrapPF, ModelL96
    from libbi_b200 import _native as N

    model = ModelL96(dim=40, sigma_eta=0.5, sigma_y=0.1)
    n, dt = 1 << 16, 0.05
    pf = BootstrapPF(model, n, seed=9)
    for k in range(40):  # onto the attractor
        pf.step(k * dt, (k + 1) * dt, None)
    x, _, _ = pf.state()
    xt = x[:, :n].T.contiguous().clone()
    pf.step(40 * dt, 41 * dt, None)
    x, _, _ = pf.state()
    xt1 = x[:, :n].T.contiguous().clone()
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    y = (xt1 + model.sigma_y * torch.randn(xt1.shape, generator=g, device="cuda")).contiguous()
    pf.close()
    h = _make(model, max_batch=4096)
    N.check(N.lib().bpf_proposal_set_data(h, xt.data_ptr(), xt1.data_ptr(), y.data_ptr(), n),
            "bpf_proposal_set_data")
    steps = 1500
    trace = np.zeros(steps, np.float32)
    N.check(N.lib().bpf_proposal_train(h, steps, 4096, 2e-3, trace.ctypes.data), "bpf_proposal_train")
    # per-dimension NLL: transition alone log(0.5) + 1/2 = -0.193; the optimal
    # proposal log(sigma_post) + 1/2 with sigma_post^2 = 0.25*0.01/0.26 -> -1.82
    first, last = float(trace[:10].mean()) / 40, float(trace[-50:].mean()) / 40
    assert np.isfinite(trace).all()
    assert first > -0.6
    assert last < -1.6, (first, last)
    N.lib().bpf_proposal_destroy(h)
