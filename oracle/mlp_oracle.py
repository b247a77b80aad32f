"""ORACLE — test infrastructure only.  CPU restatement (numpy, FP64
accumulation) of the learned proposal's loss and gradient
(libbi_b200/csrc/proposal.cu): the same BF16 roundings of weights,
activations and back-propagated errors as the tensor-core path, so that the
only differences left are the order of the FP32 sums on the GPU."""
from __future__ import annotations

import numpy as np

S_MIN, S_MAX = -7.0, 3.0


def bf16(x):
    """Round FP32 values to BF16 (round to nearest even), returned as FP32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def unpack(params, d=40, hidden=128, din=None):
    din = 2 * d if din is None else din
    dout = 2 * d
    o = 0
    out = {}
    for name, shape in (("W1", (hidden, din)), ("b1", (hidden,)), ("W2", (hidden, hidden)), ("b2", (hidden,)),
                        ("W3", (dout, hidden)), ("b3", (dout,))):
        n = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + n], np.float32).reshape(shape)
        o += n
    return out


def loss_grad(params, U, r0, d=40, hidden=128):
    """Mean Gaussian NLL and its gradient (flat, the parameter layout) for a
    minibatch: U [B x din] (BF16 values; din = 2d for Lorenz '96, 3 for
    PZ), r0 [B x d] = x_{t+1} - m(x_t) (Lorenz '96) or log alpha - mu (PZ)."""
    U = np.asarray(U, np.float64)
    P = unpack(params, d, hidden, U.shape[1])
    W1h, W2h, W3h = bf16(P["W1"]), bf16(P["W2"]), bf16(P["W3"])
    B = U.shape[0]
    H1 = bf16(np.maximum((U @ W1h.T.astype(np.float64)) + P["b1"], 0.0).astype(np.float32))
    H2 = bf16(np.maximum((H1.astype(np.float64) @ W2h.T) + P["b2"], 0.0).astype(np.float32))
    O = ((H2.astype(np.float64) @ W3h.T) + P["b3"]).astype(np.float32)
    delta, sr = O[:, :d], O[:, d:]
    s = np.clip(sr, S_MIN, S_MAX)
    e = np.exp(-2.0 * s.astype(np.float32))
    r = (np.asarray(r0, np.float32) - delta).astype(np.float32)
    loss = float(np.sum(s + 0.5 * r * r * e, dtype=np.float64) / B)
    inside = (sr > S_MIN) & (sr < S_MAX)
    dO = bf16(np.concatenate([-r * e / B, np.where(inside, (1.0 - r * r * e) / B, 0.0)], axis=1).astype(np.float32))
    dO64 = dO.astype(np.float64)
    gW3 = dO64.T @ H2
    gb3 = dO64.sum(0)
    dZ2 = bf16(np.where(H2 > 0, (dO64 @ W3h).astype(np.float32), 0.0).astype(np.float32)).astype(np.float64)
    gW2 = dZ2.T @ H1
    gb2 = dZ2.sum(0)
    dZ1 = bf16(np.where(H1 > 0, (dZ2 @ W2h).astype(np.float32), 0.0).astype(np.float32)).astype(np.float64)
    gW1 = dZ1.T @ U
    gb1 = dZ1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def forward(params, shift, scale, x_t, innov, d=40, hidden=128):
    """(delta, s) of the proposal for rows [x_t, y - m(x_t)] (FP32 arrays),
    with the tensor-core path's BF16 roundings."""
    P = unpack(params, d, hidden)
    W1h, W2h, W3h = bf16(P["W1"]), bf16(P["W2"]), bf16(P["W3"])
    U = bf16((np.concatenate([x_t, innov], axis=1).astype(np.float32) - shift) * scale).astype(np.float64)
    H1 = bf16(np.maximum(U @ W1h.T + P["b1"], 0.0).astype(np.float32)).astype(np.float64)
    H2 = bf16(np.maximum(H1 @ W2h.T + P["b2"], 0.0).astype(np.float32)).astype(np.float64)
    O = (H2 @ W3h.T + P["b3"]).astype(np.float32)
    return O[:, :d], np.clip(O[:, d:], S_MIN, S_MAX)


def guided_step(delta, s, m, z, y, sigma_eta, sigma_y, lw0):
    """The guided step's new state and log-weights given the network output,
    the RK4 means m, the standard normals z and the observation y (all
    [n x d] except y [d]): x' = m + delta + exp(s) z and
    lw = lw0 + log N(y; x', sigma_y) + log N(x'; m, sigma_eta) - log N(x'; m + delta, exp(s))."""
    dx = delta + np.exp(s) * z
    x = m + dx
    c2 = 0.91893853320467274178032973640562
    obs = np.sum(-0.5 * ((y - x) / sigma_y) ** 2 - c2 - np.log(sigma_y), axis=1)
    corr = np.sum(-0.5 * (dx / sigma_eta) ** 2 - np.log(sigma_eta), axis=1) - np.sum(-0.5 * z * z - s, axis=1)
    return x, lw0 + obs + corr


def forward_rows(params, shift, scale, feats, d, hidden=128):
    """(delta, s) of the proposal for raw input rows feats [B x din] (the
    PZ proposal: [log P, log Z, y - log P], d = 1), with the tensor-core
    path's BF16 roundings."""
    din = feats.shape[1]
    P = unpack(params, d, hidden, din)
    W1h, W2h, W3h = bf16(P["W1"]), bf16(P["W2"]), bf16(P["W3"])
    U = bf16((np.asarray(feats, np.float32) - shift) * scale).astype(np.float64)
    H1 = bf16(np.maximum(U @ W1h.T + P["b1"], 0.0).astype(np.float32)).astype(np.float64)
    H2 = bf16(np.maximum(H1 @ W2h.T + P["b2"], 0.0).astype(np.float32)).astype(np.float64)
    O = (H2 @ W3h.T + P["b3"]).astype(np.float32)
    return O[:, :d], np.clip(O[:, d:], S_MIN, S_MAX)
