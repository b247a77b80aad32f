"""The documented random stream and the portable elementary functions
(include/bpf_philox.h, include/bpf_math.h), on the host."""
import ctypes

import numpy as np


def test_philox_known_answers(oracle):
    # Philox4x32-10 known-answer vectors published with the algorithm (Random123)
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
        ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
        ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
         (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
    ]
    for c, k, want in kat:
        cc = (ctypes.c_uint32 * 4)(*c)
        kk = (ctypes.c_uint32 * 2)(*k)
        out = (ctypes.c_uint32 * 4)()
        oracle.L.orc_philox(cc, kk, out)
        assert tuple(out) == want


def _eval(oracle, fn, x):
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros_like(x)
    oracle.L.orc_math_eval(fn, x.ctypes.data, y.ctypes.data, x.size)
    return y


def _ulps(a, b, dtype):
    a = np.asarray(a, dtype)
    b = np.asarray(b, dtype)
    return np.abs(a - b) / np.spacing(np.abs(b).astype(dtype))


def test_double_functions_within_2ulp(oracle):
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-700, 700, 20000), rng.uniform(-1, 1, 20000), [0.0, 1e-300, -745.0]])
    assert np.max(_ulps(_eval(oracle, 0, x), np.exp(x), np.float64)) <= 2
    x = np.concatenate([rng.uniform(1e-300, 1e300, 5000), np.exp(rng.uniform(-700, 700, 20000)),
                        rng.uniform(0.5, 2.0, 20000), [1.0, 2.0, 0.5]])
    y = _eval(oracle, 1, x)
    ref = np.log(x)
    big = np.abs(ref) > 1e-3
    assert np.max(_ulps(y[big], ref[big], np.float64)) <= 2
    assert np.max(np.abs(y[~big] - ref[~big])) <= 4e-16
    t = rng.uniform(0, 2, 40000)
    np.testing.assert_allclose(_eval(oracle, 2, t), np.sin(np.pi * t), rtol=0, atol=1e-15)  # numpy rounds pi*t first
    np.testing.assert_allclose(_eval(oracle, 3, t), np.cos(np.pi * t), rtol=0, atol=1e-15)  # numpy rounds pi*t first


def test_float_functions(oracle):
    rng = np.random.default_rng(2)
    x = rng.uniform(-80, 80, 20000).astype(np.float32).astype(np.float64)
    assert np.max(_ulps(_eval(oracle, 4, x), np.exp(x), np.float32)) <= 2
    x = rng.uniform(1e-7, 1.0, 20000).astype(np.float32).astype(np.float64)
    ref = np.log(x)
    y = _eval(oracle, 5, x)
    big = np.abs(ref) > 1e-2
    assert np.max(_ulps(y[big], ref[big], np.float32)) <= 2
    t = (rng.uniform(0, 1, 20000).astype(np.float32) * 2).astype(np.float64)
    np.testing.assert_allclose(_eval(oracle, 6, t), np.sin(np.pi * t), rtol=0, atol=3e-7)
    np.testing.assert_allclose(_eval(oracle, 7, t), np.cos(np.pi * t), rtol=0, atol=3e-7)


def test_normals_are_standard(oracle):
    z = np.zeros(400000)
    for p in range(10):
        chunk = np.zeros(40000)
        oracle.L.orc_noise_normals(ctypes.c_uint64(5), p, 1, 40000, 0, chunk.ctypes.data)
        z[p * 40000:(p + 1) * 40000] = chunk
    assert abs(z.mean()) < 0.01
    assert abs(z.std() - 1.0) < 0.01
    assert abs(np.mean(z ** 3)) < 0.03
    assert abs(np.mean(z ** 4) - 3.0) < 0.05
