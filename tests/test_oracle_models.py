"""The model half of the oracle (process noise, RK4, RK4(3), observation
log-density; oracle/bpf_oracle.c) against the reference's OWN host updaters
run on hand-rendered model classes (oracle/ref/model_l96.cpp, model_pz.cpp):
committed fixtures (tests/golden/model_golden.npz, made by
tests/golden/make_model_golden.py) and, where the reference build is present,
fresh runs.  Differences are the rounding of fused multiply-adds and of the
order of additions: the oracle uses explicit FMAs, the reference is built
with contraction off, and the reference accumulates log-densities in `real`."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "model_golden.npz")

# (state rtol, state atol, log-weight rtol)
TOL = {"l96_f64": (1e-13, 1e-13, 1e-13), "l96_f32": (2e-6, 2e-6, 2e-6), "pz": (1e-12, 1e-14, 1e-13)}


def _model(which):
    from libbi_b200 import ModelL96, ModelPZ

    return {"l96_f64": ModelL96(dim=40, precision="f64"), "l96_f32": ModelL96(dim=40), "pz": ModelPZ()}[which]


@pytest.fixture(scope="module")
def model_golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("which", ["l96_f64", "l96_f32", "pz"])
def test_noise_draws_are_the_fixture_draws(oracle, model_golden, which):
    g = {k.split("/", 1)[1]: model_golden[k] for k in model_golden.files if k.startswith(which + "/")}
    seed = int(g["seed"][0])
    T, P = g["z"].shape[0], g["z"].shape[1]
    f32 = which == "l96_f32"
    for k in range(1, T + 1):
        for p in range(0, P, 7):
            if which == "pz":
                assert oracle.noise_normals(seed, p, k, 2, False)[0] == g["z"][k - 1][p]
            else:
                np.testing.assert_array_equal(oracle.noise_normals(seed, p, k, 40, f32), g["z"][k - 1][p])


@pytest.mark.parametrize("which", ["l96_f64", "l96_f32", "pz"])
def test_oracle_steps_match_reference_updaters(oracle, model_golden, which):
    g = {k.split("/", 1)[1]: model_golden[k] for k in model_golden.files if k.startswith(which + "/")}
    desc = _model(which).desc()
    seed, dt = int(g["seed"][0]), float(g["dt"][0])
    x = g["x0"].copy()
    P = x.shape[1]
    x_init, _ = oracle.init(desc, P, seed)
    np.testing.assert_array_equal(x_init[:, :P], x)
    lw = np.zeros(P)
    rt, at, lrt = TOL[which]
    for k in range(1, g["x"].shape[0] + 1):
        x, lw = oracle.transition(desc, x, P, None, False, lw, g["y"][k - 1], (k - 1) * dt, k * dt, seed, k, 0.0)
        np.testing.assert_allclose(x, g["x"][k - 1], rtol=rt, atol=at)
        np.testing.assert_allclose(lw, g["lw"][k - 1], rtol=lrt, atol=1e-12)


@pytest.mark.parametrize("which", ["l96_f64", "l96_f32", "pz"])
def test_oracle_matches_live_reference(oracle, which):
    from oracle.oracle import REF_F32_SO, REF_SO, RefModels

    if not os.path.exists(REF_F32_SO if which == "l96_f32" else REF_SO):
        pytest.skip("reference build absent")
    R = RefModels(f32=which == "l96_f32")
    model = _model(which)
    desc = model.desc()
    f32 = which == "l96_f32"
    P, seed = (1024, 123) if which != "pz" else (2048, 321)
    dt = 0.05 if which != "pz" else 1.0
    ys, _ = oracle.simulate(desc, seed + 5, 2, 0.0, dt)
    x, _ = oracle.init(desc, P, seed)
    x = x[:, :P].copy()
    xr = x.T.astype(np.float64)
    lw, lr = np.zeros(P), np.zeros(P)
    rt, at, lrt = TOL[which]
    for k in (1, 2):
        x, lw = oracle.transition(desc, x, P, None, False, lw, ys[k - 1], (k - 1) * dt, k * dt, seed, k, 0.0)
        if which == "pz":
            z = np.array([oracle.noise_normals(seed, p, k, 2, False)[0] for p in range(P)])
            xr, lr = R.pz_transition(xr, z, (k - 1) * dt, k * dt, ys[k - 1], lr)
        else:
            z = np.stack([oracle.noise_normals(seed, p, k, 40, f32) for p in range(P)])
            xr, lr = R.l96_transition(xr, z, (k - 1) * dt, k * dt, ys[k - 1], lr)
        np.testing.assert_allclose(x, xr.T, rtol=rt, atol=at)
        np.testing.assert_allclose(lw, lr, rtol=lrt, atol=1e-12)
