"""Generate tests/golden/model_golden.npz from the reference's OWN host
updaters (RK4IntegratorHost, RK43IntegratorHost, StaticSamplerHost,
StaticUpdaterHost, SparseStaticLogDensityHost) run on hand-rendered L96 and
PZ model classes (oracle/ref/model_l96.cpp, oracle/ref/model_pz.cpp ->
oracle/_ref/libbiref.so and libbiref_f32.so, built by `make -C oracle ref`).

Each case is T filter steps of P particles without resampling, from the
initial draw the CUDA path makes for seed SEED (oracle.Oracle.init), with the
process noise of each step served to the reference from a tape of the
documented counter-based normals (include/bpf_philox.h) in the order
StaticSamplerHost consumes them.  Stored: the initial state, the normals and
observations of every step, and the reference's state and accumulated
log-weights after every step.

  l96_f64  Lorenz-96 d = 40, real = double, P = 64, T = 3, dt = 0.05
  l96_f32  the same model, real = float
  pz       PZ, RK4(3) h0 = 0.1, atoler = rtoler = 1e-3, P = 256, T = 3, dt = 1

Run from the repository root:  python tests/golden/make_model_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import Oracle, RefModels  # noqa: E402
from libbi_b200.filter import ModelL96, ModelPZ  # noqa: E402

SEED = 17
T = 3


def run_case(O, name, model, P, dt, f32):
    R = RefModels(f32=f32)
    desc = model.desc()
    x0, _ = O.init(desc, P, SEED)
    x = np.ascontiguousarray(x0[:, :P].T, np.float64)  # particle-major for the reference
    lp = np.zeros(P)
    ys, _ = O.simulate(desc, SEED + 1, T, 0.0, dt)
    out = {"x0": x0[:, :P].copy(), "seed": np.array([SEED]), "dt": np.array([dt]), "y": ys}
    zs, xs, lps = [], [], []
    for k in range(1, T + 1):
        if model.dim == 40:
            z = np.stack([O.noise_normals(SEED, p, k, 40, f32) for p in range(P)])
            x, lp = R.l96_transition(x, z, (k - 1) * dt, k * dt, ys[k - 1], lp)
        else:
            z = np.array([O.noise_normals(SEED, p, k, 2, False)[0] for p in range(P)])
            x, lp = R.pz_transition(x, z, (k - 1) * dt, k * dt, ys[k - 1], lp)
        zs.append(z)
        xs.append(x.T.copy())
        lps.append(lp.copy())
    out.update(z=np.stack(zs), x=np.stack(xs), lw=np.stack(lps))
    if f32:
        out["x"] = out["x"].astype(np.float32)
    return {f"{name}/{k}": v for k, v in out.items()}


def main():
    O = Oracle()
    data = {}
    data.update(run_case(O, "l96_f64", ModelL96(dim=40, precision="f64"), 64, 0.05, False))
    data.update(run_case(O, "l96_f32", ModelL96(dim=40), 64, 0.05, True))
    data.update(run_case(O, "pz", ModelPZ(), 256, 1.0, False))
    path = os.path.join(ROOT, "tests", "golden", "model_golden.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path}: {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
