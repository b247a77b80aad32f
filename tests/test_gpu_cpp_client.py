"""The C++ interface (include/libbi_b200.hpp) driven like LibBi's generated
filter client (tests/cpp/filter_client.cpp: Filter<BootstrapPF>::filter over
a Schedule of sparse observations) against the Python mirror over the same
C ABI: the same calls, so the same numbers bit for bit; status codes
become exceptions."""
import subprocess

import numpy as np
import pytest

from tests.test_library_cpu import build_cpp_client

pytestmark = pytest.mark.gpu


def _sparse_obs(y, dt, rng, every=1):
    T, d = y.shape
    t, c, v = [], [], []
    for k in range(T):
        if k % every:
            continue
        keep = np.nonzero(rng.random(d) < 0.6)[0] if d > 1 else np.arange(d)
        if keep.size == 0:
            keep = np.array([0])
        for j in keep:
            t.append((k + 1) * dt)
            c.append(int(j))
            v.append(float(y[k, j]))
    return np.array(t), np.array(c), np.array(v)


def _write(path, t, c, v):
    with open(path, "w") as f:
        for a, b, x in zip(t, c, v):
            f.write(f"{float(a)!r} {int(b)} {float(x)!r}\n")


def _python(model, n, seed, ess_rel, t, c, v, dt):
    from libbi_b200 import BootstrapPF, Observer, Schedule

    pf = BootstrapPF(model, n, resampler="systematic", ess_rel=ess_rel, seed=seed)
    try:
        return Schedule(0.0, dt, Observer(t, c, v)).run(pf)
    finally:
        pf.close()


@pytest.mark.parametrize("which", ["l96", "pz"])
def test_cpp_client_equals_python_schedule_run(cuda, oracle, tmp_path, which):
    from libbi_b200 import ModelL96, ModelPZ

    exe = build_cpp_client(tmp_path)
    model, dt, T, n = (ModelL96(dim=8), 0.05, 14, 1500) if which == "l96" else (ModelPZ(), 1.0, 10, 800)
    y, _ = oracle.simulate(model.desc(), 17, T, 0.0, dt)
    t, c, v = _sparse_obs(np.asarray(y, np.float64), dt, np.random.default_rng(3), every=1 if which == "l96" else 2)
    obs = tmp_path / "obs.txt"
    _write(obs, t, c, v)
    out = subprocess.run([str(exe), which, str(n), "5", "0.5", str(obs)], capture_output=True, text=True,
                         check=True).stdout.split()
    want = _python(model, n, 5, 0.5, t, c, v, dt)
    got = np.array([float(s) for s in out])
    assert got[0] == want["loglik"]
    np.testing.assert_array_equal(got[1:], want["log_increments"])


def test_cpp_client_path_and_errors(cuda, oracle, tmp_path):
    from libbi_b200 import ModelPZ

    exe = build_cpp_client(tmp_path)
    model, dt, T = ModelPZ(), 1.0, 6
    y, _ = oracle.simulate(model.desc(), 4, T, 0.0, dt)
    t = (np.arange(T) + 1.0) * dt
    c = np.zeros(T, np.int64)
    v = np.asarray(y[:, 0], np.float64)
    obs = tmp_path / "obs.txt"
    _write(obs, t, c, v)
    # a path reserved before Filter::filter survives its init: T + 1 states
    out = subprocess.run([str(exe), "pz", "500", "7", "1.0", str(obs), "path"], capture_output=True, text=True,
                         check=True).stdout.splitlines()
    tag, particle, length = out[-1].split()
    assert tag == "path" and 0 <= int(particle) < 500 and int(length) == T + 1
    # the C ABI's status codes become exceptions: N = 0 is rejected by bpf_create
    r = subprocess.run([str(exe), "pz", "0", "7", "1.0", str(obs)], capture_output=True, text=True)
    assert r.returncode == 1 and "bpf_create" in r.stderr
