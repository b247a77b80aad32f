"""Models compiled outside the library (include/bpf_model.cuh,
bpf_create_model): model classes in the shape LibBi's code generator emits
(tests/cpp/model_test_ar1.cuh, the reference's Test.bi; and
tests/cpp/model_l96_generated.cuh), compiled by nvcc with -fmad=false and
run by the library's filter, against the oracle's restatement of the same
expressions: states bit-identical, log-likelihood increments equal to
reduction rounding."""
import subprocess

import numpy as np
import pytest

from libbi_b200 import _native as N
from tests.test_library_cpu import ar1_desc, build_test_models, l96_gen_desc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def model_libs(cuda, tmp_path_factory):
    d = tmp_path_factory.mktemp("models")
    return {p: str(build_test_models(d, p)[0]) for p in ("double", "float")}


def _ar1(model_libs, precision):
    from libbi_b200 import ExternalModel

    return ExternalModel(model_libs[precision], "test_ar1_ops", [0.9, 0.25])


def _ar1_obs(T, precision, seed=7):
    """y_t = x_t + N(0, 0.5^2) of one AR(1) run (theta 0.9, sigma2 0.25)."""
    rng = np.random.default_rng(seed)
    x, y = 0.0, np.zeros((T, 1))
    for t in range(T):
        x = 0.9 * x + 0.5 * rng.standard_normal()
        y[t, 0] = x + 0.5 * rng.standard_normal()
    return y.astype(np.float64 if precision == "double" else np.float32)


def _compare(pf, want, n):
    x, lw, _ = pf.state()
    np.testing.assert_array_equal(x.cpu().numpy()[:, :n], want["x"][:, :n])
    np.testing.assert_allclose(lw.cpu().numpy(), want["lw"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("precision", ["double", "float"])
@pytest.mark.parametrize("n,resampler,B", [(4096, "systematic", 0), (20000, "systematic", 0),
                                           (3000, "multinomial", 0), (2048, "metropolis", 6)])
def test_test_bi_model_matches_oracle(cuda, oracle, model_libs, precision, n, resampler, B):
    """The reference's Test.bi (AR(1)) with an observation block, in the
    generated form, through bpf_create_model: every increment, the ESS and
    the final state against the oracle, with the one-CTA (n <= 4096) and
    grid-wide resamplers."""
    from libbi_b200 import BootstrapPF

    model = _ar1(model_libs, precision)
    T = 50
    y = _ar1_obs(T, precision)
    pf = BootstrapPF(model, n, resampler=resampler, ess_rel=0.5, seed=11, metropolis_steps=B)
    ll, inc, ess = pf.filter(y, 0.0, 1.0)
    prec = N.BPF_F64 if precision == "double" else N.BPF_F32
    want = oracle.filter(ar1_desc(prec), pf._cfg, y, T, 0.0, 1.0)
    assert want["rc"] == 0 and want["resampled"].sum() > 0
    np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(ess, want["ess"], rtol=1e-9)
    np.testing.assert_allclose(ll, want["ll"], rtol=1e-10)
    _compare(pf, want, n)
    pf.close()


def test_generated_l96_matches_oracle(cuda, oracle, model_libs):
    """Lorenz '96 in the generated form (noise block, RK4 ode block with the
    dfdt action, eval block, observation block), FP32, 8192 particles over
    10 observations: the generic fused kernel against the oracle's
    restatement of the generated expressions, bit for bit."""
    from libbi_b200 import BootstrapPF, ExternalModel, ModelL96

    F = 8.0
    model = ExternalModel(model_libs["float"], "test_l96_ops", [F])
    assert (model.dim, model.nobs, model.precision) == (40, 40, "f32")
    T, dt, n = 10, 0.05, 8192
    y, _ = oracle.simulate(ModelL96(dim=40).desc(), 33, T, 0.0, dt)
    pf = BootstrapPF(model, n, resampler="systematic", ess_rel=0.5, seed=4)
    ll, inc, ess = pf.filter(y, 0.0, dt)
    want = oracle.filter(l96_gen_desc(N.BPF_F32, F), pf._cfg, y, T, 0.0, dt)
    assert want["rc"] == 0 and want["resampled"].sum() > 0
    np.testing.assert_allclose(inc, want["inc"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(ess, want["ess"], rtol=1e-9)
    _compare(pf, want, n)
    pf.close()


def test_generated_l96_is_the_builtin_model(cuda, oracle, model_libs):
    """The generated-form Lorenz '96 and the library's built-in kernel are
    the same model up to rounding: FP64, no resampling (essRel 0), three
    observations; the increments agree to 1e-9 relative."""
    from libbi_b200 import BootstrapPF, ExternalModel, ModelL96

    T, dt, n = 3, 0.05, 1024
    y, _ = oracle.simulate(ModelL96(dim=40, precision="f64").desc(), 5, T, 0.0, dt)
    gen = BootstrapPF(ExternalModel(model_libs["double"], "test_l96_ops", [8.0]), n, ess_rel=0.0, seed=9)
    ref = BootstrapPF(ModelL96(dim=40, precision="f64"), n, ess_rel=0.0, seed=9)
    _, inc_g, _ = gen.filter(np.asarray(y, np.float64), 0.0, dt)
    _, inc_r, _ = ref.filter(np.asarray(y, np.float64), 0.0, dt)
    np.testing.assert_allclose(inc_g, inc_r, rtol=1e-9)
    gen.close()
    ref.close()


def test_external_model_checkpoint_and_path(cuda, model_libs):
    """The library's checkpoint and path output work unchanged on a model
    compiled outside it."""
    from libbi_b200 import BootstrapPF

    model = _ar1(model_libs, "double")
    y = _ar1_obs(8, "double")
    pf = BootstrapPF(model, 1000, ess_rel=1.0, seed=3)
    pf.path_cache(8)
    steps = [pf.step(float(k), float(k + 1), y[k]) for k in range(4)]
    blob = pf.snapshot()
    a = [pf.step(float(k), float(k + 1), y[k]) for k in range(4, 8)]
    p, path = pf.sample_path()
    assert 0 <= p < 1000 and path.shape == (9, 1)
    pf.restore(blob)
    b = [pf.step(float(k), float(k + 1), y[k]) for k in range(4, 8)]
    assert a == b and len(steps) == 4
    pf.close()


def test_external_model_rejects_bad_tables(cuda, model_libs):
    """bpf_create_model checks the table before any device work."""
    import ctypes

    from libbi_b200 import BpfError, ExternalModel

    model = _ar1(model_libs, "double")
    bad = N.ModelOps.from_buffer_copy(model.ops)
    bad.nobs = 65
    cfg = N.Config()
    cfg.nparticles, cfg.ess_rel = 100, 0.5
    h = ctypes.c_void_p()
    p = model.params.ctypes.data_as(ctypes.c_void_p)
    assert N.lib().bpf_create_model(ctypes.byref(bad), p, ctypes.byref(cfg), ctypes.byref(h)) == N.BPF_E_INVALID
    assert N.lib().bpf_create_model(ctypes.byref(model.ops), None, ctypes.byref(cfg),
                                    ctypes.byref(h)) == N.BPF_E_INVALID
    with pytest.raises(ValueError):
        ExternalModel(model_libs["double"], "test_ar1_ops", [0.9])
    bad = N.ModelOps.from_buffer_copy(model.ops)
    bad.transition = None
    assert N.lib().bpf_create_model(ctypes.byref(bad), p, ctypes.byref(cfg), ctypes.byref(h)) == N.BPF_E_INVALID
    cfg.nparticles = 0
    with pytest.raises(BpfError):
        N.check(N.lib().bpf_create_model(ctypes.byref(model.ops), p, ctypes.byref(cfg), ctypes.byref(h)),
                "bpf_create_model")


def test_cpp_client_with_generated_model(cuda, model_libs, tmp_path):
    """LibBi's filter client shape over the C++ interface with the
    generated-form Test.bi model compiled into the client
    (tests/cpp/model_client.cu: Filter<BootstrapPF<DeviceModel<ModelTest>,
    ...>>::filter over a Schedule): the same numbers as the Python mirror
    over the same C ABI, bit for bit."""
    import pathlib

    from libbi_b200 import BootstrapPF, Observer, Schedule

    root = pathlib.Path(__file__).resolve().parents[1]
    lib = root / "libbi_b200" / "_lib"
    exe = tmp_path / "model_client"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-fmad=false",
                    f"-I{root / 'include'}", str(root / "tests" / "cpp" / "model_client.cu"), f"-L{lib}",
                    "-lbi_b200", "-Xlinker", f"-rpath={lib}", "-o", str(exe)], check=True)
    T = 30
    y = _ar1_obs(T, "double", seed=21)
    t = np.arange(1, T + 1, dtype=np.float64)
    c = np.zeros(T, np.int64)
    v = y[:, 0]
    obs = tmp_path / "obs.txt"
    with open(obs, "w") as f:
        for a, b, x in zip(t, c, v):
            f.write(f"{float(a)!r} {int(b)} {float(x)!r}\n")
    out = subprocess.run([str(exe), "2000", "13", "0.5", str(obs)], capture_output=True, text=True,
                         check=True).stdout.split()
    pf = BootstrapPF(_ar1(model_libs, "double"), 2000, resampler="systematic", ess_rel=0.5, seed=13)
    try:
        want = Schedule(0.0, 1.0, Observer(t, c, v)).run(pf)
    finally:
        pf.close()
    got = np.array([float(s) for s in out])
    assert got[0] == want["loglik"]
    np.testing.assert_array_equal(got[1:], want["log_increments"])


@pytest.mark.parametrize("which,precision", [("l96", "float"), ("l96", "double"), ("ar1", "double")])
def test_unfused_block_updaters_equal_the_fused_step(cuda, model_libs, which, precision):
    """The bi:: block updaters of include/bpf_model.cuh (StaticSampler,
    RK4Integrator, StaticUpdater, SparseStaticLogDensity on a device
    State<B, ON_DEVICE>, one kernel each, called in the order of the
    generated transition and observation blocks) give the fused step's
    states and log-weights bit for bit, from the same initial particles."""
    import ctypes

    import torch
    from libbi_b200 import BootstrapPF, ExternalModel

    lib = ctypes.CDLL(model_libs[precision])
    f = getattr(lib, f"test_{which}_unfused_step")
    P = ctypes.c_void_p
    f.argtypes = [P, P, ctypes.c_int, ctypes.c_int, P, P, ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                  ctypes.c_int, P]
    f.restype = ctypes.c_int
    tdt = torch.float32 if precision == "float" else torch.float64
    if which == "l96":
        model = ExternalModel(model_libs[precision], "test_l96_ops", [8.0])
        n, t1, t2, nr = 3000, 0.0, 0.05, 40
        y = 8.0 + torch.randn(40, generator=torch.Generator().manual_seed(2), dtype=torch.float64)
    else:
        model = ExternalModel(model_libs[precision], "test_ar1_ops", [0.9, 0.25])
        n, t1, t2, nr = 3000, 0.0, 1.0, 1
        y = torch.tensor([0.3], dtype=torch.float64)
    seed = 5
    pf = BootstrapPF(model, n, ess_rel=0.0, seed=seed)
    x0, _, _ = pf.state()
    xs = x0.clone()
    pf.step(t1, t2, y.numpy())
    x1, lw1, _ = pf.state()
    ld = xs.shape[1]
    r = torch.zeros((nr, ld), dtype=tdt, device="cuda")
    prm = torch.as_tensor(model.params, dtype=tdt, device="cuda")
    yd = y.to(device="cuda", dtype=tdt)
    lp = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert f(xs.data_ptr(), r.data_ptr(), ld, n, prm.data_ptr(), yd.data_ptr(), t1, t2, seed, 1, lp.data_ptr()) == 0
    assert torch.equal(xs[:, :n], x1[:, :n])
    assert torch.equal(lp, lw1)
    pf.close()
