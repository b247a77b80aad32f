"""The CUDA filter step (fused noise + RK4 / RK4(3) + observation density)
against the reference's OWN host updaters on hand-rendered model classes,
through the committed fixtures (tests/golden/model_golden.npz): the same
initial draw, the same process-noise normals, no resampling (ess_rel = 0),
T steps.  Tolerances as for the oracle (tests/test_oracle_models.py): the
rounding of fused multiply-adds and of the order of additions."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "model_golden.npz")
TOL = {"l96_f64": (1e-13, 1e-13, 1e-13), "l96_f32": (2e-6, 2e-6, 2e-6), "pz": (1e-12, 1e-14, 1e-13)}


@pytest.mark.parametrize("which", ["l96_f64", "l96_f32", "pz"])
def test_cuda_steps_match_reference_updaters(cuda, which):
    from libbi_b200 import BootstrapPF, ModelL96, ModelPZ

    d = np.load(GOLDEN)
    g = {k.split("/", 1)[1]: d[k] for k in d.files if k.startswith(which + "/")}
    model = {"l96_f64": ModelL96(dim=40, precision="f64"), "l96_f32": ModelL96(dim=40), "pz": ModelPZ()}[which]
    seed, dt = int(g["seed"][0]), float(g["dt"][0])
    P = g["x0"].shape[1]
    pf = BootstrapPF(model, P, resampler="systematic", ess_rel=0.0, seed=seed)
    x, lw, _ = pf.state()
    np.testing.assert_array_equal(x.cpu().numpy()[:, :P], g["x0"])
    rt, at, lrt = TOL[which]
    for k in range(1, g["x"].shape[0] + 1):
        res = pf.step((k - 1) * dt, k * dt, g["y"][k - 1])
        assert not res.resampled
        x, lw, _ = pf.state()
        np.testing.assert_allclose(x.cpu().numpy()[:, :P], g["x"][k - 1], rtol=rt, atol=at)
        np.testing.assert_allclose(lw.cpu().numpy()[:P], g["lw"][k - 1], rtol=lrt, atol=1e-12)
    pf.close()
