"""The C-ABI library loads and exports every entry point include/*.h
declares, and rejects invalid arguments before touching a GPU."""
import ctypes
import os
import re

import pytest

from libbi_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:int|const char\*|void)\s+(bpf_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def L():
    from libbi_b200 import build

    build.build()
    return N.load_library()


def test_exports_every_declared_symbol(L):
    declared = _declared()
    assert declared, "no declarations found"
    assert declared <= set(N.EXPORTS) | declared
    for name in declared:
        assert hasattr(L, name), name
    assert set(N.EXPORTS) == declared


def test_version_and_status_strings(L):
    assert b"sm_100a" in L.bpf_version()
    assert L.bpf_status_string(N.BPF_E_DEGENERATE).startswith(b"particle filter degenerated")


def test_invalid_arguments_rejected_on_host(L):
    from libbi_b200 import ModelL96, ModelPZ

    h = ctypes.c_void_p()
    cfg = N.Config()
    cfg.nparticles = 0
    cfg.ess_rel = 0.5
    d = ModelL96().desc()
    assert L.bpf_create(ctypes.byref(d), ctypes.byref(cfg), ctypes.byref(h)) == N.BPF_E_INVALID
    cfg.nparticles = 1024
    cfg.ess_rel = 1.5
    assert L.bpf_create(ctypes.byref(d), ctypes.byref(cfg), ctypes.byref(h)) == N.BPF_E_INVALID
    cfg.ess_rel = 0.5
    bad = ModelL96(dim=39).desc()
    assert L.bpf_create(ctypes.byref(bad), ctypes.byref(cfg), ctypes.byref(h)) == N.BPF_E_INVALID
    bad = ModelL96(sigma_y=0.0).desc()
    assert L.bpf_create(ctypes.byref(bad), ctypes.byref(cfg), ctypes.byref(h)) == N.BPF_E_INVALID
    bad = ModelPZ().desc()
    bad.precision = N.BPF_F32
    assert L.bpf_create(ctypes.byref(bad), ctypes.byref(cfg), ctypes.byref(h)) == N.BPF_E_INVALID
    cfg.resampler = 7
    assert L.bpf_create(ctypes.byref(d), ctypes.byref(cfg), ctypes.byref(h)) == N.BPF_E_INVALID
    r = ctypes.c_void_p()
    assert L.bpf_resampler_create(9, 100, 0, None, ctypes.byref(r)) == N.BPF_E_INVALID
    assert L.bpf_resampler_create(0, 0, 0, None, ctypes.byref(r)) == N.BPF_E_INVALID
    assert L.bpf_gather_rows(None, None, None, 1, 1, 1, 4, None) == N.BPF_E_INVALID


def test_python_api_refuses_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from libbi_b200 import BootstrapPF, ModelL96

    with pytest.raises(RuntimeError, match="no CPU fallback"):
        BootstrapPF(ModelL96(), 1024)


def build_cpp_client(outdir):
    """Compile tests/cpp/filter_client.cpp against include/libbi_b200.hpp and
    the built library; returns the executable's path."""
    import pathlib
    import subprocess

    root = pathlib.Path(__file__).resolve().parents[1]
    lib = root / "libbi_b200" / "_lib"
    exe = pathlib.Path(outdir) / "filter_client"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{root / 'include'}",
                    str(root / "tests" / "cpp" / "filter_client.cpp"), f"-L{lib}", "-lbi_b200",
                    f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    return exe


def test_cpp_interface_compiles(tmp_path):
    """The header-only C++ interface and a client in the shape of LibBi's
    filter client compile and link against the library (no GPU needed)."""
    exe = build_cpp_client(tmp_path)
    assert exe.exists()



def build_test_models(outdir, precision="double"):
    """Compile the models in the generated form (tests/cpp/test_models.cu:
    the reference's Test.bi AR(1) model and Lorenz '96, against
    include/bpf_model.cuh, -fmad=false) into a shared library; returns
    (path, ptxas report)."""
    import pathlib
    import subprocess

    root = pathlib.Path(__file__).resolve().parents[1]
    lib = root / "libbi_b200" / "_lib"
    out = pathlib.Path(outdir) / f"libtest_models_{precision}.so"
    r = subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-fmad=false",
                        f"-DBPF_REAL={precision}", f"-I{root / 'include'}", "-Xcompiler", "-fPIC", "-shared",
                        "-Xptxas", "-v", str(root / "tests" / "cpp" / "test_models.cu"), f"-L{lib}", "-lbi_b200",
                        "-Xlinker", f"-rpath={lib}", "-o", str(out)], capture_output=True, text=True, check=True)
    return out, r.stderr


@pytest.mark.parametrize("precision", ["double", "float"])
def test_generated_form_models_compile_without_local_memory(L, tmp_path, precision):
    """A model class in the shape LibBi's generator emits compiles against
    include/bpf_model.cuh (cross-compiled for sm_100a, no GPU needed), and
    every variable fetch of its actions resolves to a register or shared
    memory: no state array is placed in local memory (a 40-element array
    would take 160 bytes or more of stack), only a few spilled registers at
    the register cap."""
    import re as _re

    so, report = build_test_models(tmp_path, precision)
    assert so.exists()
    blocks = _re.findall(r"Function properties for (\S*k_model_\S*)\n\s*(\d+) bytes stack frame, (\d+) bytes spill "
                         r"stores, (\d+) bytes spill loads", report)
    assert len(blocks) == 4, report
    for name, frame, st, ld in blocks:
        assert int(frame) <= 32 and int(st) <= 64 and int(ld) <= 64, (name, frame, st, ld)


# the oracle's kinds for the generated-form models (oracle/bpf_oracle.c)
ORC_MODEL_TEST_AR1 = 101
ORC_MODEL_L96_GEN = 102


def ar1_desc(precision, theta=0.9, sigma2=0.25):
    """Oracle description of tests/cpp/model_test_ar1.cuh (precision:
    N.BPF_F32 or N.BPF_F64)."""
    d = N.ModelDesc()
    d.kind, d.dim, d.precision, d.h = ORC_MODEL_TEST_AR1, 1, precision, 1.0
    d.theta[0], d.theta[1] = theta, sigma2
    return d


def l96_gen_desc(precision, F):
    """Oracle description of tests/cpp/model_l96_generated.cuh."""
    d = N.ModelDesc()
    d.kind, d.dim, d.precision, d.h = ORC_MODEL_L96_GEN, 40, precision, 0.01
    for i, v in enumerate((F, 0.1, 1.0, F, 0.01)):
        d.theta[i] = v
    return d


def test_oracle_runs_generated_form_models():
    """The oracle's restatements of the generated-form models (AR(1) and
    Lorenz '96) run a filter on the CPU."""
    import numpy as np

    from oracle.oracle import Oracle

    O = Oracle()
    for desc, nobs in ((ar1_desc(N.BPF_F64), 1), (l96_gen_desc(N.BPF_F32, 8.0), 40)):
        cfg = N.Config()
        cfg.nparticles, cfg.resampler, cfg.ess_rel, cfg.seed = 256, N.BPF_RESAMPLER_SYSTEMATIC, 0.5, 3
        dt = np.float32 if desc.precision == N.BPF_F32 else np.float64
        y = np.random.default_rng(1).standard_normal((5, nobs)).astype(dt)
        out = O.filter(desc, cfg, y, 5, 0.0, 1.0 if nobs == 1 else 0.05)
        assert out["rc"] == 0 and np.isfinite(out["ll"])
