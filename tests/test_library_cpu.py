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

