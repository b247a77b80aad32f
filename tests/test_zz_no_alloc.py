"""The allocation-free systematic resampler (bpf_systematic_ancestors_static).

It serves callers that cannot let the library allocate device memory, such
as an application that has reserved all of the GPU's memory for its own
allocator, or a real-time loop in which cudaMalloc is not allowed.  Its
scratch is a fixed array inside the library, shared by every call and kept
between calls, so this test calls it twice in a row on different inputs and
checks each result against the allocating entry point
(bpf_resampler_ancestors), which must agree exactly: ancestors are integers.
This file is collected last so that a failure here stops a -x run only after
every other test has run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_call(lw, a, permute, as_, Os):
    from libbi_b200 import _native as N

    return N.lib().bpf_systematic_ancestors_static(lw.data_ptr(), lw.numel(), None if a is None else a.data_ptr(),
                                                    int(permute), as_.data_ptr(),
                                                    None if Os is None else Os.data_ptr(), None)


def test_static_matches_allocating_entry_point_twice(cuda):
    import torch
    from libbi_b200 import SystematicResampler
    from libbi_b200 import _native as N

    ref = SystematicResampler(max_n=N.BPF_STATIC_MAX_PARTICLES)
    rng = np.random.default_rng(11)
    # two calls in a row, the second smaller and with different weights, so
    # that stale scratch from the first call would show
    for n, scale, permute in ((N.BPF_STATIC_MAX_PARTICLES, 3.0, 1), (20001, 0.5, 1), (777, 8.0, 0)):
        lw = torch.as_tensor(rng.standard_normal(n) * scale, device="cuda", dtype=torch.float64)
        a = torch.as_tensor(rng.random(1), device="cuda", dtype=torch.float64)
        as_ = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        Os = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        assert _static_call(lw, a, permute, as_, Os) == N.BPF_OK
        want_as, want_Os = ref.ancestors(lw, a, permute=bool(permute), with_offspring=True)
        np.testing.assert_array_equal(as_.cpu().numpy(), want_as.cpu().numpy())
        np.testing.assert_array_equal(Os.cpu().numpy(), want_Os.cpu().numpy())
    ref.close()


def test_static_rejects_oversize_and_degenerate(cuda):
    import torch
    from libbi_b200 import _native as N

    n = N.BPF_STATIC_MAX_PARTICLES + 1
    lw = torch.zeros(n, dtype=torch.float64, device="cuda")
    a = torch.full((1,), 0.5, dtype=torch.float64, device="cuda")
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    assert _static_call(lw, a, 1, out, out) == N.BPF_E_TOO_LARGE
    assert b"BPF_STATIC_MAX_PARTICLES" in N.lib().bpf_status_string(N.BPF_E_TOO_LARGE)
    bad = torch.full((100,), float("-inf"), dtype=torch.float64, device="cuda")
    o1 = torch.empty(100, dtype=torch.int32, device="cuda")
    o2 = torch.empty(100, dtype=torch.int32, device="cuda")
    assert _static_call(bad, a, 1, o1, o2) == N.BPF_E_DEGENERATE
    # the next call starts from cleared scratch
    ok = torch.zeros(100, dtype=torch.float64, device="cuda")
    assert _static_call(ok, a, 1, o1, o2) == N.BPF_OK
    np.testing.assert_array_equal(o1.cpu().numpy(), np.arange(100))


def test_static_built_in_offset_and_no_offspring_output(cuda):
    """Without a caller-supplied offset the library draws it from its own
    generator (the allocating entry point draws the same one), and without
    an Os buffer the cumulative offspring stay in the scratch array."""
    import torch
    from libbi_b200 import SystematicResampler
    from libbi_b200 import _native as N

    ref = SystematicResampler(max_n=N.BPF_STATIC_MAX_PARTICLES)
    rng = np.random.default_rng(5)
    for n in (40000, 513):
        lw = torch.as_tensor(rng.standard_normal(n) * 2.0, device="cuda", dtype=torch.float64)
        as_ = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        assert _static_call(lw, None, 1, as_, None) == N.BPF_OK
        want = ref.ancestors(lw, None, permute=True)
        np.testing.assert_array_equal(as_.cpu().numpy(), want.cpu().numpy())
    ref.close()


def test_static_matches_reference_golden_vectors(cuda, oracle, golden):
    """Tied to the reference's own output, not only to the other CUDA entry
    point: the golden cases that the reference's resampler code produced
    (cumulative offspring, permuted and sorted ancestors on the same
    offsets), for every case within the static limit."""
    import torch
    from libbi_b200 import _native as N
    from tests.golden.make_golden import UNIFORM_SEED

    checked = 0
    for name, c in golden.items():
        lw = c["lw"]
        n = lw.size
        if n > N.BPF_STATIC_MAX_PARTICLES:
            continue
        a = oracle.resample_uniforms(0, n, 0, UNIFORM_SEED, int(c["step"][0]))
        lw_d = torch.as_tensor(lw, device="cuda", dtype=torch.float64)
        a_d = torch.as_tensor(a, device="cuda", dtype=torch.float64)
        as_ = torch.empty(n, dtype=torch.int32, device="cuda")
        Os = torch.empty(n, dtype=torch.int32, device="cuda")
        assert _static_call(lw_d, a_d, 1, as_, Os) == N.BPF_OK, name
        np.testing.assert_array_equal(Os.cpu().numpy(), c["Os"], err_msg=name)
        np.testing.assert_array_equal(as_.cpu().numpy(), c["sys_perm"], err_msg=name)
        assert _static_call(lw_d, a_d, 0, as_, Os) == N.BPF_OK, name
        np.testing.assert_array_equal(as_.cpu().numpy(), c["sys_sorted"], err_msg=name)
        checked += 1
    assert checked >= 10
