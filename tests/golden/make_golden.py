"""Generate tests/golden/resampler_golden.npz from the reference's OWN
resampler and reduction code, compiled from the reference sources
(oracle/ref/ref_resampler.cpp -> oracle/_ref/libbiref.so, built by
`make -C oracle ref`), fed a tape of uniforms.

Uniforms are not stored: they are the documented counter-based draws
(include/bpf_philox.h) for seed UNIFORM_SEED at step = case index, exactly
what the CUDA path draws for a resample (oracle.Oracle.resample_uniforms).

Log-weight cases follow the reference's resampler test harness
(share/tt/cpp/test/test_resampler_cpu.cpp.tt:118-131): x ~ N(0,1) drawn once;
for Z = 0, 0.5, 1, ...: lw = log N(x; 0, 1) of the current x, then x += 0.5.
The Metropolis step count B follows the same harness (:156-162, C = 1).
Further edge cases: n = 1, 2 and tile-boundary sizes, equal weights, one
dominant weight, NaN and -inf entries.

Run from the repository root:  python tests/golden/make_golden.py
"""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import Oracle, RefResampler  # noqa: E402

HALF_LOG_TWO_PI = 0.91893853320467274178032973640562
UNIFORM_SEED = 7


def metropolis_steps(Z):
    EW = math.exp(-0.25 * Z * Z) / (2.0 * math.sqrt(math.pi))
    wmax = 1.0 / math.sqrt(math.pi)
    beta = EW / wmax
    return int(math.ceil(math.log(1.0e-2) / math.log(1.0 - beta)))


def cases(rng):
    out = []
    x = rng.standard_normal(1 << 12)
    for z in range(5):
        lp = -0.5 * x * x - HALF_LOG_TWO_PI
        x = x + 0.5
        for P in (16, 256, 4096):
            out.append((f"harness_z{z}_p{P}", lp[:P].copy(), metropolis_steps(0.5 * z)))
    out.append(("n1", np.array([-3.0]), 3))
    out.append(("n2", np.array([-1.0, 0.5]), 3))
    for n in (2047, 2048, 2049, 4097):
        out.append((f"ragged_{n}", rng.standard_normal(n) * 2.0, 4))
    out.append(("equal_1000", np.zeros(1000), 4))
    dom = np.full(3000, -50.0)
    dom[1234] = 0.0
    out.append(("dominant_3000", dom, 4))
    w = rng.standard_normal(2500)
    w[rng.integers(0, 2500, 40)] = np.nan
    w[rng.integers(0, 2500, 40)] = -np.inf
    out.append(("nan_inf_2500", w, 4))
    out.append(("wide_5000", rng.standard_normal(5000) * 30.0, 4))
    return out


def main():
    R = RefResampler()
    O = Oracle()
    rng = np.random.default_rng(20241203)
    data = {}
    names = []
    for idx, (name, lw, B) in enumerate(cases(rng)):
        n = lw.size
        a = float(O.resample_uniforms(0, n, B, UNIFORM_SEED, idx)[0])
        u_mult = O.resample_uniforms(1, n, B, UNIFORM_SEED, idx)
        u_metro = O.resample_uniforms(2, n, B, UNIFORM_SEED, idx)
        rc, _, Os, as_perm = R.systematic(lw, a, permute=True)
        assert rc == 0, name
        _, _, _, as_sorted = R.systematic(lw, a, permute=False)
        _, am = R.multinomial(lw, u_mult, permute=0)
        _, am_p = R.multinomial(lw, u_mult, permute=1)
        _, amh = R.metropolis(lw, B, u_metro, permute=0)
        _, amh_p = R.metropolis(lw, B, u_metro, permute=1)
        ess, lW = R.ess_reduce(lw)
        lse = R.logsumexp(lw)
        small = lambda v: v.astype(np.int16) if n < 32768 else v  # noqa: E731
        Os, as_perm, as_sorted, am, am_p, amh, amh_p = map(small, (Os, as_perm, as_sorted, am, am_p, amh, amh_p))
        for k, v in dict(lw=lw, step=np.array([idx]), Os=Os, sys_perm=as_perm, sys_sorted=as_sorted,
                         mult=am, mult_refperm=am_p, B=np.array([B]),
                         metro=amh, metro_refperm=amh_p, ess=np.array([ess]), lW=np.array([lW]),
                         lse=np.array([lse])).items():
            data[f"{name}/{k}"] = v
        names.append(name)
    data["names"] = np.array(names)
    path = os.path.join(ROOT, "tests", "golden", "resampler_golden.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path}: {len(names)} cases, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
