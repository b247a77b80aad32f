"""The benchmark workloads, by what they are.

pz_n4096:    plankton (PZ) model, RK4(3) h0=0.1 rtol=atol=1e-3, N=4096 FP64
             particles, systematic resampling whenever ESS < N (ess_rel=1),
             T=100 daily observations of log P with N(0, 0.2^2) noise.
l96_d40_n65536: Lorenz '96 d=40, F=8, RK4 h=0.01, N(0, 0.1^2) noise every
             0.05, all 40 components observed with N(0, 1) noise every 0.05,
             T=200, N=65536 FP32 particles, systematic at ESS < 0.5 N.
"""
from __future__ import annotations

import math

from .filter import ModelL96, ModelPZ

PZ_N4096 = dict(name="pz_n4096", model=ModelPZ(), nparticles=4096, resampler="systematic", ess_rel=1.0,
                T=100, t0=0.0, dt=1.0, seed=1, data_seed=101)
L96_D40_N65536 = dict(name="l96_d40_n65536", model=ModelL96(dim=40, F=8.0, sigma_eta=0.1, sigma_y=1.0, h=0.01,
                                                            x0_std=0.01, precision="f32"),
                      nparticles=65536, resampler="systematic", ess_rel=0.5, T=200, t0=0.0, dt=0.05, seed=2,
                      data_seed=102)
