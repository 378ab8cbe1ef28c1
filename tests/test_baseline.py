"""The timed CPU baseline (oracle/baseline_simd.cpp) against the scalar oracle (CPU).

The baseline is the oracle's reference-order path with the Metropolis
batches' sincos and exp on glibc's vector math library, as the reference's
batches run on sleef's (src/updates.rs:21-53, :300-408).  Vector and scalar
functions differ in the last bits, so trajectories part after a while; the
equilibrium must not: at L = 8, T = 1.1 the two agree on <E> and <m^2> over
independent replicas within 3 sigma.
"""
import math

import numpy as np


def test_simd_baseline_loads_the_host_build(orc):
    cpu = orc.host_cpu()
    lib = orc.baseline_lib()
    assert lib.name == ("libbaseline_v4.so" if cpu["avx512f"] else "libbaseline_v3.so")
    assert cpu["physical_cores"] >= 1 and cpu["logical_cpus"] >= 1


def test_simd_baseline_equilibrium_equals_oracle(orc):
    L, T, R, therm, meas = 8, 1.1, 32, 100, 400
    jxy = np.full(L, 1.2)
    jz = orc.uniform_disorder(L, 0.5, 1.5, 20260710)
    args = ((L, L, L), np.tile(jxy, (R, 1)), np.tile(jz, (R, 1)), [T] * R)
    scalar = orc.series_tasks(*args, [10 + r for r in range(R)], therm, meas, 20)
    simd = orc.series_tasks(*args, [5000 + r for r in range(R)], therm, meas, 20, simd=True)
    for col in (0, 2):
        a, b = scalar[:, :, col].mean(axis=1), simd[:, :, col].mean(axis=1)
        z = (a.mean() - b.mean()) / math.sqrt(a.var(ddof=1) / R + b.var(ddof=1) / R)
        assert abs(z) < 3.0, (col, a.mean(), b.mean(), z)


def test_simd_baseline_first_sweep_follows_the_oracle(orc):
    # Same seed, same draw order: the first sweep's energies agree to the
    # vector functions' rounding unless a decision flips on a near-tie.
    L = 8
    jxy = np.full(L, 1.2)
    jz = orc.uniform_disorder(L, 0.5, 1.5, 7)
    args = ((L, L, L), jxy[None, :], jz[None, :], [1.3], [99], 0, 1, 1)
    a = orc.series_tasks(*args)
    b = orc.series_tasks(*args, simd=True)
    assert abs(a[0, 0, 0] - b[0, 0, 0]) < 1e-9
