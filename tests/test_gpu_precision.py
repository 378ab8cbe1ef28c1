"""Measured precision of the device observables against FP64 (marked gpu).

The reference accumulates every observable in FP64 from FP64 angles
(src/observables.rs:80-154).  The device keeps FP32 angles, evaluates each
site's bond terms in FP32 with fast sincos, and sums them in FP64.  On the
same FP32 state, the oracle's `measure_f32` evaluates the reference's
formulas in FP64 throughout; the difference is the error the device's
arithmetic adds.  This test measures it on states of the benchmarked sizes
-- L = 32 (batched replicas), L = 64 (single large replica), L = 256 (large
lattice near the transition) -- for the single-task measurement
(`slsf_task_measure`) and for the measurement the batched kernels fuse into
their sweeps (read from per-sweep bins of one bin row per sweep), prints a
table of max / mean absolute and relative errors, and holds them to the
parity bars:
  |d(E/V)| < 2e-5, |d m^2| < 1e-5, |d helicity sum| < 2e-5 V.
Relative errors are |d| / |value|; for the sin sums, whose values are
fluctuations around zero, the table gives |d| / V instead.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("energy", "magnetization_squared", "cos_x", "cos_y", "cos_z", "sin_x", "sin_y", "sin_z")
BIN_COL = {"energy": 0, "magnetization_squared": 2, "cos_x": 3, "cos_y": 4, "cos_z": 5, "sin_x": 6, "sin_y": 7,
           "sin_z": 8}
BASE_SEED = 20260710


@pytest.fixture(scope="module")
def ctx(slsf):
    slsf.build()
    c = slsf.Context()
    yield c
    c.close()


def errors(rows, volume):
    """rows: list of (device dict, oracle dict). Max / mean abs and rel error per field."""
    out = {}
    for f in FIELDS:
        d = np.array([abs(g[f] - r[f]) for g, r in rows])
        if f.startswith("sin"):
            rel = d / volume
        else:
            rel = d / np.array([max(abs(r[f]), 1e-300) for _, r in rows])
        out[f] = (d.max(), d.mean(), rel.max(), rel.mean())
    return out


def check_and_print(label, errs, volume):
    print(f"precision {label}:")
    for f, (amax, amean, rmax, rmean) in errs.items():
        kind = "|d|/V" if f.startswith("sin") else "rel"
        print(f"  {f:<22s} abs max {amax:.2e} mean {amean:.2e}  {kind} max {rmax:.2e} mean {rmean:.2e}")
    assert errs["energy"][0] < 2e-5
    assert errs["magnetization_squared"][0] < 1e-5
    for f in FIELDS[2:]:
        assert errs[f][0] < 2e-5 * volume


@pytest.mark.parametrize("L,T,states,kernel", [(32, 1.3, 8, ("resident", 1, 1024)),
                                               (64, 1.3, 8, ("cluster", 8, 1024)),
                                               (256, 1.22, 3, None)])
def test_observable_error_against_fp64(slsf, ctx, orc, L, T, states, kernel):
    dims = (L, L, L)
    jxy = np.full(L, 1.2)
    jz = slsf.uniform_layer_disorder(L, 0.5, 1.5, BASE_SEED)
    jx32, jz32 = jxy.astype(np.float32), jz.astype(np.float32)
    seed = slsf.task_seed(BASE_SEED, L, 1, T)
    v = float(L ** 3)
    # single-task path: measure after each sweep, the oracle on the same state
    plain = slsf.Task(ctx, dims, jxy, jz, T, wolff_steps=1, seed=seed)
    plain.init_random()
    rows, thetas = [], []
    for _ in range(states):
        plain.sweep(1)
        th = plain.theta
        thetas.append(th)
        rows.append((plain.measure(), orc.measure_f32(dims, th, jx32, jz32)))
    plain.close()
    check_and_print(f"L={L} single-task measurement", errors(rows, v), v)
    if kernel is None:
        return
    # batched path: the measurement fused into the sweeps, one bin row per
    # sweep; the trajectory is bit-identical to the single-task one
    ctx.tune_set(dims, *kernel)
    t = slsf.Task(ctx, dims, jxy, jz, T, wolff_steps=1, seed=seed, thermalization=0, binsize=1, n_bins=states)
    t.init_random()
    ctx.batch_run([t], states)
    assert np.array_equal(t.theta.view(np.uint32), thetas[-1].view(np.uint32))
    bins, m = t.bins()
    assert m == states
    t.close()
    fused = []
    for s in range(states):
        got = {f: bins[s, BIN_COL[f]] for f in FIELDS}
        fused.append((got, rows[s][1]))
    check_and_print(f"L={L} batched fused measurement ({kernel[0]})", errors(fused, v), v)
