"""The batched persistent kernel against the single-task path and the oracle (marked gpu).

The batched kernel and the single-task kernels share the decision code and
the Philox keys, so a task's trajectory is bit-identical whichever path runs
it and whatever else shares the launch.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(slsf):
    slsf.build()
    c = slsf.Context()
    yield c
    c.close()


def couplings(orc, lz, seed):
    return np.full(lz, 1.2), orc.uniform_disorder(lz, 0.5, 1.5, seed)


def plain_run(slsf, ctx, orc, dims, T, seed, sweeps, wolff, therm=0, binsize=1, n_bins=0, dseed=1):
    jxy, jz = couplings(orc, dims[2], dseed)
    t = slsf.Task(ctx, dims, jxy, jz, T, wolff_steps=wolff, seed=seed, thermalization=therm, binsize=binsize,
                  n_bins=n_bins)
    t.init_random()
    series = []
    for s in range(sweeps):
        t.sweep(1)
        if s + 1 > therm:
            series.append(t.measure())
    return t, series


def batched_tasks(slsf, ctx, orc, specs):
    out = []
    for dims, T, seed, wolff, therm, binsize, n_bins, dseed in specs:
        jxy, jz = couplings(orc, dims[2], dseed)
        t = slsf.Task(ctx, dims, jxy, jz, T, wolff_steps=wolff, seed=seed, thermalization=therm, binsize=binsize,
                      n_bins=n_bins)
        t.init_random()
        out.append(t)
    return out


@pytest.mark.parametrize("dims,wolff", [((8, 8, 8), 0), ((8, 8, 8), 1), ((32, 32, 32), 1), ((16, 8, 12), 2),
                                        ((24, 24, 24), 1), ((32, 16, 8), 1), ((12, 10, 6), 1),
                                        ((32, 32, 48), 1), ((32, 32, 96), 1), ((20, 24, 16), 1),
                                        ((48, 48, 48), 1), ((64, 64, 64), 1), ((40, 16, 8), 1), ((64, 8, 6), 1),
                                        ((8, 6, 6), 1), ((4, 4, 10), 2), ((4, 2, 2), 1), ((16, 10, 2), 1),
                                        ((64, 6, 10), 1), ((6, 6, 6), 1), ((10, 10, 10), 2), ((14, 6, 8), 1),
                                        ((18, 18, 18), 1), ((30, 8, 4), 1), ((34, 34, 34), 1), ((50, 10, 8), 1),
                                        ((26, 12, 6), 1), ((28, 6, 10), 2)])
def test_batched_equals_plain_bitwise(slsf, ctx, orc, dims, wolff):
    ref, _ = plain_run(slsf, ctx, orc, dims, 1.1, seed=42, sweeps=4, wolff=wolff)
    [t] = batched_tasks(slsf, ctx, orc, [(dims, 1.1, 42, wolff, 0, 1, 0, 1)])
    stats = ctx.batch_run([t], 4)
    assert np.array_equal(t.theta.view(np.uint32), ref.theta.view(np.uint32))
    assert t.counters == ref.counters
    assert stats[0]["sweeps"] == 4


def test_same_alone_and_in_the_mix(slsf, ctx, orc):
    specs = [((8, 8, 8), 1.0, 1, 1, 0, 1, 0, 1), ((16, 16, 16), 1.3, 2, 1, 0, 1, 0, 2),
             ((32, 32, 32), 1.5, 3, 1, 0, 1, 0, 3), ((24, 24, 24), 1.2, 4, 1, 0, 1, 0, 4),
             ((8, 16, 4), 0.9, 5, 2, 0, 1, 0, 5), ((48, 48, 48), 1.1, 6, 1, 0, 1, 0, 6)] * 2 + \
            [((64, 64, 64), 1.4, 7, 1, 0, 1, 0, 7)]
    mix = batched_tasks(slsf, ctx, orc, specs)
    ctx.batch_run(mix, 5)
    for spec, t in zip(specs, mix):
        [alone] = batched_tasks(slsf, ctx, orc, [spec])
        ctx.batch_run([alone], 5)
        assert np.array_equal(t.theta.view(np.uint32), alone.theta.view(np.uint32))


def test_bins_match_plain_measure_stream(slsf, ctx, orc):
    dims, T = (8, 8, 8), 1.1
    therm, binsize, sweeps = 3, 4, 19
    n_bins = (sweeps - therm + binsize - 1) // binsize
    ref, series = plain_run(slsf, ctx, orc, dims, T, seed=8, sweeps=sweeps, wolff=1, therm=therm, binsize=binsize)
    [t] = batched_tasks(slsf, ctx, orc, [(dims, T, 8, 1, therm, binsize, n_bins, 1)])
    ctx.batch_run([t], 7)
    ctx.batch_run([t], sweeps - 7)  # bins continue across launches
    bins, m = t.bins()
    assert m == sweeps - therm
    v = t.volume
    rows = []
    for o in series:
        rows.append([o["energy"], o["energy"] ** 2, o["magnetization_squared"], o["cos_x"], o["cos_y"], o["cos_z"],
                     o["sin_x"], o["sin_y"], o["sin_z"], o["sin_x"] ** 2, o["sin_y"] ** 2, o["sin_z"] ** 2])
    rows = np.array(rows)
    # The batched kernels measure inside the next sweep's colour-0 half-sweep
    # (the launch's last state in a separate pass); both paths sum the same
    # FP32 bond terms in FP64, in different orders.
    for b in range(n_bins):
        expect = rows[b * binsize:(b + 1) * binsize].mean(axis=0)
        assert np.allclose(bins[b], expect, rtol=1e-10, atol=1e-10 * v), (b, bins[b], expect)


def test_checkpoint_resume_is_bit_exact(slsf, ctx, orc):
    # Philox keys depend only on (seed, counters, site): N + N sweeps == 2N sweeps.
    dims = (16, 16, 16)
    [a] = batched_tasks(slsf, ctx, orc, [(dims, 1.2, 9, 1, 0, 1, 0, 1)])
    ctx.batch_run([a], 6)
    [b] = batched_tasks(slsf, ctx, orc, [(dims, 1.2, 9, 1, 0, 1, 0, 1)])
    ctx.batch_run([b], 3)
    saved_theta, saved_counters = b.theta, b.counters
    [c] = batched_tasks(slsf, ctx, orc, [(dims, 1.2, 9, 1, 0, 1, 0, 1)])
    c.theta = saved_theta
    c.counters = saved_counters
    ctx.batch_run([c], 3)
    assert np.array_equal(a.theta.view(np.uint32), c.theta.view(np.uint32))
    assert a.counters == c.counters


def test_batched_grid_tasks_in_the_mix(slsf, ctx, orc):
    # Lattices too large for one cluster's shared memory run through the
    # grid-wide kernels inside the same batch call: same trajectory as the
    # single-task path, bins equal to the plain measure stream.
    dims, T, therm, binsize, sweeps = (128, 4, 4), 1.2, 1, 2, 5
    n_bins = (sweeps - therm) // binsize
    ref, series = plain_run(slsf, ctx, orc, dims, T, seed=11, sweeps=sweeps, wolff=1, therm=therm)
    specs = [(dims, T, 11, 1, therm, binsize, n_bins, 1), ((8, 8, 8), 1.0, 3, 1, 0, 1, 0, 2),
             ((48, 48, 48), 1.1, 6, 1, 0, 1, 0, 6)]
    mix = batched_tasks(slsf, ctx, orc, specs)
    stats = ctx.batch_run(mix, sweeps)
    big = mix[0]
    assert np.array_equal(big.theta.view(np.uint32), ref.theta.view(np.uint32))
    assert big.counters == ref.counters
    assert stats[0]["sweeps"] == sweeps and stats[0]["wolff_clusters"] == sweeps
    bins, m = big.bins()
    assert m == sweeps - therm
    rows = np.array([[o["energy"], o["energy"] ** 2, o["magnetization_squared"], o["cos_x"], o["cos_y"], o["cos_z"],
                      o["sin_x"], o["sin_y"], o["sin_z"], o["sin_x"] ** 2, o["sin_y"] ** 2, o["sin_z"] ** 2]
                     for o in series])
    for b in range(n_bins):
        # the same FP32 bond terms on both paths (the grid path measures most states inside the next
        # sweep's colour-0 kernel): equal up to the FP64 summation and averaging order
        assert np.allclose(bins[b], rows[b * binsize:(b + 1) * binsize].mean(axis=0), rtol=1e-12, atol=1e-12)
    for spec, t in zip(specs[1:], mix[1:]):
        [alone] = batched_tasks(slsf, ctx, orc, [spec])
        ctx.batch_run([alone], sweeps)
        assert np.array_equal(t.theta.view(np.uint32), alone.theta.view(np.uint32))


def _binned(bin_means):
    """Mean and standard error over bins (BinnedEstimate, src/tests.rs:436-446)."""
    return bin_means.mean(axis=0), bin_means.std(axis=0, ddof=1) / math.sqrt(len(bin_means))


def test_two_sigma_config0(slsf, ctx, orc):
    """Config 0: L=8, J_xy=1.2, J_z ~ U[0.5,1.5] (one disorder draw), T=1.1, width pi,
    500 sweeps + 1 Wolff per sweep, measured every sweep; first 100 sweeps
    discarded.  R independent replicas per side; the replica means give the
    error bars.  Device: batched kernel (Philox streams); reference: the
    oracle's reference-order CPU path (FastRng streams)."""
    L, T, sweeps, therm = 8, 1.1, 500, 100
    R = 48
    jxy, jz = couplings(orc, L, 20260710)
    nbins = 25
    binsize = (sweeps - therm) // nbins
    tasks = [slsf.Task(ctx, (L, L, L), jxy, jz, T, wolff_steps=1, seed=1000 + r, thermalization=therm,
                       binsize=binsize, n_bins=nbins) for r in range(R)]
    for t in tasks:
        t.init_random()
    ctx.batch_run(tasks, sweeps)
    v, beta = float(L ** 3), 1.0 / T
    gpu = []
    for t in tasks:
        bins, _ = t.bins()
        gpu.append(bins.mean(axis=0))
    cpu = []
    for r in range(R):
        m = orc.Model(L, L, L, jxy, jz, T, wolff_steps=1, seed=5000 + r)
        m.init()
        series, _ = m.run_series(therm, sweeps - therm)
        cpu.append(series.mean(axis=0))
    gpu, cpu = np.array(gpu), np.array(cpu)

    def rho(c, k):  # rho_mu from replica means (src/model.rs:878-886)
        return c[:, 3 + k] / v - beta * (c[:, 9 + k] - c[:, 6 + k] ** 2) / v

    obs = {
        "Energy": (gpu[:, 0], cpu[:, 0]),
        "MagnetizationSquared": (gpu[:, 2], cpu[:, 2]),
        "RhoXY": ((rho(gpu, 0) + rho(gpu, 1)) / 2, (rho(cpu, 0) + rho(cpu, 1)) / 2),
        "RhoZ": (rho(gpu, 2), rho(cpu, 2)),
    }
    report = {}
    for name, (g, c) in obs.items():
        sigma = math.sqrt(g.var(ddof=1) / len(g) + c.var(ddof=1) / len(c))
        z = (g.mean() - c.mean()) / sigma
        report[name] = (g.mean(), c.mean(), sigma, z)
    print("config0 2-sigma:", report)
    for name, (_, _, _, z) in report.items():
        assert abs(z) < 2.0, (name, report)


def test_session_graph_replay_equals_batch_run(slsf, ctx, orc):
    # One step captured in a CUDA graph and replayed: same trajectories, bins and
    # counters as batch_run, with tasks of several kernels in the session.
    specs = [((8, 8, 8), 1.0, 1, 1, 2, 2, 4, 1), ((16, 16, 16), 1.3, 2, 1, 2, 2, 4, 2),
             ((32, 32, 32), 1.5, 3, 1, 2, 2, 4, 3), ((48, 48, 48), 1.1, 6, 1, 2, 2, 4, 6),
             ((24, 16, 32), 1.2, 7, 2, 2, 2, 4, 7)]
    a = batched_tasks(slsf, ctx, orc, specs)
    b = batched_tasks(slsf, ctx, orc, specs)
    with ctx.session(a, 3) as ses:
        for _ in range(3):
            st = ses.step()
        with pytest.raises(slsf.SlsfError) as e:
            a[0].sweep(1)  # the session owns the task's device view
        assert e.value.code == slsf.ERR_STATE
        assert a[0].counters == (9, 9) and a[4].counters == (9, 18)
    for _ in range(3):
        ref = ctx.batch_run(b, 3)
    for ta, tb in zip(a, b):
        assert np.array_equal(ta.theta.view(np.uint32), tb.theta.view(np.uint32))
        assert ta.counters == tb.counters
        ba, ma = ta.bins()
        bb, mb = tb.bins()
        assert ma == mb and np.array_equal(ba, bb)
    assert [s["accepted"] for s in st] == [s["accepted"] for s in ref]
    a[0].sweep(1)  # usable again after close


def test_wolff_dynamics_equal_metropolis_dynamics(slsf, ctx, orc):
    """Wolff against Metropolis, which the reference never checks: the same
    lattice (L=8, J_xy = 1.2, J_z ~ U[0.5, 1.5], T = 1.6) under Metropolis
    sweeps alone (width pi, no Wolff) and under Wolff updates alone (width 0,
    which accepts without moving, and three Wolff steps per sweep) reaches
    the same equilibrium: <E> and <m^2> over 48 independent replicas each
    agree within 3 sigma.  This pins the device's cluster labelling and
    reflection physically, without the oracle."""
    L, T, therm, sweeps, n_bins = 8, 1.6, 400, 1600, 16
    jxy, jz = couplings(orc, L, 20260710)

    def run(width, wolff, seed0):
        tasks = [slsf.Task(ctx, (L, L, L), jxy, jz, T, proposal_width=width, wolff_steps=wolff, seed=seed0 + r,
                           thermalization=therm, binsize=sweeps // n_bins, n_bins=n_bins) for r in range(48)]
        for t in tasks:
            t.init_random()
        ctx.batch_run(tasks, therm + sweeps)
        means = np.array([t.bins()[0].mean(axis=0) for t in tasks])
        for t in tasks:
            t.close()
        return means

    metro = run(math.pi, 0, 100)
    wolff = run(0.0, 3, 900)
    report = {}
    for name, col in (("Energy", 0), ("MagnetizationSquared", 2)):
        a, b = metro[:, col], wolff[:, col]
        sigma = math.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
        report[name] = (a.mean(), b.mean(), sigma, (a.mean() - b.mean()) / sigma)
    print("Metropolis vs Wolff:", report)
    for name, (_, _, _, z) in report.items():
        assert abs(z) < 3.0, (name, report)
