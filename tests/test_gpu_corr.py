"""Correlation bins on the device (marked gpu): one batched launch over tasks
of mixed shapes gives each task the values its own slsf_task_correlations
gives, bit for bit, and the oracle's within the FP32 bar; the bins sum the
measurements in order; set-up, budget and misuse errors."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [((8, 8, 8), 4, 4), ((16, 12, 20), 5, 10), ((2, 2, 2), 1, 1), ((6, 10, 4), 3, 0), ((32, 48, 30), 24, 9),
          ((40, 24, 256), 3, 128), ((64, 64, 64), 32, 32), ((4, 4, 12), 0, 6)]


@pytest.fixture(scope="module")
def ctx(slsf):
    slsf.build()
    c = slsf.Context()
    yield c
    c.close()


def task(slsf, ctx, orc, dims, seed):
    jxy, jz = np.full(dims[2], 1.0), orc.uniform_disorder(dims[2], 0.5, 1.5, seed)
    t = slsf.Task(ctx, dims, jxy, jz, 1.2, seed=seed)
    t.init_random()
    return t


def flat(c):
    return np.concatenate([c["corr_x"], c["corr_y"], c["corr_xy"], c["corr_xy_by_z"].ravel(), c["corr_z"]])


def test_batched_equals_single_task_and_oracle(slsf, ctx, orc):
    tasks = [task(slsf, ctx, orc, d, 10 + k) for k, (d, _, _) in enumerate(SHAPES)]
    for t, (d, rxy, rz) in zip(tasks, SHAPES):
        nv = t.corr_setup(rxy, rz, 1, 3)
        R, Rz = min(rxy, d[0] // 2, d[1] // 2), min(rz, d[2] // 2)
        assert nv == 3 * R + d[2] * R + Rz
    expect = [[] for _ in tasks]
    for step in range(3):
        ctx.batch_run(tasks, 1 + step)
        for i, (t, (d, rxy, rz)) in enumerate(zip(tasks, SHAPES)):
            expect[i].append(flat(t.correlations(rxy, rz)))
        ctx.batch_correlations(tasks)
    for i, (t, (d, rxy, rz)) in enumerate(zip(tasks, SHAPES)):
        means, count = t.corr_bins()
        assert count == 3 and means.shape == (3, t.corr_n_values)
        # bins of one measurement: the mean is the value itself
        assert np.array_equal(means, np.array(expect[i])), d
        R, Rz = min(rxy, d[0] // 2, d[1] // 2), min(rz, d[2] // 2)
        ref = orc.correlations_f32(d, t.theta, R, Rz)
        got = expect[i][-1]
        assert np.allclose(got[:R], ref["corr_x"], atol=2e-6)
        assert np.allclose(got[R:2 * R], ref["corr_y"], atol=2e-6)
        assert np.allclose(got[3 * R:3 * R + d[2] * R], ref["corr_xy_by_z"].ravel(), atol=5e-6)
        assert np.allclose(got[3 * R + d[2] * R:], ref["corr_z"], atol=2e-6)
    for t in tasks:
        t.close()


def test_bins_sum_in_measurement_order(slsf, ctx, orc):
    a, b = task(slsf, ctx, orc, (8, 8, 8), 1), task(slsf, ctx, orc, (12, 8, 6), 2)
    for t in (a, b):
        t.corr_setup(4, 3, 3, 2)  # two bins of three; the seventh measurement is not kept
    series = {id(a): [], id(b): []}
    for _ in range(7):
        ctx.batch_run([a, b], 1)
        for t in (a, b):
            series[id(t)].append(flat(t.correlations(4, 3)))
        ctx.batch_correlations([b, a])  # order of the batch does not matter
    for t in (a, b):
        means, count = t.corr_bins()
        assert count == 7
        s = np.array(series[id(t)])
        for row in range(2):
            acc = np.zeros(s.shape[1])
            for k in range(3):
                acc = acc + s[3 * row + k]
            assert np.array_equal(means[row], acc / 3.0)
        # re-setup resets the count and the bins
        t.corr_setup(4, 3, 3, 2)
        m2, c2 = t.corr_bins()
        assert c2 == 0 and not m2.any()
        t.close()


def test_setup_and_misuse_errors(slsf, ctx, orc):
    before, _ = ctx.memory()
    t = task(slsf, ctx, orc, (8, 8, 8), 3)
    u = task(slsf, ctx, orc, (8, 8, 8), 4)
    with pytest.raises(slsf.SlsfError) as e:
        ctx.batch_correlations([t])
    assert e.value.code == slsf.ERR_STATE and "slsf_task_corr_setup" in str(e.value)
    with pytest.raises(slsf.SlsfError) as e:
        t.corr_setup(2, 2, 0, 4)
    assert "binsize must be positive" in str(e.value)
    assert t.corr_setup(0, 0, 1, 4) == 0  # nothing to measure: no bins
    used0, _ = ctx.memory()
    t.corr_setup(4, 4, 1, 8)
    u.corr_setup(1, 0, 1, 1)
    assert ctx.memory()[0] > used0
    with pytest.raises(slsf.SlsfError) as e:
        ctx.batch_correlations([t, u, t])
    assert e.value.code == slsf.ERR_INVALID and "twice" in str(e.value)
    with pytest.raises(slsf.SlsfError) as e:
        t.corr_bins(9)
    assert "more bin rows requested than the task keeps" in str(e.value)
    long = slsf.Task(ctx, (800, 2, 2), np.ones(2), np.ones(2), 1.0)
    with pytest.raises(slsf.SlsfError) as e:
        long.corr_setup(1, 1, 1, 1)
    assert "longer than 775 sites" in str(e.value)
    with pytest.raises(slsf.SlsfError) as e:
        long.correlations(1, 1)
    assert "longer than 775 sites" in str(e.value)
    long.close()
    t.close()
    u.close()
    assert ctx.memory()[0] == before  # the bins went with their tasks


def test_budget_counts_correlation_bins(slsf, orc):
    one = slsf.load().slsf_task_bytes(8, 8, 8, 0)
    with slsf.Context(budget_bytes=one + 4096) as small:
        t = task(slsf, small, orc, (8, 8, 8), 5)
        with pytest.raises(slsf.SlsfError) as e:
            t.corr_setup(4, 4, 1, 1000)
        assert e.value.code == slsf.ERR_BUDGET
        assert t.corr_setup(1, 1, 1, 1) > 0
        t.close()


def test_session_cycles_equal_manual_cycles(slsf, ctx, orc):
    # slsf_batch_step_correlations: k x (session step of `interval` sweeps +
    # one correlation measurement) equals the same cycles done by hand.
    shapes = [(8, 8, 8), (16, 12, 20), (32, 32, 32), (48, 48, 48), (12, 8, 6)]
    interval, cycles = 3, 5

    def make():
        ts = []
        for k, d in enumerate(shapes):
            t = task(slsf, ctx, orc, d, 40 + k)
            t.corr_setup(d[0] // 2, d[2] // 2, 2, 3)
            ts.append(t)
        return ts

    a, b = make(), make()
    with ctx.session(a, interval) as ses:
        st = ses.step_correlations(cycles)
    manual = np.zeros((len(b), 4), dtype=np.uint64)
    for _ in range(cycles):
        for i, s in enumerate(ctx.batch_run(b, interval)):
            manual[i] += np.array([s["sweeps"], s["accepted"], s["wolff_clusters"], s["wolff_cluster_sites"]],
                                  dtype=np.uint64)
        ctx.batch_correlations(b)
    assert np.array_equal(st, manual)
    for x, y in zip(a, b):
        assert x.counters == y.counters == (interval * cycles, interval * cycles)
        assert np.array_equal(x.theta.view(np.uint32), y.theta.view(np.uint32))
        cx, nx = x.corr_bins()
        cy, ny = y.corr_bins()
        assert nx == ny == cycles and np.array_equal(cx, cy)
        x.close()
        y.close()


@pytest.mark.parametrize("dims,rxy,rz", [((4, 4, 500), 2, 250), ((4, 2, 260), 1, 130), ((8, 8, 40), 4, 20)])
def test_tall_lattices_many_lags(slsf, ctx, orc, dims, rxy, rz):
    # radii beyond the small launch sizes, few z items: every lag is formed
    t = task(slsf, ctx, orc, dims, 3)
    t.sweep(1)
    R, Rz = min(rxy, dims[0] // 2, dims[1] // 2), min(rz, dims[2] // 2)
    got = t.correlations(rxy, rz)
    ref = orc.correlations_f32(dims, t.theta, R, Rz)
    assert np.allclose(got["corr_z"], ref["corr_z"], atol=2e-6)
    assert np.allclose(got["corr_x"], ref["corr_x"], atol=2e-6)
    t.corr_setup(rxy, rz, 1, 1)
    ctx.batch_correlations([t])
    means, _ = t.corr_bins()
    assert np.array_equal(means[0], flat(got))
    t.close()


@pytest.mark.parametrize("interval", [1, 3])
def test_fused_correlations_equal_separate(slsf, ctx, orc, interval):
    # In-kernel measurement (one-CTA kernel, replica in shared memory) against
    # the separate kernels on the same trajectory: same counts and bins to
    # FP32 partial-sum rounding.
    shapes = [(8, 8, 8), (16, 12, 20), (32, 32, 32), (6, 10, 4), (12, 8, 6), (4, 4, 12)]
    therm, sweeps = 2, 9
    n_corr = (sweeps + interval - 1) // interval

    def make(fused):
        ts = []
        for k, d in enumerate(shapes):
            jxy, jz = np.full(d[2], 1.0), orc.uniform_disorder(d[2], 0.5, 1.5, 60 + k)
            t = slsf.Task(ctx, d, jxy, jz, 1.2, seed=60 + k, thermalization=therm, binsize=3, n_bins=3)
            t.init_random()
            t.corr_setup(d[0] // 2, d[2] // 2, 1, n_corr)
            if fused:
                t.corr_fuse(interval)
            ts.append(t)
        return ts

    fused, sep = make(True), make(False)
    ctx.batch_run(fused, therm + 4)
    ctx.batch_run(fused, sweeps - 4)  # the measurement schedule continues across launches
    ctx.batch_run(sep, therm)
    done = 0
    for m in range(0, sweeps, interval):
        ctx.batch_run(sep, m + 1 - done)
        done = m + 1
        ctx.batch_correlations(sep)
    ctx.batch_run(sep, sweeps - done)
    for a, b in zip(fused, sep):
        assert np.array_equal(a.theta.view(np.uint32), b.theta.view(np.uint32))
        ma, na = a.corr_bins()
        mb, nb = b.corr_bins()
        assert na == nb == n_corr
        assert np.allclose(ma, mb, rtol=0, atol=2e-6), a.dims
        a.close()
        b.close()


def test_fused_correlations_on_the_grid_path_equal_separate(slsf, ctx, orc):
    # A lattice too large for one cluster's shared memory runs through the
    # grid-wide kernels; with slsf_task_corr_fuse its correlations are launched
    # after every interval-th sweep inside the same batched call, with no host
    # round trip per sweep: the same kernels as the separate measurement, so
    # the same bits.
    d, therm, sweeps, interval = (128, 32, 32), 1, 5, 2
    n_corr = (sweeps - therm + interval - 1) // interval
    jxy, jz = np.full(d[2], 1.2), orc.uniform_disorder(d[2], 0.5, 1.5, 80)

    def make():
        t = slsf.Task(ctx, d, jxy, jz, 1.3, seed=80, thermalization=therm, binsize=2, n_bins=2)
        t.init_random()
        t.corr_setup(8, d[2] // 2, 1, n_corr)
        return t

    ctx.tune_set(d, "grid", 1, 256)
    fused, sep = make(), make()
    fused.corr_fuse(interval)
    ctx.batch_run([fused], sweeps)
    ctx.batch_run([sep], therm)
    done = therm
    for m in range(0, sweeps - therm, interval):
        ctx.batch_run([sep], therm + m + 1 - done)
        done = therm + m + 1
        ctx.batch_correlations([sep])
    ctx.batch_run([sep], sweeps - done)
    assert np.array_equal(fused.theta.view(np.uint32), sep.theta.view(np.uint32))
    ma, na = fused.corr_bins()
    mb, nb = sep.corr_bins()
    assert na == nb == n_corr
    assert np.array_equal(ma, mb)
    ba, _ = fused.bins()
    bb, _ = sep.bins()
    assert np.array_equal(ba, bb)
    fused.close()
    sep.close()


def test_fused_in_sessions_and_refusals(slsf, ctx, orc):
    t = task(slsf, ctx, orc, (16, 16, 16), 70)
    with pytest.raises(slsf.SlsfError) as e:
        t.corr_fuse(1)
    assert e.value.code == slsf.ERR_STATE  # no bins yet
    t.corr_setup(8, 8, 2, 4)
    t.corr_fuse(1)
    with pytest.raises(slsf.SlsfError) as e:
        ctx.batch_correlations([t])
    assert e.value.code == slsf.ERR_STATE and "inside the batched sweeps" in str(e.value)
    with ctx.session([t], 4) as ses:
        ses.step()
        ses.step()
        with pytest.raises(slsf.SlsfError):
            ses.step_correlations(1)
    _, n = t.corr_bins()
    assert n == 8
    big = task(slsf, ctx, orc, (48, 48, 48), 71)  # the cluster kernel by default
    big.corr_setup(4, 4, 1, 1)
    with pytest.raises(slsf.SlsfError) as e:
        big.corr_fuse(1)
    assert "one-CTA kernel" in str(e.value) and "grid-wide kernels" in str(e.value)
    # a shape that fits the one-CTA kernel but is tuned to the cluster kernel
    small = task(slsf, ctx, orc, (12, 12, 12), 72)
    small.corr_setup(6, 6, 1, 1)
    ctx.tune_set((12, 12, 12), "cluster", 1, 512)
    with pytest.raises(slsf.SlsfError) as e:
        small.corr_fuse(1)
    assert "one-CTA kernel" in str(e.value)
    ctx.tune_set((12, 12, 12), "resident", 1, 128)
    small.corr_fuse(1)
    t.close()
    big.close()
    small.close()
