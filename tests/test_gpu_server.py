"""Host layer on the GPU (marked gpu): per-task sweep counts in one batched
call, the model driver on both paths, and the continuous-batching server
(results the same alone and in the mix, budget admission, validation,
cancellation, idle waits)."""
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
    return np.full(lz, 1.0), orc.uniform_disorder(lz, 0.5, 1.5, seed)


def make_task(slsf, ctx, orc, dims, T, seed, **kw):
    jxy, jz = couplings(orc, dims[2], seed)
    t = slsf.Task(ctx, dims, jxy, jz, T, seed=seed, **kw)
    t.init_random()
    return t


def test_batch_run_v_per_task_sweeps(slsf, ctx, orc):
    specs = [((16, 16, 16), 1.2, 1, 3), ((8, 8, 8), 0.9, 2, 7), ((32, 32, 32), 1.4, 3, 0), ((48, 48, 48), 1.1, 4, 2)]
    tasks = [make_task(slsf, ctx, orc, d, T, s) for d, T, s, _ in specs]
    before = [t.theta for t in tasks]
    sweeps = np.array([n for *_, n in specs], dtype=np.uint32)
    arr = ctx.handle_array(tasks)
    stats = (slsf.SweepStats * len(tasks))()
    slsf.check(slsf.load().slsf_batch_run_v(ctx.h, arr, len(tasks), sweeps.ctypes.data_as(slsf._U32P), stats))
    for (d, T, s, n), t, st, b0 in zip(specs, tasks, stats, before):
        assert st.sweeps == n
        assert t.counters == (n, n)
        if n == 0:
            assert np.array_equal(t.theta.view(np.uint32), b0.view(np.uint32))
            continue
        alone = make_task(slsf, ctx, orc, d, T, s)
        alone.sweep(n)
        assert np.array_equal(t.theta.view(np.uint32), alone.theta.view(np.uint32))


def test_model_run_batched_equals_plain(slsf, ctx):
    d = slsf.theta_task((8, 8, 8), 1.1, sweeps=48, thermalization=10, binsize=8, seed=77, disorder_seed=5,
                        j_xy=1.0, j_z_mean=1.0, delta_j_z=0.5)
    a = slsf.model_run(ctx, d, batched=True)
    b = slsf.model_run(ctx, d, batched=False)
    assert a["measurements"] == b["measurements"] == 48
    assert a["n_bins"] == b["n_bins"] == 6
    # same trajectory on both paths: identical acceptance; observables differ
    # only by the FP32 (batched) vs FP64 (grid kernel) reduction order
    assert a["acceptance"] == b["acceptance"]
    for name in slsf.BIN_NAMES + slsf.DERIVED:
        x, y = a[name][0], b[name][0]
        assert abs(x - y) <= 1e-4 * max(1.0, abs(y)), (name, x, y)


def requests(orc):
    # (tag, dims, T, seed, sweeps, thermalization, n_bins)
    return [(1, (8, 8, 8), 1.0, 11, 30, 5, 5), (2, (16, 16, 16), 1.3, 12, 55, 10, 9),
            (3, (32, 32, 32), 1.5, 13, 20, 4, 4), (4, (48, 48, 48), 1.1, 14, 25, 5, 2),
            (5, (16, 8, 12), 0.9, 15, 41, 1, 8), (6, (128, 4, 4), 1.2, 16, 12, 2, 5),
            (7, (24, 24, 24), 1.25, 17, 33, 3, 10)]


def drain(srv, limit=100000):
    """Runs epochs on this thread until nothing is queued or active."""
    for _ in range(limit):
        active, pending = srv.step()
        if active == 0 and pending == 0:
            return
    raise AssertionError("server did not drain")


def submit(srv, orc, req):
    tag, dims, T, seed, sweeps, therm, n_bins = req
    jxy, jz = couplings(orc, dims[2], seed)
    srv.submit(tag, dims, T, seed, jxy, jz, sweeps, thermalization=therm, n_bins=n_bins)


def test_server_results_same_alone_and_in_mix(slsf, ctx, orc):
    srv = slsf.Server(ctx, epoch_sweeps=10)
    for r in requests(orc):
        submit(srv, orc, r)
    srv.start()
    srv.wait_idle(120)
    srv.stop()
    mix = {r["tag"]: r for r in srv.poll()}
    st = srv.stats()
    srv.close()
    assert sorted(mix) == [r[0] for r in requests(orc)]
    assert st["completed"] == len(mix) and st["failed"] == 0
    for req in requests(orc):
        tag, dims, T, seed, sweeps, therm, n_bins = req
        got = mix[tag]
        assert got["status"] == slsf.OK, got["message"]
        assert got["sweeps"] == sweeps
        assert got["est"]["measurements"] == sweeps - therm
        assert got["submit_s"] <= got["admit_s"] <= got["finish_s"]
        one = slsf.Server(ctx, epoch_sweeps=10)
        submit(one, orc, req)
        drain(one)
        [alone] = one.poll()
        one.close()
        assert alone["accepted"] == got["accepted"] and alone["cluster_sites"] == got["cluster_sites"]
        for name in slsf.BIN_NAMES + slsf.DERIVED:
            assert alone["est"][name] == got["est"][name], (tag, name)


def test_server_result_matches_task_api(slsf, ctx, orc):
    # A served request equals the same task driven through the task API.
    tag, dims, T, seed, sweeps, therm, n_bins = 9, (16, 16, 16), 1.2, 21, 40, 8, 4
    srv = slsf.Server(ctx, epoch_sweeps=7)
    submit(srv, orc, (tag, dims, T, seed, sweeps, therm, n_bins))
    drain(srv)
    [res] = srv.poll()
    srv.close()
    binsize = (sweeps - therm) // n_bins
    t = make_task(slsf, ctx, orc, dims, T, seed, thermalization=therm, binsize=binsize, n_bins=n_bins)
    for n in (7, 7, 7, 7, 7, 5):
        ctx.batch_run([t], n)
    bins, m = t.bins()
    assert m == res["est"]["measurements"]
    assert np.allclose(bins.mean(axis=0), [res["est"][n][0] for n in slsf.BIN_NAMES], rtol=1e-14, atol=0)


def test_server_budget_admission(slsf, ctx, orc):
    one = slsf.load().slsf_task_bytes(16, 16, 16, 4)
    srv = slsf.Server(ctx, epoch_sweeps=5, budget_bytes=one + one // 2)
    for tag in (1, 2, 3):
        submit(srv, orc, (tag, (16, 16, 16), 1.2, tag, 12, 2, 4))
    submit(srv, orc, (4, (32, 32, 32), 1.2, 4, 12, 2, 4))
    drain(srv, 100)
    res = {r["tag"]: r for r in srv.poll()}
    st = srv.stats()
    srv.close()
    assert res[4]["status"] == slsf.ERR_BUDGET
    assert "does not fit in the server's device memory budget" in res[4]["message"]
    assert all(res[t]["status"] == slsf.OK for t in (1, 2, 3))
    assert st["peak_active"] == 1 and st["completed"] == 3 and st["failed"] == 1
    # FIFO: the three fitting requests finish in submission order
    assert res[1]["finish_s"] <= res[2]["admit_s"] and res[2]["finish_s"] <= res[3]["admit_s"]


@pytest.mark.parametrize("change,message", [
    (dict(dims=(7, 8, 8)), "red-black Metropolis sweep requires even lattice dimensions"),
    (dict(T=0.0), "temperature T must be positive and finite"),
    (dict(dims=(0, 8, 8)), "L_x must be positive"),
    (dict(width=-1.0), "proposal_width must be nonnegative and finite"),
    (dict(jz_value=-0.5), "theta simulation requires nonnegative layer couplings"),
])
def test_server_rejects_invalid_requests_alone(slsf, ctx, orc, change, message):
    srv = slsf.Server(ctx, epoch_sweeps=5)
    dims = change.get("dims", (8, 8, 8))
    jz = np.full(dims[2], change.get("jz_value", 1.0))
    srv.submit(1, dims, change.get("T", 1.0), 1, np.ones(dims[2]), jz, 10,
               proposal_width=change.get("width", np.pi))
    submit(srv, orc, (2, (8, 8, 8), 1.0, 2, 10, 0, 1))
    drain(srv)
    res = {r["tag"]: r for r in srv.poll()}
    srv.close()
    assert res[1]["status"] == slsf.ERR_INVALID and message in res[1]["message"]
    assert res[2]["status"] == slsf.OK


def test_server_cancel(slsf, ctx, orc):
    used0, _ = ctx.memory()
    srv = slsf.Server(ctx, epoch_sweeps=10)
    submit(srv, orc, (1, (8, 8, 8), 1.0, 1, 100000, 0, 1))
    srv.step()
    srv.cancel(1)
    submit(srv, orc, (2, (8, 8, 8), 1.0, 2, 100, 0, 1))
    srv.cancel(2)  # still queued
    with pytest.raises(slsf.SlsfError) as e:
        srv.cancel(99)
    assert e.value.code == slsf.ERR_INVALID and "unknown request tag" in str(e.value)
    srv.step()
    res = {r["tag"]: r for r in srv.poll()}
    st = srv.stats()
    srv.close()
    assert res[1]["status"] == slsf.ERR_STATE and res[1]["message"] == "cancelled" and res[1]["sweeps"] == 10
    assert res[2]["status"] == slsf.ERR_STATE and res[2]["sweeps"] == 0
    assert st["cancelled"] == 2
    assert ctx.memory()[0] == used0  # the cancelled task's memory is back


def test_server_worker_and_idle(slsf, ctx, orc):
    srv = slsf.Server(ctx, epoch_sweeps=10)
    submit(srv, orc, (1, (8, 8, 8), 1.0, 1, 40, 0, 2))
    with pytest.raises(slsf.SlsfError) as e:
        srv.wait_idle(0.05)  # nothing runs epochs yet
    assert e.value.code == slsf.ERR_TIMEOUT
    srv.start()
    with pytest.raises(slsf.SlsfError) as e:
        srv.step()
    assert e.value.code == slsf.ERR_STATE
    srv.wait_idle(60)
    srv.stop()
    [r] = srv.poll()
    assert r["status"] == slsf.OK and r["sweeps"] == 40
    assert srv.stats()["launches"] >= 4
    srv.close()


def test_server_admits_while_submissions_continue(slsf, ctx, orc):
    # Requests arrive while the worker thread admits and runs others; every
    # one completes, and each equals the same request run alone.
    import time

    srv = slsf.Server(ctx, epoch_sweeps=4)
    srv.start()
    reqs = [(k + 1, ((8, 8, 8), (16, 16, 16), (16, 8, 4))[k % 3], 1.0 + 0.01 * k, 100 + k, 12 + (k % 5), 2, 2)
            for k in range(150)]
    for r in reqs:
        submit(srv, orc, r)
        if r[0] % 10 == 0:
            srv.cancel(r[0])  # queued, being admitted or running: all are cancellable
        time.sleep(0.0005)
    srv.wait_idle(120)
    srv.stop()
    res = {r["tag"]: r for r in srv.poll(1000)}
    srv.close()
    assert sorted(res) == [r[0] for r in reqs]
    for r in reqs:
        got = res[r[0]]
        if r[0] % 10 == 0:
            assert got["status"] in (slsf.OK, slsf.ERR_STATE)
            continue
        assert got["status"] == slsf.OK, got["message"]
        assert got["sweeps"] == r[4]
    one = slsf.Server(ctx, epoch_sweeps=4)
    submit(one, orc, reqs[4])
    drain(one)
    [alone] = one.poll()
    one.close()
    assert alone["est"]["Energy"] == res[reqs[4][0]]["est"]["Energy"]


def test_served_stream_passes_two_sigma(slsf, ctx, orc):
    """Served results are statistically those of the reference algorithm.  A
    mixed stream of 24 requests (L = 8, 12, 16; T ~ U[1.0, 1.6]; J_z drawn per
    request) is served in one pass; each request runs again on the oracle's
    reference-order CPU path (FastRng streams, independent of the device's
    Philox streams) with the same couplings.  Per request and observable,
    z = (device - oracle) / sqrt(err_device^2 + err_oracle^2) over 20-sweep
    bins.  A request passes 2 sigma when its Energy and MagnetizationSquared
    both do; the latencies of passing requests are reported.  Over the whole
    stream, the pooled z of each of the two observables must be within 2."""
    rng = np.random.default_rng(20260710)
    therm, measured, binsize = 100, 800, 20
    srv = slsf.Server(ctx, epoch_sweeps=50)
    reqs = []
    for tag in range(1, 25):
        L, T, seed = int(rng.choice([8, 12, 16])), float(rng.uniform(1.0, 1.6)), 7000 + tag
        jxy, jz = couplings(orc, L, seed)
        reqs.append((tag, L, T, jxy, jz))
        srv.submit(tag, (L, L, L), T, seed, jxy, jz, therm + measured, thermalization=therm, binsize=binsize)
    drain(srv)
    res = {r["tag"]: r for r in srv.poll()}
    srv.close()
    assert sorted(res) == [r[0] for r in reqs]
    zs, passing = [], []
    diff = {"Energy": [], "MagnetizationSquared": []}
    var = {"Energy": [], "MagnetizationSquared": []}
    n_bins = measured // binsize
    for tag, L, T, jxy, jz in reqs:
        got = res[tag]
        assert got["status"] == slsf.OK, got["message"]
        assert got["est"]["measurements"] == measured and got["est"]["n_bins"] == n_bins
        m = orc.Model(L, L, L, jxy, jz, T, wolff_steps=1, seed=90000 + tag)
        m.init()
        series, _ = m.run_series(therm, measured)
        bins = series.reshape(n_bins, binsize, slsf.BIN_COLS).mean(axis=1)
        c_mean, c_err = bins.mean(axis=0), bins.std(axis=0, ddof=1) / np.sqrt(n_bins)
        z = {}
        for k, name in enumerate(slsf.BIN_NAMES):
            g_mean, g_err = got["est"][name]
            z[name] = (g_mean - c_mean[k]) / np.hypot(g_err, c_err[k])
            if name in diff:
                diff[name].append(g_mean - c_mean[k])
                var[name].append(g_err ** 2 + c_err[k] ** 2)
        zs.extend(z.values())
        if abs(z["Energy"]) < 2 and abs(z["MagnetizationSquared"]) < 2:
            passing.append(got["finish_s"] - got["submit_s"])
    zs = np.array(zs)
    print(f"served 2-sigma: {len(passing)} of {len(reqs)} pass; mean z^2 {np.mean(zs ** 2):.2f}; "
          f"max |z| {np.abs(zs).max():.2f}; latency of passing requests p50 {np.percentile(passing, 50):.3f} s, "
          f"p99 {np.percentile(passing, 99):.3f} s")
    # a bias shared by the requests shows in the pooled z: the differences summed
    # over the requests against their summed variances
    pooled = {k: float(np.sum(diff[k]) / np.sqrt(np.sum(var[k]))) for k in diff}
    print("served pooled z:", pooled)
    for k, pz in pooled.items():
        assert abs(pz) < 2.0, (k, pooled)
    # |z| < 2 holds for about 91% of requests when both observables are unbiased
    assert len(passing) >= 0.7 * len(reqs)
    assert np.mean(zs ** 2) < 2.0 and np.abs(zs).max() < 5.0


def test_server_keeps_bins_for_take_bins(slsf, ctx, orc):
    # keep_bins: each completed request's bin means stay until taken once; they
    # are the bins its estimates came from
    import ctypes

    srv = slsf.Server(ctx, epoch_sweeps=5, keep_bins=True)
    reqs = [(1, (8, 8, 8), 1.0, 11, 40, 5, 5), (2, (16, 16, 16), 1.3, 12, 55, 10, 9), (3, (6, 6, 4), 1.1, 14, 25, 5, 2)]
    for r in reqs:
        submit(srv, orc, r)
    drain(srv)
    res = {r["tag"]: r for r in srv.poll()}
    for tag, dims, T, _, _, _, n_bins in reqs:
        bins = srv.take_bins(tag)
        assert bins.shape == (n_bins, slsf.BIN_COLS)
        e = slsf.Estimates()
        b = np.ascontiguousarray(bins)
        slsf.host_check(slsf.load_host().slsf_estimates_from_bins(
            b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(b), float(np.prod(dims)), 1.0 / T,
            ctypes.byref(e)))
        for name in slsf.BIN_NAMES + slsf.DERIVED:
            assert e.as_dict()[name] == res[tag]["est"][name], (tag, name)
        with pytest.raises(slsf.SlsfError) as err:
            srv.take_bins(tag)  # released by the first take
        assert "no bins kept" in str(err.value)
    srv.close()
    plain = slsf.Server(ctx, epoch_sweeps=5)
    submit(plain, orc, reqs[0])
    drain(plain)
    plain.poll()
    with pytest.raises(slsf.SlsfError):
        plain.take_bins(1)
    plain.close()
