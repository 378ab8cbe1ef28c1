"""Checkpoints (marked gpu): a task's device state saved, loaded into a new
task and continued gives bit for bit what the uninterrupted task gives
(angles, bins, correlation bins, counters); mismatched states are refused;
a server checkpointed mid-run and restored in a new server finishes every
request with the results of an uninterrupted run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(slsf):
    slsf.build()
    c = slsf.Context()
    yield c
    c.close()


def make(slsf, ctx, orc, dims, seed, T=1.2, corr=(3, 2), **kw):
    jxy, jz = np.full(dims[2], 1.0), orc.uniform_disorder(dims[2], 0.5, 1.5, seed)
    t = slsf.Task(ctx, dims, jxy, jz, T, seed=seed, thermalization=2, binsize=3, n_bins=4, **kw)
    if corr:
        t.corr_setup(*corr, 2, 3)
    return t


@pytest.mark.parametrize("dims", [(8, 8, 8), (6, 6, 4), (32, 32, 32), (48, 48, 48)])
def test_state_resume_is_bitwise(slsf, ctx, orc, dims):
    a = make(slsf, ctx, orc, dims, 7)
    a.init_random()
    for _ in range(3):
        ctx.batch_run([a], 2)
        ctx.batch_correlations([a])
    blob = a.save_state(user=(11, 22, 33, 2 ** 64 - 1))
    b = make(slsf, ctx, orc, dims, 7)
    b.init_random()
    ctx.batch_run([b], 1)  # whatever b held before is replaced
    assert b.load_state(blob) == (11, 22, 33, 2 ** 64 - 1)
    assert b.counters == a.counters == (6, 6)
    assert b.corr_bins()[1] == 3
    for t in (a, b):
        for _ in range(4):
            ctx.batch_run([t], 2)
            ctx.batch_correlations([t])
    assert np.array_equal(a.theta.view(np.uint32), b.theta.view(np.uint32))
    assert a.counters == b.counters
    ba, ma = a.bins()
    bb, mb = b.bins()
    assert ma == mb == 12 and np.array_equal(ba, bb)
    ca, na = a.corr_bins()
    cb, nb = b.corr_bins()
    assert na == nb == 7 and np.array_equal(ca, cb)
    assert a.save_state() == b.save_state()
    a.close()
    b.close()


def test_state_mismatch_is_refused(slsf, ctx, orc):
    a = make(slsf, ctx, orc, (8, 8, 8), 3)
    a.init_random()
    blob = a.save_state()

    def refused(t, data, fragment):
        with pytest.raises(slsf.SlsfError) as e:
            t.load_state(data)
        assert e.value.code == slsf.ERR_INVALID and fragment in str(e.value), str(e.value)
        t.close()

    refused(make(slsf, ctx, orc, (8, 8, 8), 4), blob, "seed")
    refused(make(slsf, ctx, orc, (8, 8, 10), 3), blob, "size")
    refused(make(slsf, ctx, orc, (8, 8, 8), 3, T=1.3), blob, "temperature")
    refused(make(slsf, ctx, orc, (8, 8, 8), 3, corr=(2, 2)), blob, "")
    t = make(slsf, ctx, orc, (8, 8, 8), 3)
    refused(t, b"XXXXXXXX" + blob[8:], "bad magic")
    refused(make(slsf, ctx, orc, (8, 8, 8), 3), blob[:100], "")
    jxy, jz = np.full(8, 1.5), orc.uniform_disorder(8, 0.5, 1.5, 3)
    other = slsf.Task(ctx, (8, 8, 8), jxy, jz, 1.2, seed=3, thermalization=2, binsize=3, n_bins=4)
    other.corr_setup(3, 2, 2, 3)
    refused(other, blob, "layer couplings")
    a.close()


def requests(orc):
    # (tag, dims, T, seed, sweeps, thermalization, binsize)
    return [(1, (8, 8, 8), 1.0, 11, 40, 5, 5), (2, (16, 16, 16), 1.3, 12, 55, 10, 9),
            (3, (32, 32, 32), 1.5, 13, 33, 4, 4), (4, (6, 6, 4), 1.1, 14, 25, 5, 2),
            (5, (16, 8, 12), 0.9, 15, 41, 1, 8), (6, (24, 24, 24), 1.25, 17, 30, 3, 10)]


def submit(srv, orc, req):
    tag, dims, T, seed, sweeps, therm, binsize = req
    srv.submit(tag, dims, T, seed, np.ones(dims[2]), orc.uniform_disorder(dims[2], 0.5, 1.5, seed), sweeps,
               thermalization=therm, binsize=binsize)


def drain(srv):
    for _ in range(10000):
        a, p = srv.step()
        if a == 0 and p == 0:
            return
    raise AssertionError("server did not drain")


def test_server_checkpoint_restore(slsf, ctx, orc, tmp_path):
    whole = slsf.Server(ctx, epoch_sweeps=5)
    for r in requests(orc):
        submit(whole, orc, r)
    drain(whole)
    ref = {r["tag"]: r for r in whole.poll()}
    whole.close()

    first = slsf.Server(ctx, epoch_sweeps=5, max_active=3)  # some stay queued
    for r in requests(orc):
        submit(first, orc, r)
    for _ in range(4):
        first.step()
    done = {r["tag"]: r for r in first.poll()}
    n = first.checkpoint(tmp_path / "ckpt")
    assert n == len(requests(orc)) - len(done) and n > 0
    first.close()  # the interrupted run ends here

    second = slsf.Server(ctx, epoch_sweeps=5)
    assert second.restore(tmp_path / "ckpt") == n
    drain(second)
    rest = {r["tag"]: r for r in second.poll()}
    second.close()
    assert sorted({**done, **rest}) == sorted(ref)
    for tag, got in {**done, **rest}.items():
        want = ref[tag]
        assert got["status"] == slsf.OK, got["message"]
        assert got["sweeps"] == want["sweeps"]
        assert (got["accepted"], got["cluster_sites"]) == (want["accepted"], want["cluster_sites"])
        for name in slsf.BIN_NAMES + slsf.DERIVED:
            assert got["est"][name] == want["est"][name], (tag, name)
        assert got["est"]["measurements"] == want["est"]["measurements"]


def test_server_checkpoint_needs_stopped_worker(slsf, ctx, orc, tmp_path):
    srv = slsf.Server(ctx, epoch_sweeps=5)
    srv.start()
    with pytest.raises(slsf.SlsfError) as e:
        srv.checkpoint(tmp_path)
    assert e.value.code == slsf.ERR_STATE
    srv.stop()
    assert srv.checkpoint(tmp_path / "empty") == 0
    (tmp_path / "bad").mkdir()
    (tmp_path / "bad" / "request_9.ckpt").write_bytes(b"not a checkpoint")
    with pytest.raises(slsf.SlsfError) as e:
        srv.restore(tmp_path / "bad")
    assert "not a request checkpoint" in str(e.value)
    srv.close()
