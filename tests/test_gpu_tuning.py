"""Kernel choices per lattice shape (marked gpu): every feasible choice (the
one-CTA kernel at each CTA size, the cluster kernel at each cluster size,
the grid-wide kernels) gives the same trajectory bit for bit and the same
bins to FP64 summation order; the autotuner keeps a feasible choice; the table
survives a save / load round trip."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(slsf):
    slsf.build()
    c = slsf.Context()
    yield c
    c.close()


CHOICES = [("resident", 1, 128), ("resident", 1, 256), ("resident", 1, 512), ("resident", 1, 1024),
           ("cluster", 1, 512), ("cluster", 2, 1024), ("cluster", 4, 512), ("cluster", 8, 1024),
           ("cluster", 16, 1024), ("grid", 1, 256)]


def run(slsf, ctx, dims, choice, sweeps=4):
    jz = np.linspace(0.5, 1.5, dims[2])
    t = slsf.Task(ctx, dims, np.full(dims[2], 1.2), jz, 1.2, wolff_steps=1, seed=5, thermalization=1, binsize=1,
                  n_bins=sweeps)
    t.init_random()
    ctx.tune_set(dims, *choice)
    ctx.batch_run([t], 2)
    ctx.batch_run([t], sweeps - 2)
    theta, bins = t.theta, t.bins()[0]
    t.close()
    return theta, bins


@pytest.mark.parametrize("dims", [(8, 8, 8), (16, 16, 16), (32, 32, 32), (48, 48, 48), (64, 64, 64), (24, 16, 32),
                                  (8, 80, 8), (8, 8, 64), (40, 34, 8)])
def test_every_choice_gives_the_same_trajectory(slsf, ctx, dims):
    ref = None
    tried = 0
    for choice in CHOICES:
        try:
            theta, bins = run(slsf, ctx, dims, choice)
        except slsf.SlsfError as e:
            assert "does not hold this lattice" in str(e)
            continue
        tried += 1
        if ref is None:
            ref = (theta, bins)
            continue
        assert np.array_equal(theta.view(np.uint32), ref[0].view(np.uint32)), choice
        assert np.allclose(bins, ref[1], rtol=1e-10, atol=1e-10 * np.prod(dims)), choice
    assert tried >= 3


def test_autotune_and_table_round_trip(slsf, ctx, tmp_path):
    best = ctx.autotune((16, 16, 16))
    assert best["site_updates_per_s"] > 0
    assert ctx.tune_get((16, 16, 16)) == {k: best[k] for k in ("kind", "cluster", "threads")}
    ctx.tune_set((32, 32, 32), "cluster", 2, 512)
    path = tmp_path / "tune.txt"
    ctx.tune_save(path)
    with slsf.Context() as other:
        assert other.tune_get((32, 32, 32))["kind"] == "resident"  # the default
        other.tune_load(path)
        assert other.tune_get((32, 32, 32)) == {"kind": "cluster", "cluster": 2, "threads": 512}
        assert other.tune_get((16, 16, 16)) == ctx.tune_get((16, 16, 16))
    with pytest.raises(slsf.SlsfError):
        ctx.tune_set((64, 64, 64), "resident", 1, 1024)  # 64-bit rows do not fit the one-CTA kernel
