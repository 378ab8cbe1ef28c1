"""Failure detection without a GPU fault (marked gpu): every device loop is
bounded; with the bound lowered to 1 (slsf_ctx_set_loop_limit) the Wolff
labelling of the single-task and batched kernels gives up, the kernel records
it and returns, the call reports SLSF_ERR_TIMEOUT, and the context stays
usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def task(slsf, ctx, dims, T=0.5, seed=3):
    t = slsf.Task(ctx, dims, np.full(dims[2], 1.2), np.full(dims[2], 1.0), T, wolff_steps=1, seed=seed)
    t.init_random()
    return t


@pytest.mark.parametrize("dims,path", [((64, 64, 64), "single"), ((256, 128, 128), "single"), ((32, 32, 32), "batched"),
                                       ((48, 48, 48), "batched"), ((128, 8, 8), "batched")])
def test_bounded_loop_reports_timeout_and_context_recovers(slsf, dims, path):
    ctx = slsf.Context()
    try:
        ctx.set_loop_limit(1)
        t = task(slsf, ctx, dims)
        with pytest.raises(slsf.SlsfError) as e:
            if path == "single":
                t.sweep(3)
            else:
                ctx.batch_run([t], 3)
        assert e.value.code == slsf.ERR_TIMEOUT
        assert "bounded device loop" in str(e.value)
        t.close()
        # defaults back: the same context runs a task bit-identically to a fresh context
        ctx.set_loop_limit(0)
        a = task(slsf, ctx, dims, T=1.1, seed=9)
        ctx.batch_run([a], 2)
        with slsf.Context() as other:
            b = task(slsf, other, dims, T=1.1, seed=9)
            other.batch_run([b], 2)
            assert np.array_equal(a.theta.view(np.uint32), b.theta.view(np.uint32))
            b.close()
    finally:
        ctx.close()
