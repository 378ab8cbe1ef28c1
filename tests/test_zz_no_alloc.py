"""slsf_measure_noalloc: the fused measurement for callers that cannot allocate.

Hosts that own all device memory through their own pool, services under a
fixed device-memory budget, and loops that must not risk the device-wide
synchronisation of cudaMalloc/cudaFree pass their own device buffers and get
the observables back; the entry point's scratch is a static device array.
This file is collected last so that a failure here comes after every other
test has run; it passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_measure_matches_task_measure(slsf, orc):
    import torch

    slsf.build()
    lib = slsf.load()
    L = 24
    dims = (L, L, L)
    rng = np.random.default_rng(7)
    jxy = np.full(L, 1.2)
    jz = rng.uniform(0.5, 1.5, L)
    with slsf.Context(0) as ctx:
        task = slsf.Task(ctx, dims, jxy, jz, 1.1, seed=99)
        task.init_random()
        task.sweep(2)
        theta = task.theta
        ref = task.measure()
        dev = torch.device("cuda", 0)
        th_d = torch.from_numpy(theta).to(dev)
        jxy_d = torch.from_numpy(jxy.astype(np.float32)).to(dev)
        jz_d = torch.from_numpy(jz.astype(np.float32)).to(dev)
        torch.cuda.synchronize(dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        exact = orc.measure_f32(dims, theta, jxy.astype(np.float32), jz.astype(np.float32))
        free_before = None
        for call in range(2):  # two calls in a row share the static scratch
            if call == 1:
                torch.cuda.synchronize(dev)
                free_before = torch.cuda.mem_get_info(dev)[0]
            out = slsf.Observables()
            rc = lib.slsf_measure_noalloc(C.c_void_p(th_d.data_ptr()), C.c_void_p(jxy_d.data_ptr()),
                                          C.c_void_p(jz_d.data_ptr()), L, L, L, C.c_void_p(stream), C.byref(out))
            assert rc == slsf.OK, slsf.last_error()
            got = out.as_dict()
            v = L ** 3
            assert abs(got["energy"] - ref["energy"]) < 2e-5
            assert abs(got["magnetization_squared"] - ref["magnetization_squared"]) < 1e-5
            for k in ("cos_x", "cos_y", "cos_z", "sin_x", "sin_y", "sin_z"):
                assert abs(got[k] - ref[k]) < 2e-5 * v + 1e-5, (k, got[k], ref[k])
            # and against the oracle's FP64 evaluation of the same FP32 state
            assert abs(got["energy"] - exact["energy"]) < 2e-5
            assert abs(got["magnetization_squared"] - exact["magnetization_squared"]) < 1e-5
            for k in ("cos_x", "cos_y", "cos_z", "sin_x", "sin_y", "sin_z"):
                assert abs(got[k] - exact[k]) < 2e-5 * v + 1e-5, (k, got[k], exact[k])
        # the second call took no device memory
        torch.cuda.synchronize(dev)
        assert torch.cuda.mem_get_info(dev)[0] == free_before
        task.close()


def test_noalloc_rejects_bad_sizes(slsf):
    lib = slsf.load()
    out = slsf.Observables()
    one = C.c_void_p(1)
    assert lib.slsf_measure_noalloc(one, one, one, 0, 4, 4, None, C.byref(out)) == slsf.ERR_INVALID
    assert slsf.last_error() == "L_x must be positive"
    big = 2048  # 2048^3 > 2^31 - 1 sites
    assert lib.slsf_measure_noalloc(one, one, one, big, big, big, None, C.byref(out)) == slsf.ERR_INVALID
    assert "no-allocation measurement limit" in slsf.last_error()
