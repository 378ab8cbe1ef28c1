"""Host layer (libslsf_host.so, include/slsf_host.h) on the CPU: binning,
derived estimates, the task seed formula and the layer-coupling draw, each
checked against the oracle's restatement of the reference.  Nothing here
launches a kernel."""
import ctypes

import numpy as np
import pytest


def test_host_library_exports_every_declared_symbol(slsf):
    slsf.build()
    declared = slsf.host_declared_symbols()
    assert len(declared) >= 16
    lib = ctypes.CDLL(slsf.HOST_LIB_PATH)
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(slsf.HOST_SIGNATURES) == declared


def test_binned_estimate_known_answer(slsf):
    # binned_estimate_reports_mean_and_standard_error (src/tests.rs:436-446)
    r = slsf.binned_estimate([1.0, 3.0, 5.0, 7.0], 2)
    assert r["mean"] == pytest.approx(4.0, abs=1e-12)
    assert r["stderr"] == pytest.approx(2.0, abs=1e-12)
    assert r["n_bins"] == 2


def test_binned_estimate_rejects_oversized_bins(slsf):
    with pytest.raises(slsf.SlsfError) as e:
        slsf.binned_estimate([1.0, 2.0], 3)
    assert e.value.code == slsf.ERR_INVALID
    assert "binsize is larger than the sample series" in str(e.value)


@pytest.mark.parametrize("n,binsize", [(100, 7), (64, 8), (5, 5), (1000, 33)])
def test_binned_estimate_matches_oracle(slsf, orc, n, binsize):
    x = np.random.default_rng(n * 31 + binsize).normal(size=n)
    mine = slsf.binned_estimate(x, binsize)
    ref = orc.binned_estimate(x, binsize)
    assert mine["mean"] == pytest.approx(ref["mean"], rel=1e-13, abs=1e-15)
    assert mine["stderr"] == pytest.approx(ref["stderr"], rel=1e-12, abs=1e-15)
    assert mine["n_bins"] == ref["bins"].size


@pytest.mark.parametrize("nb", [1, 2, 9])
def test_estimates_from_bins_match_oracle(slsf, orc, nb):
    rng = np.random.default_rng(nb)
    bm = np.abs(rng.normal(size=(nb, slsf.BIN_COLS))) + 0.1
    vol, beta = 512.0, 1.0 / 1.3
    e = slsf.Estimates()
    slsf.host_check(slsf.load_host().slsf_estimates_from_bins(
        bm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nb, vol, beta, ctypes.byref(e)))
    d = e.as_dict()
    ref = orc.evaluate_derived(bm, vol, beta)
    for name in slsf.DERIVED:
        assert d[name][0] == pytest.approx(ref[name][0], rel=1e-13, abs=1e-14), name
        assert d[name][1] == pytest.approx(ref[name][1], rel=1e-10, abs=1e-14), name
    assert np.allclose([d[n][0] for n in slsf.BIN_NAMES], bm.mean(axis=0), rtol=1e-14)


@pytest.mark.parametrize("args", [
    (0, 32, 0, 1.0, 0.0, 0.0), (20260410, 8, 3, 1.225, 0.0, 0.5), (7, 16, 12, 0.005, 0.0005, 0.0015),
    (2 ** 63, 64, 999, 2.345, 0.25, 0.75)])
def test_task_seed_matches_formula(slsf, args):
    # make_theta_tasks (src/model.rs:741-747), halves rounding away from zero
    assert slsf.load_host().slsf_task_seed(*args) == slsf.task_seed(*args)


@pytest.mark.parametrize("seed", [0, 1, 12345, 2 ** 64 - 1])
def test_task_couplings_follow_two_point_draw(slsf, orc, seed):
    # ThetaModel::new draws J_xy then J_z from one FastRng(disorder_seed)
    d = slsf.theta_task((4, 4, 12), 1.0, 10, 0, 1, seed=1, disorder_seed=seed, j_xy=1.0, delta_j_xy=0.25,
                        j_z_mean=0.5, delta_j_z=0.5)
    jx, jz = slsf.task_couplings(d)
    rng = orc.FastRng(seed)
    ref_x = orc.two_point_disorder(12, 1.0, 0.25, rng, "J_xy")
    ref_z = orc.two_point_disorder(12, 0.5, 0.5, rng, "J_z")
    assert np.array_equal(jx, ref_x) and np.array_equal(jz, ref_z)


def test_task_couplings_explicit_arrays_and_errors(slsf):
    d = slsf.theta_task((4, 4, 3), 1.0, 10, 0, 1, seed=1, j_xy_array=[1.0, 2.0, 3.0], j_z_array=[0.1, 0.2, 0.3])
    jx, jz = slsf.task_couplings(d)
    assert list(jx) == [1.0, 2.0, 3.0] and list(jz) == [0.1, 0.2, 0.3]
    bad = slsf.theta_task((4, 4, 3), 1.0, 10, 0, 1, seed=1, j_z_mean=0.1, delta_j_z=0.5)
    with pytest.raises(slsf.SlsfError) as e:
        slsf.task_couplings(bad)
    assert "two-point layer disorder requires J_z_mean - δJ_z >= 0" in str(e.value)
    neg = slsf.theta_task((4, 4, 3), 1.0, 10, 0, 1, seed=1, j_xy_array=[1.0, -1.0, 1.0])
    with pytest.raises(slsf.SlsfError) as e:
        slsf.task_couplings(neg)
    assert "nonnegative layer couplings" in str(e.value)


def test_server_rejects_null_context(slsf):
    h = ctypes.c_void_p()
    cfg = slsf.ServerConfig(epoch_sweeps=10)
    with pytest.raises(slsf.SlsfError) as e:
        slsf.host_check(slsf.load_host().slsf_server_create(None, ctypes.byref(cfg), ctypes.byref(h)))
    assert e.value.code == slsf.ERR_INVALID
