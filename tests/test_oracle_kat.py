"""The oracle against every known-answer test the reference holds for this path.

Each test names the reference test it ports (src/tests.rs) and asserts the
same values, tolerances and error strings.  The published vectors of the two
random generators (Vigna's SplitMix64 vector, the Random123 Philox4x32-10
known-answer vectors) are fixtures under tests/golden/, checked in
test_golden.py.
"""
import math

import numpy as np
import pytest

TWO_PI = 2.0 * math.pi


def test_fastrng_set_position_matches_stream(orc):
    # FastRng::set_position (src/types.rs:31-36) must land on the same stream position.
    a = orc.FastRng(99)
    words = [a.next_u64() for _ in range(10)]
    b = orc.FastRng(99)
    b.set_position(6)
    assert b.next_u64() == words[6]
    assert a.draws == 10


def test_keyed_init_angles(orc):
    # The INIT stream of the shared Philox generator (slsf-rs_b200/csrc/xy_rng.h;
    # its published vectors are checked in test_golden.py).
    th = orc.keyed_init_angles(1024, 12345)
    assert th.dtype == np.float32
    assert np.all((th >= 0) & (th < np.float32(TWO_PI)))
    assert np.array_equal(th, orc.keyed_init_angles(1024, 12345))
    assert not np.array_equal(th, orc.keyed_init_angles(1024, 12346))


def test_fast_math_matches_std(orc):
    # fast_math_x8_matches_scalar_regression (src/tests.rs:11-23): the oracle's
    # sin/cos/exp are libm, the reference's sleef is pinned to them within 1e-14.
    for v in [-2.0, -1.25, -0.5, -0.125, 0.0, 0.125, 0.5, 1.75]:
        th = np.array([v, 0.0])
        m2 = orc.magnetization_squared(th)
        exp_m2 = ((math.cos(v) + 1) ** 2 + math.sin(v) ** 2) / 4
        assert abs(m2 - exp_m2) < 1e-14


def test_metropolis_accept_probability_form(orc):
    # metropolis_batch_acceptance_probabilities_match_scalar (src/tests.rs:25-43):
    # the accept probability is exp(-beta dE) for dE > 0 and 1 otherwise.
    # The keyed half-sweep exports the probability it compared against.
    dims = (4, 4, 4)
    rng = orc.FastRng(3)
    th = orc.init_angles(64, rng).astype(np.float32)
    j = np.ones(4, np.float32)
    beta = np.float32(0.75)
    res = orc.keyed_metro_half(dims, th, j, j, beta, np.float32(math.pi), 7, 0, 0, 0.0)
    p = res["prob"][res["decision"] >= 0]
    assert np.all((p > 0) & (p <= 1.0))


def test_theta_lattice_initialization_and_disorder(orc):
    # theta_lattice_initialization_and_disorder (src/tests.rs:45-91).
    for dims, msg in [((0, 2, 2), "L_x must be positive"), ((2, 0, 2), "L_y must be positive"),
                      ((2, 2, 0), "L_z must be positive")]:
        with pytest.raises(orc.OracleError, match=msg):
            orc.Model(*dims, np.ones(dims[2]), np.ones(dims[2]), 2.0)
    rng = orc.FastRng(12345)
    jz = orc.two_point_disorder(5, 0.7, 0.0, rng)
    assert np.all(jz == 0.7)
    big = orc.two_point_disorder(200_000, 1.0, 0.5, rng)
    assert np.all((big == 0.5) | (big == 1.5))
    assert abs(big.mean() - 1.0) < 5e-3
    assert abs(big.std(ddof=1) - 0.5) < 5e-3
    with pytest.raises(orc.OracleError) as e:
        orc.two_point_disorder(5, 1.0, -0.1, rng)
    assert str(e.value) == "δJ_z must be nonnegative"
    with pytest.raises(orc.OracleError) as e:
        orc.two_point_disorder(5, 0.05, 0.1, rng)
    assert str(e.value) == "two-point layer disorder requires J_z_mean - δJ_z >= 0"
    cold = orc.init_angles(60, rng, cold=True)
    assert np.all(cold == 0.0)
    hot = orc.init_angles(60, rng)
    assert np.all((hot >= 0.0) & (hot < TWO_PI))


def test_theta_energy_magnetization_and_correlations(orc):
    # theta_energy_magnetization_and_correlations (src/tests.rs:93-153).
    dims = (2, 2, 2)
    jxy, jz = np.full(2, 1.5), np.full(2, 0.5)
    th = np.zeros(8)
    expected = -(2 * 1.5 + 0.5)
    assert abs(orc.measure_energy(dims, th, jxy, jz) - expected) < 1e-12
    assert abs(math.sqrt(orc.magnetization_squared(th)) - 1.0) < 1e-12
    obs = orc.measure_observables(dims, th, jxy, jz)
    h = orc.helicity_sums(dims, th, jxy, jz)
    assert abs(obs["energy"] - orc.measure_energy(dims, th, jxy, jz)) < 1e-12
    assert abs(obs["magnetization_squared"] - 1.0) < 1e-12
    for k, name in enumerate(["cos_x", "cos_y", "cos_z", "sin_x", "sin_y", "sin_z"]):
        assert abs(obs[name] - h[k]) < 1e-12
    corr = orc.measure_correlations(dims, th, rmax=1)
    assert corr["r_xy"] == [1]
    for key in ("corr_x", "corr_y", "corr_xy", "corr_z"):
        assert abs(corr[key][0] - 1.0) < 1e-12
    assert corr["corr_xy_by_z"].shape == (2, 1)
    assert np.all(np.abs(corr["corr_xy_by_z"] - 1.0) < 1e-12)
    th3 = th.reshape(2, 2, 2).copy()  # [z][y][x]
    for y in range(2):
        for x in range(2):
            th3[1, y, x] = -1.0 if (x + y) % 2 == 0 else 1.0
    th = th3.ravel()
    lc = orc.measure_correlations(dims, th, rmax=1)
    assert abs(lc["corr_xy_by_z"][0, 0] - 1.0) < 1e-12
    assert lc["corr_xy_by_z"][1, 0] < 0.0
    assert abs(lc["corr_xy"][0] - (lc["corr_xy_by_z"][0, 0] + lc["corr_xy_by_z"][1, 0]) / 2) < 1e-12
    th[0] = math.pi
    m = math.sqrt(orc.magnetization_squared(th))
    assert 0.0 <= m <= 1.0


def test_theta_metropolis_updates_validate_and_keep_angles_wrapped(orc):
    # theta_metropolis_updates_validate_and_keep_angles_wrapped (src/tests.rs:155-193).
    rng = orc.FastRng(12)
    jz = orc.two_point_disorder(3, 0.8, 0.0, rng)
    m = orc.Model(3, 3, 3, np.full(3, 1.0), jz, 2.0, proposal_width=0.5, seed=12)
    m.init()
    old = m.theta
    assert m.local_metropolis_step(0.0) is True
    assert np.array_equal(m.theta, old)
    with pytest.raises(orc.OracleError, match="^red-black Metropolis sweep requires even lattice dimensions$"):
        m.metropolis_sweep()
    assert np.all((m.theta >= 0) & (m.theta < TWO_PI))
    with pytest.raises(orc.OracleError, match="^proposal_width must be nonnegative and finite$"):
        m.local_metropolis_step(-0.1)
    bad = orc.Model(4, 4, 4, np.ones(4), np.full(4, 0.8), 2.0, proposal_width=math.inf, seed=1)
    with pytest.raises(orc.OracleError, match="^proposal_width must be nonnegative and finite$"):
        bad.metropolis_sweep()
    even = orc.Model(4, 4, 4, np.ones(4), np.full(4, 0.8), 2.0, proposal_width=0.5, seed=13)
    even.init()
    acc = even.metropolis_sweep()
    assert 0.0 <= acc <= 1.0
    assert np.all((even.theta >= 0) & (even.theta < TWO_PI))
    assert 0.0 <= even.metropolis_sweep(batch8=False) <= 1.0


def test_theta_temperature_validation_and_helicity(orc):
    # theta_temperature_validation_and_helicity (src/tests.rs:195-239).
    dims = (3, 3, 3)
    th = np.zeros(27)
    rho = orc.helicity_modulus(dims, th, np.full(3, 1.2), np.full(3, 0.6), 0.5)
    assert abs(rho[0] - 1.2) < 1e-12 and abs(rho[1] - 1.2) < 1e-12 and abs(rho[2] - 0.6) < 1e-12
    for bad_t in [0.0, -1.0, math.inf, math.nan]:
        m = orc.Model(4, 4, 4, np.full(4, 1.2), np.full(4, 0.6), bad_t, seed=1)
        for call in (lambda: m.local_metropolis_step(math.pi), m.metropolis_sweep, m.wolff_step,
                     lambda: orc.helicity_modulus(dims, th, np.full(3, 1.2), np.full(3, 0.6), bad_t)):
            with pytest.raises(orc.OracleError) as e:
                call()
            assert str(e.value) == "temperature T must be positive and finite"


def test_theta_simulation_driver(orc):
    # theta_simulation_driver (src/tests.rs:241-370).
    rng = orc.FastRng(14)
    res = orc.run_theta_simulation((4, 4, 4), 1.0, 1.0, 0.0, 0.5, rng, thermal_sweeps=5, measure_sweeps=10,
                                   measure_interval=2, proposal_width=0.4, correlation_rmax=1, init_cold=True)
    for k in ("energy", "rho_sx", "rho_sy", "rho_sz", "chi"):
        assert math.isfinite(res[k])
    assert 0.0 <= res["magnetization_squared"] <= 1.0
    assert len(res["corr_x"]) == 1 and len(res["corr_z"]) == 1
    assert res["num_correlation_measurements"] == res["num_measurements"]
    assert math.isfinite(res["corr_z"][0])
    assert 0.0 <= res["acceptance"] <= 1.0
    r2 = orc.run_theta_simulation((2, 2, 2), 1.0, 1.0, 0.0, 0.5, rng, thermal_sweeps=0, measure_sweeps=1,
                                  measure_interval=1, init_cold=True)
    assert math.isfinite(r2["energy"])
    cases = [
        (dict(measure_interval=0), "measure_interval must be positive"),
        (dict(thermal_sweeps=0, measure_sweeps=1, measure_interval=2),
         "measure_sweeps must include at least one measurement; require measure_sweeps >= measure_interval"),
        (dict(correlation_interval=0), "correlation_interval must be positive"),
        (dict(thermal_sweeps=0, measure_sweeps=1, measure_interval=1, proposal_width=math.nan),
         "proposal_width must be nonnegative and finite"),
    ]
    for opts, msg in cases:
        with pytest.raises(orc.OracleError) as e:
            orc.run_theta_simulation((2, 2, 2), 1.0, 1.0, 0.0, 0.5, rng, **opts)
        assert str(e.value) == msg
    thr = orc.run_theta_simulation((2, 2, 2), 1.0, 1.0, 0.0, 0.5, rng, thermal_sweeps=0, measure_sweeps=5,
                                   measure_interval=1, proposal_width=0.0, wolff_steps=0, correlation_rmax=1,
                                   correlation_interval=2, init_cold=True)
    assert thr["num_measurements"] == 5
    assert thr["num_correlation_measurements"] == 3
    assert abs(thr["corr_x"][0] - 1.0) < 1e-12
    with pytest.raises(orc.OracleError) as e:
        orc.run_theta_simulation((2, 2, 2), 1.0, -0.1, 0.0, 1.0, rng, thermal_sweeps=0, measure_sweeps=1,
                                 measure_interval=1)
    assert str(e.value) == "two-point layer disorder requires J_z_mean - δJ_z >= 0"


def test_theta_wolff_cluster_update(orc):
    # theta_wolff_cluster_update (src/tests.rs:372-432).
    assert abs(orc.lib().or_wolff_add_probability(1.0, 1.0, 1.0, 1.0) - (1.0 - math.exp(-2.0))) < 1e-12
    for ri, rj in [(1.0, -1.0), (-1.0, 1.0), (0.0, 1.0)]:
        assert abs(orc.lib().or_wolff_add_probability(1.0, 1.0, ri, rj)) < 1e-12
    refl = orc.lib().or_wolff_reflect_angle(0.37, 1.20)
    assert abs(orc.lib().or_wolff_reflect_angle(refl, 1.20) - 0.37) < 1e-12
    assert 0.0 <= refl < TWO_PI
    m = orc.Model(4, 4, 4, np.ones(4), np.ones(4), 1.0, seed=15)
    m.init()
    for _ in range(2):
        size = m.wolff_step()
        assert 1 <= size <= 64
    # Scratch is cleared after each step: a third step still returns a valid
    # size and the state stays finite.
    assert 1 <= m.wolff_step() <= 64
    assert np.all(np.isfinite(m.theta))


def test_binning_kat(orc):
    # theta_carlo_entrypoint_job_config_and_binning, binning part (src/tests.rs:436-446).
    est = orc.binned_estimate([1.0, 3.0, 5.0, 7.0], 2)
    assert abs(est["mean"] - 4.0) < 1e-12
    assert abs(est["stderr"] - 2.0) < 1e-12
    assert list(est["bins"]) == [2.0, 6.0]
    with pytest.raises(orc.OracleError) as e:
        orc.binned_estimate([1.0], 2)
    assert str(e.value) == "binsize is larger than the sample series"


@pytest.mark.parametrize("L", [2, 4, 8, 32])
def test_cold_state_kat_any_size(orc, L):
    # Cold state: E/V = -(2 J_xy + J_z), m^2 = 1, rho_mu = J_mu, all C = 1 for uniform J at any L.
    jxy, jz = np.full(L, 1.2), np.full(L, 0.6)
    th = np.zeros(L ** 3)
    o = orc.measure_observables((L, L, L), th, jxy, jz)
    assert abs(o["energy"] + (2 * 1.2 + 0.6)) < 1e-12
    assert abs(o["magnetization_squared"] - 1.0) < 1e-12
    rho = orc.helicity_modulus((L, L, L), th, jxy, jz, 1.0)
    assert np.allclose(rho, [1.2, 1.2, 0.6], atol=1e-12)


def test_rand_range_and_bool_sampling(orc):
    # rand's range and bool sampling from FastRng, used by the Wolff seed
    # (src/updates.rs:566-568) and the two-point disorder (initialization.rs:27).
    r = orc.FastRng(5)
    vals = [r.range(10) for _ in range(20000)]
    assert min(vals) == 0 and max(vals) == 9
    counts = np.bincount(vals, minlength=10)
    assert np.all(np.abs(counts - 2000) < 250)
    r = orc.FastRng(6)
    bools = [r.bool() for _ in range(20000)]
    assert abs(sum(bools) - 10000) < 400


def test_keyed_metropolis_width_zero_keeps_state(orc):
    # Width 0 proposes theta itself: dE = 0, always accepted, state unchanged
    # (src/tests.rs:163-165 in counter-based form).
    dims = (4, 4, 4)
    th = orc.keyed_init_angles(64, 3)
    j = np.ones(4, np.float32)
    for color in (0, 1):
        res = orc.keyed_metro_half(dims, th, j, j, np.float32(1.0), np.float32(0.0), 3, 0, color, 0.0)
        assert np.array_equal(res["theta"], th)
        assert np.all(res["decision"][res["decision"] >= 0] == 1)


def test_keyed_wolff_component_is_order_free(orc):
    # The cluster is the seed's connected component over active bonds, so it
    # equals the DFS of src/updates.rs:577-597 fed the same per-bond randoms.
    dims = (6, 4, 8)
    th = orc.keyed_init_angles(6 * 4 * 8, 11)
    jxy = np.full(8, 1.2, np.float32)
    jz = np.linspace(0.5, 1.5, 8).astype(np.float32)
    res = orc.keyed_wolff(dims, th, jxy, jz, np.float32(1 / 1.1), 11, 4, 0, 0.0)
    phi, site = orc.keyed_wolff_pick(dims, 11, 4, 0)
    seed_idx = site[0] + 6 * (site[1] + 4 * site[2])
    assert res["cluster"][seed_idx] == 1
    cl, size = orc.cluster_from_bonds(dims, res["bonds"] & 7, seed_idx)
    assert size == res["size"] and np.array_equal(cl, res["cluster"])
    # Reflection is an involution up to FP32 rounding.
    back = orc.keyed_wolff(dims, res["theta"], jxy, jz, np.float32(1 / 1.1), 11, 4, 0, 0.0)
    diff = np.abs(back["theta"] - th)
    diff = np.minimum(diff, 2 * np.pi - diff)
    assert np.all(diff[res["cluster"] == 1] < 4e-6)
