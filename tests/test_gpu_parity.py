"""GPU parity against the oracle through the C ABI (marked gpu).

Bars:
  - initial angles, proposals, reflections: bit-exact FP32 (shared Philox
    streams and explicitly rounded FP32 operations);
  - Metropolis decisions: identical on every site whose accept probability
    is farther than EPS_METRO from its accept random (the FP32 fast-sincos
    error bound); those "tie" sites are counted and reported;
  - Wolff bonds: identical outside the EPS_WOLFF tie band; the cluster is
    bit-exact against the oracle's DFS labelling of the device's bonds;
  - reductions: FP64 sums of FP32 per-site terms, tolerances per observable.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# |dE| <= 2 |c - c'| |dh| + ... with |d trig| <= 2e-6 and |h| <= 9 gives
# |d dE| <= 1.6e-4; |d p| <= beta |d dE| + exp rounding.
EPS_METRO = 2e-4
# |d r| <= 2.5e-6 (cos of a rounded FP32 difference), |d p| <= 2 beta J |d(r r)|.
EPS_WOLFF = 1e-4


def c0_couplings(orc, lz, seed=20260710):
    """Config-0 style couplings: J_xy = 1.2 on all layers, J_z(z) ~ U[0.5, 1.5] from seed."""
    return np.full(lz, 1.2), orc.uniform_disorder(lz, 0.5, 1.5, seed)


@pytest.fixture(scope="module")
def ctx(slsf):
    slsf.build()
    c = slsf.Context()
    yield c
    c.close()


def make_task(slsf, ctx, orc, dims, T, seed, width=math.pi, wolff=1, **kw):
    jxy, jz = c0_couplings(orc, dims[2])
    return slsf.Task(ctx, dims, jxy, jz, T, proposal_width=width, wolff_steps=wolff, seed=seed, **kw), jxy, jz


@pytest.mark.parametrize("dims", [(8, 8, 8), (6, 4, 10), (64, 64, 64)])
def test_init_random_bit_exact(slsf, ctx, orc, dims):
    t, _, _ = make_task(slsf, ctx, orc, dims, 1.1, seed=123)
    t.init_random()
    ref = orc.keyed_init_angles(t.volume, 123)
    assert np.array_equal(t.theta.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("dims,T", [((8, 8, 8), 1.1), ((16, 8, 4), 0.7), ((64, 64, 64), 1.3), ((10, 6, 4), 2.5)])
def test_metropolis_decisions_match_oracle(slsf, ctx, orc, dims, T):
    t, jxy, jz = make_task(slsf, ctx, orc, dims, T, seed=77)
    t.init_random()
    beta = np.float32(1.0 / T)
    jx32, jz32 = jxy.astype(np.float32), jz.astype(np.float32)
    total_ties = 0
    for sweep in range(3):
        t.counters = (sweep, 0)
        for colour in (0, 1):
            before = t.theta
            acc, mask = t.metropolis_color(colour)
            after = t.theta
            ref = orc.keyed_metro_half(dims, before, jx32, jz32, beta, np.float32(math.pi), 77, sweep, colour,
                                       EPS_METRO)
            is_col = ref["decision"] >= 0
            tie = ref["tie"].astype(bool)
            sure = is_col & ~tie
            assert np.array_equal(mask[sure], ref["decision"][sure].astype(np.uint8))
            assert np.all(mask[~is_col] == 0)
            same = ~tie
            assert np.array_equal(after.view(np.uint32)[same], ref["theta"].view(np.uint32)[same])
            assert acc == int(mask.sum())
            total_ties += int(tie.sum())
            # Sites where the decisions agree also agree bitwise on the new angle.
            agree = is_col & (mask == ref["decision"].astype(np.uint8))
            assert np.array_equal(after.view(np.uint32)[agree], ref["theta"].view(np.uint32)[agree])
    sites = 6 * t.volume // 2
    assert total_ties <= max(3, 4 * EPS_METRO * sites), (total_ties, sites)


def test_metropolis_width_zero_and_wrap(slsf, ctx, orc):
    # local_metropolis_step with width 0 accepts and keeps theta (src/tests.rs:163-165);
    # angles stay in [0, 2 pi) (src/tests.rs:171, :186).
    t, _, _ = make_task(slsf, ctx, orc, (8, 8, 8), 1.1, seed=5, width=0.0)
    t.init_random()
    before = t.theta
    acc = t.metropolis_sweep()
    assert acc == 1.0
    assert np.array_equal(t.theta, before)
    for width in (0.5, math.pi, 2 * math.pi):
        t2, _, _ = make_task(slsf, ctx, orc, (8, 8, 8), 0.3, seed=6, width=width)
        t2.init_random()
        for _ in range(20):
            t2.metropolis_sweep()
        th = t2.theta
        assert np.all((th >= 0) & (th < np.float32(2 * np.pi)))
    # Wider proposals keep the reference's one-step wrap (src/types.rs:334-343),
    # which can leave a representative outside [0, 2 pi); the oracle agrees bitwise.
    t3, jxy, jz = make_task(slsf, ctx, orc, (8, 8, 8), 0.3, seed=7, width=7.0)
    t3.init_random()
    before = t3.theta
    t3.counters = (0, 0)
    t3.metropolis_color(0)
    ref = orc.keyed_metro_half((8, 8, 8), before, jxy.astype(np.float32), jz.astype(np.float32),
                               np.float32(1 / 0.3), np.float32(7.0), 7, 0, 0, EPS_METRO)
    same = ref["tie"] == 0
    assert np.array_equal(t3.theta.view(np.uint32)[same], ref["theta"].view(np.uint32)[same])


@pytest.mark.parametrize("dims,T,cold", [((8, 8, 8), 1.1, False), ((12, 6, 8), 0.9, False), ((64, 64, 64), 1.3, False),
                                         ((32, 32, 32), 3.0, False), ((40, 12, 6), 1.0, False),
                                         ((96, 16, 10), 0.8, False), ((128, 24, 10), 1.2, False),
                                         ((32, 32, 32), 1.1, True), ((64, 64, 64), 1.22, True),
                                         ((96, 32, 64), 1.5, False), ((128, 64, 32), 1.22, True),
                                         ((64, 32, 96), 1.3, True), ((256, 128, 128), 1.22, True),
                                         ((128, 256, 128), 1.5, False)])
def test_wolff_cluster_bit_exact(slsf, ctx, orc, dims, T, cold):
    # Lattices of 2^22 sites and more whose sides are multiples of 32 grow
    # the seed's cluster on bit-packed bonds; the others label 32x8x4 tiles by
    # union-find.  Cold starts give clusters that span the lattice and cross
    # every region face.
    t, jxy, jz = make_task(slsf, ctx, orc, dims, T, seed=31)
    if cold:
        t.init_cold()
    else:
        t.init_random()
    for _ in range(2):
        t.metropolis_sweep()
    beta = np.float32(1.0 / T)
    jx32, jz32 = jxy.astype(np.float32), jz.astype(np.float32)
    lx, ly, lz = dims
    for step in range(3):
        t.counters = (t.counters[0], step)
        before = t.theta
        dbg = t.wolff_step_debug()
        after = t.theta
        ref = orc.keyed_wolff(dims, before, jx32, jz32, beta, 31, step, 0, EPS_WOLFF)
        phi, site = orc.keyed_wolff_pick(dims, 31, step, 0)
        assert dbg["phi"] == phi and dbg["seed_site"] == site
        tie_bits = (ref["bonds"] >> 3) & 7
        differ = (dbg["bonds"] ^ ref["bonds"]) & 7
        assert np.all((differ & ~tie_bits) == 0)
        # labelling is integer work: bit-exact against the oracle's DFS of the device bonds
        seed_idx = site[0] + lx * (site[1] + ly * site[2])
        cl, size = orc.cluster_from_bonds(dims, dbg["bonds"], seed_idx)
        assert np.array_equal(cl, dbg["cluster"])
        assert size == dbg["size"]
        if not differ.any():
            assert np.array_equal(ref["cluster"], dbg["cluster"])
        # reflection is bit-exact FP32
        expect = before.copy()
        refl = orc.keyed_wolff(dims, before, jx32, jz32, beta, 31, step, 0, 0.0)
        members = dbg["cluster"] == 1
        if np.array_equal(refl["cluster"], dbg["cluster"]):
            expect = refl["theta"]
            assert np.array_equal(after.view(np.uint32), expect.view(np.uint32))
        assert np.array_equal(after[~members], before[~members])
        assert 1 <= dbg["size"] <= t.volume


def test_large_lattice_near_transition_decisions_and_cluster(slsf, ctx, orc):
    """Large lattice near the transition (L = 256, 16.8M sites, J_xy = 1.2,
    J_z ~ U[0.5, 1.5], T = 1.22), where Wolff clusters span the lattice: from
    the cold state and 20 device sweeps (Metropolis + Wolff), both colour
    half-sweeps' accept decisions equal the oracle's outside the tie band, and
    two Wolff updates' bonds equal the oracle's outside their tie band with
    the cluster bit-exact against the oracle's DFS of the device bonds
    (src/updates.rs:238-271, :551-620)."""
    L, T, seed = 256, 1.22, 4242
    dims = (L, L, L)
    t, jxy, jz = make_task(slsf, ctx, orc, dims, T, seed=seed)
    t.init_cold()
    t.sweep(20)
    beta = np.float32(1.0 / T)
    jx32, jz32 = jxy.astype(np.float32), jz.astype(np.float32)
    sweep = t.counters[0]
    ties = 0
    for colour in (0, 1):
        before = t.theta
        acc, mask = t.metropolis_color(colour)
        ref = orc.keyed_metro_half(dims, before, jx32, jz32, beta, np.float32(math.pi), seed, sweep, colour,
                                   EPS_METRO)
        sure = (ref["decision"] >= 0) & (ref["tie"] == 0)
        assert np.array_equal(mask[sure], ref["decision"][sure].astype(np.uint8))
        assert acc == int(mask.sum())
        ties += int(ref["tie"].sum())
    assert ties <= 4 * EPS_METRO * t.volume, ties
    fractions = []
    w0 = t.counters[1]
    for step in range(2):
        t.counters = (sweep, w0 + step)  # a Wolff update's randoms are keyed by the Wolff counter
        before = t.theta
        dbg = t.wolff_step_debug()
        ref = orc.keyed_wolff(dims, before, jx32, jz32, beta, seed, w0 + step, 0, EPS_WOLFF)
        phi, site = orc.keyed_wolff_pick(dims, seed, w0 + step, 0)
        assert dbg["phi"] == phi and dbg["seed_site"] == site
        tie_bits = (ref["bonds"] >> 3) & 7
        differ = (dbg["bonds"] ^ ref["bonds"]) & 7
        assert np.all((differ & ~tie_bits) == 0)
        seed_idx = site[0] + L * (site[1] + L * site[2])
        cl, size = orc.cluster_from_bonds(dims, dbg["bonds"], seed_idx)
        assert size == dbg["size"]
        assert np.array_equal(cl, dbg["cluster"])
        members = dbg["cluster"] == 1
        assert np.array_equal(t.theta[~members], before[~members])
        fractions.append(size / t.volume)
    print(f"L=256 T=1.22: {ties} Metropolis tie sites, Wolff cluster fractions {fractions}")


@pytest.mark.parametrize("dims", [(8, 8, 8), (16, 8, 4), (64, 64, 64), (30, 14, 22)])
def test_measure_matches_oracle(slsf, ctx, orc, dims):
    t, jxy, jz = make_task(slsf, ctx, orc, dims, 1.3, seed=9)
    t.init_random()
    for _ in range(3):
        t.sweep(1)
    got = t.measure()
    ref = orc.measure_f32(dims, t.theta, jxy.astype(np.float32), jz.astype(np.float32))
    v = t.volume
    assert abs(got["energy"] - ref["energy"]) < 2e-5
    assert abs(got["magnetization_squared"] - ref["magnetization_squared"]) < 1e-5
    for k in ("cos_x", "cos_y", "cos_z", "sin_x", "sin_y", "sin_z"):
        assert abs(got[k] - ref[k]) < 2e-5 * v + 1e-5, (k, got[k], ref[k])


@pytest.mark.parametrize("L", [8, 32, 64, 256])
def test_cold_state_kat(slsf, ctx, L):
    # Cold state (src/tests.rs:93-133, :195-206): E/V = -(2 J_xy + J_z), m^2 = 1,
    # helicity cos sums = J_mu V, sin sums = 0, every correlation = 1.
    jxy, jz = np.full(L, 1.2), np.full(L, 0.6)
    t = slsf.Task(ctx, (L, L, L), jxy, jz, 1.0)
    t.init_cold()
    o = t.measure()
    v = L ** 3
    assert abs(o["energy"] + 3.0) < 1e-6
    assert abs(o["magnetization_squared"] - 1.0) < 1e-6
    assert abs(o["cos_x"] - 1.2 * v) < 1e-6 * v and abs(o["cos_z"] - 0.6 * v) < 1e-6 * v
    assert abs(o["sin_x"]) < 1e-9 * v
    c = t.correlations(4, 4)
    for key in ("corr_x", "corr_y", "corr_xy", "corr_z"):
        assert np.allclose(c[key], 1.0, atol=1e-6)
    assert np.allclose(c["corr_xy_by_z"], 1.0, atol=1e-6)


@pytest.mark.parametrize("dims,rxy,rz", [((8, 8, 8), 4, 4), ((16, 12, 20), 5, 10), ((64, 64, 64), 32, 32),
                                         ((40, 24, 256), 3, 128), ((32, 48, 30), 24, 9)])
def test_correlations_match_oracle(slsf, ctx, orc, dims, rxy, rz):
    t, _, _ = make_task(slsf, ctx, orc, dims, 1.3, seed=4)
    t.init_random()
    t.sweep(2)
    got = t.correlations(rxy, rz)
    # lags clamp to L/2 (src/observables.rs:177-181); the oracle entry takes clamped lags
    lx, ly, lz = dims
    ref = orc.correlations_f32(dims, t.theta, min(rxy, lx // 2, ly // 2), min(rz, lz // 2))
    assert len(got["corr_x"]) == min(rxy, lx // 2, ly // 2) and len(got["corr_z"]) == min(rz, lz // 2)
    assert np.allclose(got["corr_x"], ref["corr_x"], atol=2e-6)
    assert np.allclose(got["corr_y"], ref["corr_y"], atol=2e-6)
    assert np.allclose(got["corr_z"], ref["corr_z"], atol=2e-6)
    assert np.allclose(got["corr_xy_by_z"], ref["corr_xy_by_z"], atol=5e-6)
    assert np.allclose(got["corr_xy"], (got["corr_x"] + got["corr_y"]) / 2, atol=1e-12)


def test_checkerboard_layer_correlation(slsf, ctx):
    # src/tests.rs:135-148: a checkerboard of +-1 rad in layer 1 gives a negative C_xy there.
    t = slsf.Task(ctx, (2, 2, 2), np.full(2, 1.5), np.full(2, 0.5), 1.0)
    th = np.zeros((2, 2, 2), np.float32)
    for y in range(2):
        for x in range(2):
            th[1, y, x] = -1.0 if (x + y) % 2 == 0 else 1.0
    t.theta = th.ravel()
    c = t.correlations(1, 1)
    assert abs(c["corr_xy_by_z"][0, 0] - 1.0) < 1e-6
    assert c["corr_xy_by_z"][1, 0] < 0
    assert abs(c["corr_xy"][0] - c["corr_xy_by_z"][:, 0].mean()) < 1e-9


def test_reference_error_strings(slsf, ctx):
    # Exact reference messages (src/types.rs:120-129, :373-385; updates.rs:430-438; model.rs:318-348).
    def err(fn):
        with pytest.raises(slsf.SlsfError) as e:
            fn()
        return str(e.value)

    ones = np.ones(4)
    assert err(lambda: slsf.Task(ctx, (0, 4, 4), ones, ones, 1.0)) == "L_x must be positive"
    assert err(lambda: slsf.Task(ctx, (4, 0, 4), ones, ones, 1.0)) == "L_y must be positive"
    assert err(lambda: slsf.Task(ctx, (4, 4, 0), ones[:0], ones[:0], 1.0)) == "L_z must be positive"
    assert err(lambda: slsf.Task(ctx, (4, 4, 4), ones[:3], ones, 1.0)) == "J_xy_array length must match Lz"
    assert err(lambda: slsf.Task(ctx, (4, 4, 4), ones, ones[:3], 1.0)) == "J_z_array length must match Lz"
    assert err(lambda: slsf.Task(ctx, (4, 4, 4), ones, -ones, 1.0)) == \
        "theta simulation requires nonnegative layer couplings"
    odd = slsf.Task(ctx, (3, 3, 3), np.ones(3), np.ones(3), 1.0)
    odd.init_random()
    assert err(odd.metropolis_sweep) == "red-black Metropolis sweep requires even lattice dimensions"
    assert err(lambda: odd.sweep(1)) == "red-black Metropolis sweep requires even lattice dimensions"
    odd.measure()  # measurement works on any lattice
    for bad_t in (0.0, -1.0, math.inf, math.nan):
        bt = slsf.Task(ctx, (4, 4, 4), ones, ones, bad_t)
        assert err(bt.metropolis_sweep) == "temperature T must be positive and finite"
        assert err(bt.wolff_step) == "temperature T must be positive and finite"
    for bad_w in (-0.1, math.inf, math.nan):
        bw = slsf.Task(ctx, (4, 4, 4), ones, ones, 1.0, proposal_width=bad_w)
        assert err(bw.metropolis_sweep) == "proposal_width must be nonnegative and finite"


def test_wolff_reflection_involution_and_sizes(slsf, ctx, orc):
    # src/tests.rs:372-432: cluster size in [1, V], angles wrapped, repeated steps work.
    t, _, _ = make_task(slsf, ctx, orc, (4, 4, 4), 1.0, seed=15)
    t.init_random()
    for _ in range(4):
        n = t.wolff_step()
        assert 1 <= n <= 64
    th = t.theta
    assert np.all((th >= 0) & (th < np.float32(2 * np.pi)))
