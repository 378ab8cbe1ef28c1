"""Observables at the benchmarked configurations within 2 sigma of the
reference's CPU path (marked gpu).

The reference judges a simulation by its binned estimates: Energy,
MagnetizationSquared and the helicity moduli RhoXY, RhoZ
(src/model.rs:857-888).  Each test runs the same (J_xy, J_z, T) on both
sides -- the device through the path the benchmark times, the oracle through
the reference-order CPU path with its own FastRng streams -- with
independent replicas on each side:

  - every replica runs THERM sweeps, then MEAS measured sweeps cut into
    N_BINS bins; its Energy and MagnetizationSquared are the mean of its bins,
    its RhoXY and RhoZ the evaluables of its bin means (or_evaluate_derived,
    the same plug-in estimate on both sides, so both carry the same
    finite-sample bias);
  - a side's value for a configuration is the mean over its replicas, its
    error the replicas' standard error.  Independent replicas need no
    assumption about autocorrelation times: at L = 32 in the ordered phase
    the magnetisation decorrelates over more than a bin of 20 sweeps, and
    binned errors (printed beside) come out 1.4-1.6x too small;
  - z = (device - oracle) / sqrt(err_dev^2 + err_cpu^2) per configuration and
    observable; the pooled z of an observable sums the differences over all
    configurations against the summed variances.

Bars: every pooled |z| < 2 (the 2-sigma criterion); over the per-configuration
z (Student-like with the oracle's 15 degrees of freedom) the mean z^2 < 2.2
and max |z| < 4.
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BASE_SEED = 20260710
OBS = ("Energy", "MagnetizationSquared", "RhoXY", "RhoZ")


@pytest.fixture(scope="module")
def ctx(slsf):
    slsf.build()
    c = slsf.Context()
    yield c
    c.close()


def replica_estimates(orc, bin_means, volume, beta):
    """(value, error) per replica and observable from each replica's bin means [R][n_bins][12]."""
    out = np.zeros((len(bin_means), len(OBS), 2))
    nb = bin_means.shape[1]
    for r, bm in enumerate(bin_means):
        out[r, 0] = bm[:, 0].mean(), bm[:, 0].std(ddof=1) / math.sqrt(nb)
        out[r, 1] = bm[:, 2].mean(), bm[:, 2].std(ddof=1) / math.sqrt(nb)
        d = orc.evaluate_derived(bm, volume, beta)
        out[r, 2] = d["RhoXY"]
        out[r, 3] = d["RhoZ"]
    return out


def side_summary(est):
    """Mean over replicas, its standard error over replicas, and the error the replicas' bins give."""
    r = est.shape[0]
    mean = est[:, :, 0].mean(axis=0)
    err = est[:, :, 0].std(axis=0, ddof=1) / math.sqrt(r)
    binned = np.sqrt((est[:, :, 1] ** 2).sum(axis=0)) / r
    return mean, err, binned


def compare(configs):
    """configs: list of (label, device estimates, oracle estimates). Returns the report and asserts the bars."""
    diffs = np.zeros((len(configs), len(OBS)))
    var = np.zeros_like(diffs)
    rows = []
    for k, (label, dev, cpu) in enumerate(configs):
        gm, ge, gs = side_summary(dev)
        cm, ce, cs = side_summary(cpu)
        diffs[k] = gm - cm
        var[k] = ge ** 2 + ce ** 2
        z = diffs[k] / np.sqrt(var[k])
        rows.append((label, z))
        for i, name in enumerate(OBS):
            print(f"  {label:<28s} {name:<21s} dev {gm[i]: .6f} +- {ge[i]:.2e} (binned {gs[i]:.2e})  "
                  f"cpu {cm[i]: .6f} +- {ce[i]:.2e} (binned {cs[i]:.2e})  z {z[i]: .2f}")
    zs = np.array([z for _, z in rows])
    pooled = diffs.sum(axis=0) / np.sqrt(var.sum(axis=0))
    report = {name: {"pooled_z": float(pooled[i]), "mean_z2": float((zs[:, i] ** 2).mean()),
                     "max_abs_z": float(np.abs(zs[:, i]).max())} for i, name in enumerate(OBS)}
    print("2-sigma report:", report)
    for name, r in report.items():
        assert abs(r["pooled_z"]) < 2.0, (name, report)
    assert (zs ** 2).mean() < 2.2, report
    assert np.abs(zs).max() < 4.0, report
    return report


def cpu_threads():
    return os.cpu_count() or 1


def test_two_sigma_batched_replicas_l32(slsf, ctx, orc):
    """Batched replicas (L = 32, J_xy = 1.2, J_z(z) ~ U[0.5, 1.5] per disorder
    realisation, T in [1.1, 1.5], Metropolis width pi + one Wolff per sweep):
    4 disorder realisations (disorder seeds 20260710 + s - 1, s = 1..4) x 4
    of the 16 benchmark temperatures (1.1, 1.2333, 1.3667, 1.5).  Device: 32
    replicas per configuration, 512 in one batch session whose steps replay
    the CUDA graph of the one-CTA persistent kernel (100 sweeps per step, 5
    steps: 100 thermalization + 400 measured sweeps, 20 bins of 20).  Oracle:
    16 replicas per configuration, the same sweeps and bins."""
    L, therm, meas, n_bins = 32, 100, 400, 20
    R_dev, R_cpu = 32, 16
    temps = np.linspace(1.1, 1.5, 16)[[0, 5, 10, 15]]
    ctx.tune_set((L, L, L), "resident", 1, 1024)
    configs = []
    for s in range(1, 5):
        jz = slsf.uniform_layer_disorder(L, 0.5, 1.5, BASE_SEED + s - 1)
        for T in temps:
            configs.append((s, float(T), np.full(L, 1.2), jz))
    tasks = []
    for s, T, jxy, jz in configs:
        seed0 = slsf.task_seed(BASE_SEED, L, s, T)
        for r in range(R_dev):
            t = slsf.Task(ctx, (L, L, L), jxy, jz, T, wolff_steps=1, seed=seed0 + 7919 * r, thermalization=therm,
                          binsize=meas // n_bins, n_bins=n_bins)
            t.init_random()
            tasks.append(t)
    with ctx.session(tasks, 100) as ses:
        for _ in range((therm + meas) // 100):
            ses.step()
    dev_bins, measured = ctx.batch_bins(tasks, n_bins)
    assert np.all(measured == meas)
    for t in tasks:
        t.close()

    n_cfg = len(configs)
    jxy_all = np.repeat(np.array([c[2] for c in configs]), R_cpu, axis=0)
    jz_all = np.repeat(np.array([c[3] for c in configs]), R_cpu, axis=0)
    t_all = np.repeat([c[1] for c in configs], R_cpu)
    seeds = [900_000 + k for k in range(n_cfg * R_cpu)]
    cpu_bins = orc.series_tasks((L, L, L), jxy_all, jz_all, t_all, seeds, therm, meas, n_bins,
                                threads=cpu_threads())
    v = float(L ** 3)
    rows = []
    for k, (s, T, _, _) in enumerate(configs):
        dev = replica_estimates(orc, dev_bins[k * R_dev:(k + 1) * R_dev], v, 1.0 / T)
        cpu = replica_estimates(orc, cpu_bins[k * R_cpu:(k + 1) * R_cpu], v, 1.0 / T)
        rows.append((f"L=32 sample {s} T={T:.4f}", dev, cpu))
    compare(rows)


def test_two_sigma_single_large_replica_l64(slsf, ctx, orc):
    """Single large replica (L = 64, J_xy = 1.2, J_z(z) ~ U[0.5, 1.5] from the
    disorder seed 20260710, T = 1.3, Metropolis width pi + one Wolff per sweep,
    measured every sweep): 100 thermalization + 400 measured sweeps in 20
    bins, on both device paths -- the batched cluster kernel (8 CTAs of 1024
    threads per replica; 24 replicas) and the single-task kernels driven as
    ThetaModel is, one sweep then one measurement per call (16 replicas) --
    against 16 replicas of the oracle."""
    L, T, therm, meas, n_bins = 64, 1.3, 100, 400, 20
    R_cluster, R_plain, R_cpu = 24, 16, 16
    jxy = np.full(L, 1.2)
    jz = slsf.uniform_layer_disorder(L, 0.5, 1.5, BASE_SEED)
    seed0 = slsf.task_seed(BASE_SEED, L, 1, T)
    ctx.tune_set((L, L, L), "cluster", 8, 1024)
    tasks = []
    for r in range(R_cluster):
        t = slsf.Task(ctx, (L, L, L), jxy, jz, T, wolff_steps=1, seed=seed0 + 7919 * r, thermalization=therm,
                      binsize=meas // n_bins, n_bins=n_bins)
        t.init_random()
        tasks.append(t)
    for _ in range((therm + meas) // 100):
        ctx.batch_run(tasks, 100)
    cluster_bins, measured = ctx.batch_bins(tasks, n_bins)
    assert np.all(measured == meas)
    for t in tasks:
        t.close()

    plain_bins = np.zeros((R_plain, n_bins, 12))
    for r in range(R_plain):
        t = slsf.Task(ctx, (L, L, L), jxy, jz, T, wolff_steps=1, seed=seed0 + 104_729 * (r + 1))
        t.init_random()
        t.sweep(therm)
        series = np.zeros((meas, 12))
        for s in range(meas):
            t.sweep(1)
            o = t.measure()
            series[s] = [o["energy"], o["energy"] ** 2, o["magnetization_squared"], o["cos_x"], o["cos_y"],
                         o["cos_z"], o["sin_x"], o["sin_y"], o["sin_z"], o["sin_x"] ** 2, o["sin_y"] ** 2,
                         o["sin_z"] ** 2]
        plain_bins[r] = series.reshape(n_bins, meas // n_bins, 12).mean(axis=1)
        t.close()

    cpu_bins = orc.series_tasks((L, L, L), np.tile(jxy, (R_cpu, 1)), np.tile(jz, (R_cpu, 1)), [T] * R_cpu,
                                [700_000 + r for r in range(R_cpu)], therm, meas, n_bins, threads=cpu_threads())
    v, beta = float(L ** 3), 1.0 / T
    cpu = replica_estimates(orc, cpu_bins, v, beta)
    # each device path against the oracle on its own (they share the oracle's side)
    compare([("L=64 T=1.3 cluster kernel", replica_estimates(orc, cluster_bins, v, beta), cpu)])
    compare([("L=64 T=1.3 single-task path", replica_estimates(orc, plain_bins, v, beta), cpu)])
