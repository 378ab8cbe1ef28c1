"""Job files run on the GPU (marked gpu): served tasks equal the model
driver's results, correlated task groups equal the single-task path
(sweep, measure, correlations every `correlation_interval` measurements),
the rank split covers the job, and the command line writes the reference's
result layout (src/tests.rs:568-607)."""
import ctypes
import importlib
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def jobs(slsf):
    slsf.build()
    return importlib.import_module("slsf_rs_b200.jobs")


@pytest.fixture(scope="module")
def ctx(slsf):
    c = slsf.Context()
    yield c
    c.close()


SERVED = """
name = "served_unit"
[model]
L = [4, 6]
T = [1.0, 1.5]
djz = [0.25]
j_z = 0.5
samples = 2
base_seed = 31
[run]
sweeps = 16
thermalization = 4
binsize = 4
[measure]
corr_rmax = [0, 0]
"""

CORRELATED = """
name = "corr_unit"
[model]
l_x = [8]
l_y = [4]
l_z = [4, 6]
T = [1.2]
djxy = [0.25]
samples = 2
base_seed = 5
[run]
sweeps = 12
thermalization = 3
binsize = 3
wolff_steps = 2
[measure]
corr_interval = 2
"""


def test_served_job_equals_model_driver(slsf, ctx, jobs):
    cfg = jobs.config_from_toml(SERVED)
    res = jobs.run_job(ctx, cfg, epoch_sweeps=5)
    assert res["job_name"] == "served_unit" and len(res["tasks"]) == 8
    for rec in res["tasks"]:
        t = rec["task"]
        assert rec["measurements"] == 16
        assert not any(k.startswith("Corr") for k in rec["observables"])
        d = slsf.theta_task((t["l_x"], t["l_y"], t["l_z"]), t["temperature"], t["sweeps"], t["thermalization"],
                            t["binsize"], t["seed"], j_xy_array=t["j_xy_array"], j_z_array=t["j_z_array"])
        ref = slsf.model_run(ctx, d, batched=True)
        assert rec["acceptance"] == ref["acceptance"]
        for name in slsf.BIN_NAMES + slsf.DERIVED:
            got = rec["observables"][name]
            assert got["mean"] == pytest.approx(ref[name][0], rel=1e-12, abs=1e-14), (t["name"], name)
            assert got["error"] == pytest.approx(ref[name][1], rel=1e-9, abs=1e-14), (t["name"], name)


def single_task_path(slsf, ctx, t):
    """The reference's schedule on the single-task entry points."""
    dims = (t["l_x"], t["l_y"], t["l_z"])
    task = slsf.Task(ctx, dims, t["j_xy_array"], t["j_z_array"], t["temperature"],
                     proposal_width=t["proposal_width"], wolff_steps=t["wolff_steps"], seed=t["seed"])
    task.init_random()
    accepted = task.sweep(t["thermalization"])["accepted"] if t["thermalization"] else 0
    rows, corr = [], []
    for m in range(t["sweeps"]):
        accepted += task.sweep(1)["accepted"]
        o = task.measure()
        rows.append([o["energy"], o["energy"] ** 2, o["magnetization_squared"], o["cos_x"], o["cos_y"], o["cos_z"],
                     o["sin_x"], o["sin_y"], o["sin_z"], o["sin_x"] ** 2, o["sin_y"] ** 2, o["sin_z"] ** 2])
        if m % t["correlation_interval"] == 0:
            c = task.correlations(t["correlation_rmax_xy"], t["correlation_rmax_z"])
            corr.append(np.concatenate([c["corr_x"], c["corr_y"], c["corr_xy"], c["corr_xy_by_z"].ravel(),
                                        c["corr_z"]]))
    task.close()
    b = t["binsize"]
    nb = t["sweeps"] // b
    bins = np.ascontiguousarray(np.array(rows)[: nb * b].reshape(nb, b, slsf.BIN_COLS).mean(axis=1))
    e = slsf.Estimates()
    slsf.host_check(slsf.load_host().slsf_estimates_from_bins(
        bins.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nb, float(np.prod(dims)), 1.0 / t["temperature"],
        ctypes.byref(e)))
    return e.as_dict(), np.array(corr), accepted / (np.prod(dims) * (t["thermalization"] + t["sweeps"]))


def test_correlated_job_equals_single_task_path(slsf, ctx, jobs):
    cfg = jobs.config_from_toml(CORRELATED)
    res = jobs.run_job(ctx, cfg)
    assert len(res["tasks"]) == 4
    for rec in res["tasks"]:
        t = rec["task"]
        assert t["correlation_rmax_xy"] == 2 and t["correlation_rmax_z"] == t["l_z"] // 2
        est, corr, acc = single_task_path(slsf, ctx, t)
        assert rec["measurements"] == 12 and corr.shape[0] == 6
        assert rec["acceptance"] == pytest.approx(acc, rel=0, abs=0)
        names = jobs.corr_names(t["l_z"], t["correlation_rmax_xy"], t["correlation_rmax_z"])
        assert sorted(n for n in rec["observables"] if n.startswith("Corr")) == sorted(names)
        for j, name in enumerate(names):
            # same trajectory; measured inside the sweeps (the job's lattices fit
            # the one-CTA kernel) against the separate kernels: FP32 partial sums
            ref = slsf.binned_estimate(corr[:, j], 3)
            got = rec["observables"][name]
            assert abs(got["mean"] - ref["mean"]) < 2e-6 and abs(got["error"] - ref["stderr"]) < 2e-6, name
        for name in slsf.BIN_NAMES + slsf.DERIVED:
            # batched bins reduce in FP32 per site, the grid measure in FP64
            x, y = rec["observables"][name]["mean"], est[name][0]
            assert abs(x - y) <= 1e-4 * max(1.0, abs(y)), (t["name"], name, x, y)


def test_rank_split_covers_job(slsf, ctx, jobs):
    cfg = jobs.config_from_toml(SERVED)
    tasks = jobs.make_tasks(cfg)
    whole = jobs.run_job(ctx, cfg, tasks=tasks)
    parts = [jobs.run_job(ctx, cfg, rank=r, world_size=3, tasks=tasks) for r in range(3)]
    by_name = {rec["task"]["name"]: rec for rec in whole["tasks"]}
    seen = []
    for r, p in enumerate(parts):
        assert p["rank"] == r and p["world_size"] == 3
        for rec in p["tasks"]:
            assert rec.get("task_index", 0) % 3 == r
            assert rec["observables"] == by_name[rec["task"]["name"]]["observables"]
            seen.append(rec["task"]["name"])
    assert sorted(seen) == sorted(by_name)


def test_command_line_writes_result(slsf, jobs, tmp_path):
    # theta_carlo_runner_writes_master_compatible_result (src/tests.rs:568-607)
    job = tmp_path / "carlo_unit.toml"
    job.write_text('name = "carlo_unit"\n[model]\nL = [2]\nT = [2.0]\nsamples = 1\n'
                   '[run]\nsweeps = 4\nthermalization = 2\nbinsize = 2\nwolff_steps = 1\n[measure]\ncorr_rmax = [1]\n')
    assert jobs.main([str(job), "--output-dir", str(tmp_path / "out")]) == 0
    out = json.loads((tmp_path / "out" / "carlo_unit.rank0.results.json").read_text())
    assert out["job_name"] == "carlo_unit" and out["rank"] == 0 and out["world_size"] == 1
    [task] = out["tasks"]
    assert "task_index" not in task and task["measurements"] == 4 and np.isfinite(task["acceptance"])
    for name in ("Energy", "RhoXY", "RhoZ", "Magnetization", "CorrX_r1", "CorrZ_r1", "CorrXY_z1_r1"):
        assert np.isfinite(task["observables"][name]["mean"]), name
    assert task["task"]["name"] == "L2x2x2_T2.000000_dJxy0.000000_dJz0.000000_sample1"
    # the measurement file beside it (src/tests.rs:606): bins of every measured observable
    h5 = tmp_path / "out" / "carlo_unit.data" / "task0001" / "run0001.meas.h5"
    assert h5.exists()
    check_meas_h5(slsf, h5, task, n_plain_bins=2, corr_bin_len=2, n_corr_bins=2)


def check_meas_h5(slsf, path, rec, n_plain_bins, corr_bin_len=None, n_corr_bins=None):
    """The .meas.h5 of one task read back with the specification reader: each
    measured observable's bins, whose mean is the record's estimate."""
    import h5read

    r = h5read.read(str(path))
    names = sorted(k.split("/")[2] for k in r if k.count("/") == 2 and k.startswith("/observables/"))
    corr = sorted(n for n in rec["observables"] if n.startswith("Corr"))
    assert names == sorted(list(slsf.BIN_NAMES) + corr)
    for name in names:
        bl = int(r[f"/observables/{name}/bin_length"].value)
        s = r[f"/observables/{name}/samples"].value
        if name.startswith("Corr"):
            assert (bl, len(s)) == (corr_bin_len, n_corr_bins), name
        else:
            assert (bl, len(s)) == (rec["task"]["binsize"], n_plain_bins), name
        assert s.mean() == pytest.approx(rec["observables"][name]["mean"], rel=1e-12, abs=1e-15), name
    assert r["/version/mc_package"].value == "SLSF.XYCarlo"


def test_served_job_writes_measurement_files(slsf, jobs, tmp_path):
    job = tmp_path / "served_unit.toml"
    job.write_text(SERVED)
    assert jobs.main([str(job), "--output-dir", str(tmp_path / "out")]) == 0
    out = json.loads((tmp_path / "out" / "served_unit.rank0.results.json").read_text())
    assert len(out["tasks"]) == 8
    for rec in out["tasks"]:
        k = rec.get("task_index", 0)
        check_meas_h5(slsf, tmp_path / "out" / "served_unit.data" / f"task{k + 1:04d}" / "run0001.meas.h5", rec,
                      n_plain_bins=16 // 4)


# TINY_CONFIG of theta_model_runs_through_carlo_runner (src/model.rs:484-498)
TINY = """
name = "tiny"
[model]
l = [2]
temperatures = [2.0]
samples = 1
j_xy = 1.0
j_z_mean = 0.1
delta_j_xy = [0.0]
delta_j_z = [0.0]
[run]
sweeps = 4
thermalization = 2
binsize = 2
wolff_steps = 1
"""


def test_theta_model_runs_through_runner(slsf, ctx, jobs):
    # theta_model_runs_through_carlo_runner (src/model.rs:500-515): one task,
    # not stopped early, completed, with Energy and MagnetizationSquared.
    cfg = jobs.config_from_toml(TINY)
    tasks = jobs.make_tasks(cfg)
    assert len(tasks) == 1
    res, summary = jobs.run_job_checkpointed(ctx, cfg, tasks=tasks)
    assert not summary["stopped_early"]
    assert len(res["tasks"]) == 1
    [rec] = res["tasks"]
    assert rec["measurements"] == 4  # completed: every post-thermalization sweep measured
    assert "Energy" in rec["observables"] and "MagnetizationSquared" in rec["observables"]
    assert all(np.isfinite(v["mean"]) for v in rec["observables"].values())


class StopAt:
    """A checkpoint schedule that asks for a stop at its n-th check."""

    def __init__(self, jobs, directory, n, restart=False):
        self.inner = jobs.Checkpoints(directory, restart)
        self.n = n
        self.dir = self.inner.dir
        self.restart = restart

    def wait_s(self):
        return 0.001

    def due(self):
        self.n -= 1
        return "stop" if self.n <= 0 else None

    def saved(self):
        pass

    def path(self, *parts):
        return self.inner.path(*parts)


LONG_SERVED = SERVED.replace("L = [4, 6]", "L = [16, 32]").replace("sweeps = 16", "sweeps = 3000")
# 243 sweeps: three CUDA-graph replays of at most 100 sweeps, checkpoint checks between them
LONG_CORRELATED = CORRELATED.replace("sweeps = 12", "sweeps = 240")


@pytest.mark.parametrize("text,n_stop", [(LONG_SERVED, 1), (LONG_CORRELATED, 2)])
def test_stop_and_restart_equals_uninterrupted(slsf, ctx, jobs, tmp_path, text, n_stop):
    cfg = jobs.config_from_toml(text)
    whole = jobs.run_job(ctx, cfg, epoch_sweeps=50)
    first, s1 = jobs.run_job_checkpointed(ctx, cfg, epoch_sweeps=50, ck=StopAt(jobs, tmp_path, n_stop))
    assert s1["stopped_early"] and len(first["tasks"]) < len(whole["tasks"])
    again, s2 = jobs.run_job_checkpointed(ctx, cfg, epoch_sweeps=50,
                                          ck=jobs.Checkpoints(tmp_path, restart=True))
    assert not s2["stopped_early"]
    want = {r["task"]["name"]: r for r in whole["tasks"]}
    got = {r["task"]["name"]: r for r in again["tasks"]}
    assert sorted(got) == sorted(want)
    for name, rec in got.items():
        w = want[name]
        assert rec["measurements"] == w["measurements"] and rec["acceptance"] == w["acceptance"]
        assert sorted(rec["observables"]) == sorted(w["observables"])
        for obs, v in rec["observables"].items():
            assert v["mean"] == pytest.approx(w["observables"][obs]["mean"], rel=1e-12, abs=1e-15), (name, obs)
    # a restart of a finished run reads the saved results back
    third, s3 = jobs.run_job_checkpointed(ctx, cfg, epoch_sweeps=50, ck=jobs.Checkpoints(tmp_path, restart=True))
    assert third["tasks"] == again["tasks"]


def test_merge_and_status(slsf, ctx, jobs, tmp_path):
    cfg = jobs.config_from_toml(SERVED)
    parts = [jobs.run_job(ctx, cfg, rank=r, world_size=2) for r in range(2)]
    for r, p in enumerate(parts):
        jobs.write_result(p, jobs.result_path(cfg, r, str(tmp_path)))
    assert jobs.status(cfg, 2, str(tmp_path)) == "8 theta task(s) completed; 2 of 2 rank result file(s) present"
    job = tmp_path / "job.toml"
    job.write_text(SERVED)
    assert jobs.main([str(job), "merge", "--world-size", "2", "--output-dir", str(tmp_path)]) == 0
    merged = json.loads((tmp_path / "served_unit.results.json").read_text())
    assert merged["rank"] == 0 and len(merged["tasks"]) == 8
    names = [t["task"]["name"] for t in merged["tasks"]]
    assert names == sorted(names)
    with pytest.raises(jobs.JobError):
        jobs.merge_results([parts[0], dict(parts[1], job_name="other")])
