"""Job files on the CPU: the TOML schema with its aliases and defaults,
durations, task expansion (order, names, seeds, couplings, correlation
radii), validation messages, the rank split and the result path.  The
known answers are the reference's own (src/tests.rs:448-566); nothing here
launches a kernel."""
import importlib
import os
import re
import math

import numpy as np
import pytest


@pytest.fixture(scope="module")
def jobs(slsf):
    slsf.build()
    return importlib.import_module("slsf_rs_b200.jobs")


def cfg_of(jobs, **kw):
    c = jobs.JobConfig()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def test_defaults_follow_reference(jobs):
    c = jobs.JobConfig()
    assert c.l == list(range(4, 21)) and c.temperatures == [2.8, 2.9, 3.0, 3.1, 3.2, 3.3]
    assert (c.samples, c.base_seed, c.j_xy, c.j_z_mean) == (16, 20260414, 1.0, 0.1)
    assert (c.sweeps, c.thermalization, c.binsize, c.wolff_steps) == (20000, 5000, 50, 1)
    assert c.proposal_width == math.pi and c.correlation_interval == 1
    assert (c.run_time_s, c.checkpoint_time_s, c.job_name) == (43200, 1800, "xy_theta_rust")


def test_unit_job_expansion_and_rank_split(jobs, slsf):
    # src/tests.rs:448-479
    c = cfg_of(jobs, l=[2], temperatures=[1.0, 1.5], delta_j_z=[0.0], samples=2, base_seed=17, sweeps=4,
               thermalization=1, binsize=2, wolff_steps=0, correlation_rmax=[0], correlation_interval=2,
               job_name="unit_theta_job")
    tasks = jobs.make_tasks(c)
    assert len(tasks) == 4
    t0 = tasks[0]
    assert (t0["l"], t0["l_x"], t0["l_y"], t0["l_z"]) == (2, 2, 2, 2)
    assert t0["binsize"] == 2 and t0["correlation_interval"] == 2
    assert len(t0["j_xy_array"]) == 2 and len(t0["j_z_array"]) == 2
    assert jobs.selected(len(tasks), 1, 2) == [1, 3]
    assert jobs.selected(len(tasks), 0, 1) == [0, 1, 2, 3]
    # order: temperature, then sample, innermost
    assert [(t["temperature"], t["sample"]) for t in tasks] == [(1.0, 1), (1.0, 2), (1.5, 1), (1.5, 2)]
    assert [t["disorder_seed"] for t in tasks] == [17, 18, 17, 18]
    assert tasks[0]["name"] == "L2x2x2_T1.000000_dJxy0.000000_dJz0.000000_sample1"
    # correlation_rmax given, the xy and z radii fall back to the shape (struct, not TOML)
    assert t0["correlation_rmax"] == 0 and t0["correlation_rmax_xy"] == 1 and t0["correlation_rmax_z"] == 1


def test_explicit_dims(jobs):
    # src/tests.rs:481-498
    c = cfg_of(jobs, l=[4], l_x=[2], l_y=[3], l_z=[5], temperatures=[1.0], delta_j_z=[0.0], samples=1, sweeps=2,
               binsize=1)
    [t] = jobs.make_tasks(c)
    assert (t["l"], t["l_x"], t["l_y"], t["l_z"]) == (5, 2, 3, 5)
    # per-axis lists form a product; a missing axis falls back to l
    c = cfg_of(jobs, l=[4, 6], l_x=[8], l_z=[2, 10])
    assert jobs.lattice_specs(c) == [(8, 4, 2, 2), (8, 4, 10, 10), (8, 6, 2, 2), (8, 6, 10, 10)]


def test_correlation_radii_per_lattice(jobs):
    # src/tests.rs:527-546
    c = cfg_of(jobs, l=[16, 32], temperatures=[1.0], delta_j_z=[0.0], samples=1, sweeps=2, binsize=1,
               correlation_rmax=[8, 16], correlation_rmax_xy=[7, 15], correlation_rmax_z=[6, 14])
    t = jobs.make_tasks(c)
    assert [(x["l"], x["correlation_rmax"], x["correlation_rmax_xy"], x["correlation_rmax_z"]) for x in t] == \
        [(16, 8, 7, 6), (32, 16, 15, 14)]
    d = jobs.make_tasks(cfg_of(jobs, l=[6], l_x=[10], l_y=[4], l_z=[12], temperatures=[1.0], samples=1, sweeps=2,
                               binsize=1))[0]
    assert (d["correlation_rmax"], d["correlation_rmax_xy"], d["correlation_rmax_z"]) == (6, 2, 6)


def test_seeds_and_couplings(jobs, slsf, orc):
    c = cfg_of(jobs, l=[4, 8], temperatures=[0.9, 1.25], delta_j_xy=[0.0, 0.25], delta_j_z=[0.5], samples=3,
               base_seed=20260410, j_xy=1.0, j_z_mean=0.75, sweeps=10, binsize=5)
    tasks = jobs.make_tasks(c)
    assert len(tasks) == 2 * 2 * 1 * 2 * 3
    k = 0
    for l in (4, 8):
        for djxy in (0.0, 0.25):
            for T in (0.9, 1.25):
                for s in (1, 2, 3):
                    t = tasks[k]
                    k += 1
                    assert (t["l"], t["delta_j_xy"], t["temperature"], t["sample"]) == (l, djxy, T, s)
                    assert t["seed"] == slsf.task_seed(20260410, l, s, T, djxy, 0.5)
                    rng = orc.FastRng(20260410 + s - 1)
                    assert t["j_xy_array"] == list(orc.two_point_disorder(l, 1.0, djxy, rng, "J_xy"))
                    assert t["j_z_array"] == list(orc.two_point_disorder(l, 0.75, 0.5, rng, "J_z"))
    assert tasks[-1]["name"] == "L8x8x8_T1.250000_dJxy0.250000_dJz0.500000_sample3"


def test_seed_cast_saturates(slsf):
    # `x.round() as u64` maps negatives to 0 (src/model.rs:741-747)
    host = slsf.load_host()
    assert slsf.task_seed(100, 4, 1, -1.0, 0.0, 0.0) == 100 + 400000 + 1000
    assert host.slsf_task_seed(100, 4, 1, -1.0, -0.5, 0.0) == slsf.task_seed(100, 4, 1, -1.0, -0.5, 0.0)
    assert host.slsf_task_seed(0, 2, 1, 0.005, 0.0, 0.0) == slsf.task_seed(0, 2, 1, 0.005, 0.0, 0.0) == 201001


@pytest.mark.parametrize("kw,message", [
    (dict(l=[]), "at least one lattice size must be configured"),
    (dict(l=[16, 32], correlation_rmax_xy=[16]),
     "corr_rmax_xy must contain exactly one value per lattice size: expected 2, got 1"),
    (dict(l=[4], correlation_rmax=[1, 2]), "corr_rmax must contain exactly one value per lattice size: expected 1, "
                                           "got 2"),
    (dict(temperatures=[]), "at least one temperature must be configured"),
    (dict(delta_j_xy=[]), "delta_j_xy and delta_j_z must not be empty"),
    (dict(delta_j_z=[]), "delta_j_xy and delta_j_z must not be empty"),
    (dict(samples=0), "samples must be positive"),
    (dict(binsize=0), "binsize must be positive"),
    (dict(correlation_interval=0), "correlation_interval must be positive"),
    (dict(sweeps=10, binsize=11), "sweeps must be at least binsize"),
    (dict(l=[4], delta_j_z=[0.2]), "two-point layer disorder requires J_z_mean - δJ_z >= 0"),
    (dict(l=[4], delta_j_xy=[-0.1]), "δJ_xy must be nonnegative"),
])
def test_expansion_errors(jobs, kw, message):
    with pytest.raises(jobs.JobError) as e:
        jobs.make_tasks(cfg_of(jobs, **kw))
    assert str(e.value) == message


@pytest.mark.parametrize("text,seconds", [("1-02:03:04", 93784), ("05:06", 306), ("17", 17), ("2-5", 172805),
                                          ("0:0:0", 0), ("12:00:00", 43200), ("+3", 3)])
def test_parse_duration(jobs, text, seconds):
    assert jobs.parse_duration(text) == seconds


@pytest.mark.parametrize("text,fragment", [("48:invalid:00", "failed to parse duration component in 48:invalid:00"),
                                           ("1:2:3:4", "1:2:3:4 does not match [[HH:]MM:]SS"),
                                           ("x-01:00", "failed to parse duration days in x-01:00"),
                                           ("-5", "cannot parse integer from empty string"),
                                           ("1:-2", "invalid digit found in string")])
def test_parse_duration_errors(jobs, text, fragment):
    with pytest.raises(jobs.JobError) as e:
        jobs.parse_duration(text)
    assert fragment in str(e.value)


def test_toml_top_level_and_durations(jobs):
    # src/tests.rs:500-513
    c = jobs.config_from_toml('name = "carlo_mpi_params"\nrun_time = "1-02:03:04"\ncheckpoint_time = "05:06"\n'
                              'checkpoint = true\n')
    assert c.job_name == "carlo_mpi_params" and c.run_time_s == 93784 and c.checkpoint_time_s == 306
    with pytest.raises(jobs.JobError) as e:
        jobs.config_from_toml('run_time = "48:invalid:00"\n')
    assert "invalid run_time" in str(e.value)
    with pytest.raises(jobs.JobError) as e:
        jobs.config_from_toml('checkpoint_time = "1:2:3:4"\n')
    assert str(e.value) == "invalid checkpoint_time: 1:2:3:4 does not match [[HH:]MM:]SS"


def test_toml_measure_section(jobs):
    # src/tests.rs:515-525: corr_rmax feeds the xy and z radii; corr_interval is an alias
    c = jobs.config_from_toml("[measure]\ncorr_rmax = [1, 2]\ncorr_interval = 3\n")
    assert c.correlation_rmax == [1, 2] and c.correlation_interval == 3
    assert c.correlation_rmax_xy == [1, 2] and c.correlation_rmax_z == [1, 2]
    c = jobs.config_from_toml("[measure]\ncorr_rmax = [4]\ncorr_rmax_z = [1]\ncorrelation_interval = 5\n"
                              "corr_interval = 9\n")
    assert c.correlation_rmax_xy == [4] and c.correlation_rmax_z == [1] and c.correlation_interval == 5
    # without [measure] the radii stay unset (defaults from the shape at expansion)
    assert jobs.config_from_toml("").correlation_rmax is None


def test_toml_model_and_run_aliases(jobs):
    text = """
name = "runs/aniso"
output_dir = "out"
[model]
L = [8, 12]
T = [1.1, 1.2]
djz = [0.25]
djxy = [0.125]
j_z = 0.5
samples = 3
base_seed = 99
j_xy = 1.5
[run]
sweeps = 200
thermalization = 20
binsize = 10
proposal_width = 1.0
wolff_steps = 2
"""
    c = jobs.config_from_toml(text)
    assert c.l == [8, 12] and c.temperatures == [1.1, 1.2] and c.delta_j_z == [0.25] and c.delta_j_xy == [0.125]
    assert (c.j_z_mean, c.samples, c.base_seed, c.j_xy) == (0.5, 3, 99, 1.5)
    assert (c.sweeps, c.thermalization, c.binsize, c.proposal_width, c.wolff_steps) == (200, 20, 10, 1.0, 2)
    assert c.output_dir == "out"
    # the long names win over the short ones; `t` is read after `T`/`temperatures`
    c = jobs.config_from_toml("[model]\nt = [2.0]\ndelta_j_z = [0.1]\ndjz = [0.3]\nj_z_mean = 0.2\nj_z = 0.9\n")
    assert c.temperatures == [2.0] and c.delta_j_z == [0.1] and c.j_z_mean == 0.2
    c = jobs.config_from_toml("[model]\ntemperatures = [2.5]\nt = [2.0]\n")
    assert c.temperatures == [2.5]


@pytest.mark.parametrize("text,fragment", [
    ("[model]\nL = [4]\nl = [6]\n", "duplicate field `l`"),
    ("[model]\nsamples = -1\n", "invalid type for `model.samples`"),
    ("[model]\nL = [4.5]\n", "invalid type for `model.L`"),
    ("[run]\nsweeps = \"10\"\n", "invalid type for `run.sweeps`"),
    ("run_time = 5\n", "invalid type for `run_time`"),
    ("[model\n", ""),
])
def test_toml_type_errors(jobs, text, fragment):
    with pytest.raises(jobs.JobError) as e:
        jobs.config_from_toml(text)
    assert fragment in str(e.value)


def test_result_path(jobs, monkeypatch):
    monkeypatch.delenv("XY_OUTPUT_DIR", raising=False)
    c = jobs.config_from_toml('name = "runs/aniso"\n')
    assert jobs.result_path(c, 3) == "runs/aniso.rank3.results.json"
    assert jobs.result_path(jobs.JobConfig(), 0) == "results/xy_theta_rust.rank0.results.json"
    assert jobs.result_path(c, 0, "elsewhere") == "elsewhere/aniso.rank0.results.json"
    monkeypatch.setenv("XY_OUTPUT_DIR", "envdir")
    assert jobs.result_path(c, 1) == "envdir/aniso.rank1.results.json"
    c.output_dir = "fromtoml"
    assert jobs.result_path(c, 1) == "fromtoml/aniso.rank1.results.json"


def test_correlation_names_order(jobs):
    names = jobs.corr_names(2, 2, 1)
    assert names == ["CorrX_r1", "CorrX_r2", "CorrY_r1", "CorrY_r2", "CorrXY_r1", "CorrXY_r2", "CorrXY_z0_r1",
                     "CorrXY_z0_r2", "CorrXY_z1_r1", "CorrXY_z1_r2", "CorrZ_r1"]
    assert jobs.measures_correlations({"correlation_rmax_xy": 0, "correlation_rmax_z": 1})
    assert not jobs.measures_correlations({"correlation_rmax_xy": 0, "correlation_rmax_z": 0})


def test_couplings_equal_host_draw(jobs, slsf):
    c = cfg_of(jobs, l=[6], temperatures=[1.0], delta_j_xy=[0.5], delta_j_z=[0.1], samples=2, base_seed=5,
               sweeps=2, binsize=1)
    for t in jobs.make_tasks(c):
        d = slsf.theta_task((6, 6, 6), 1.0, 2, 0, 1, t["seed"], disorder_seed=t["disorder_seed"], j_xy=1.0,
                            delta_j_xy=0.5, j_z_mean=0.1, delta_j_z=0.1)
        jx, jz = slsf.task_couplings(d)
        assert np.array_equal(jx, t["j_xy_array"]) and np.array_equal(jz, t["j_z_array"])
        assert set(jx) <= {0.5, 1.5} and set(np.round(jz, 12)) <= {0.0, 0.2}


# Directory of the reference's example job files (its `examples/`), given by
# the environment; the test is skipped where it is not set.
REFERENCE_EXAMPLES = os.environ.get("SLSF_REFERENCE_EXAMPLES", "")


@pytest.mark.skipif(not REFERENCE_EXAMPLES or not os.path.isdir(REFERENCE_EXAMPLES),
                    reason="SLSF_REFERENCE_EXAMPLES does not name the reference's example job files")
def test_reference_example_job_files_parse_and_expand(jobs):
    # Every job file the reference ships parses, and expands to one task per
    # lattice x dJxy x dJz x T x sample with the reference's name format.
    names = sorted(f for f in os.listdir(REFERENCE_EXAMPLES) if f.endswith(".toml"))
    assert names
    for name in names:
        cfg = jobs.load_job(os.path.join(REFERENCE_EXAMPLES, name))
        specs = jobs.lattice_specs(cfg)
        expected = len(specs) * len(cfg.delta_j_xy) * len(cfg.delta_j_z) * len(cfg.temperatures) * cfg.samples
        if expected > 5000:
            cfg.samples = 1  # the production files hold up to 20000 tasks: expand one sample of each
            expected = len(specs) * len(cfg.delta_j_xy) * len(cfg.delta_j_z) * len(cfg.temperatures)
        tasks = jobs.make_tasks(cfg)
        assert len(tasks) == expected, name
        assert all(re.fullmatch(r"L\d+x\d+x\d+_T\d+\.\d{6}_dJxy\d+\.\d{6}_dJz\d+\.\d{6}_sample\d+", t["name"])
                   for t in tasks), name
        assert cfg.run_time_s > 0 and cfg.checkpoint_time_s > 0


def test_tiny_config_builds_one_task(jobs):
    # the parse half of theta_model_runs_through_carlo_runner (src/model.rs:500-504);
    # the run half is in test_gpu_jobs.py
    from test_gpu_jobs import TINY

    [t] = jobs.make_tasks(jobs.config_from_toml(TINY))
    assert t["name"] == "L2x2x2_T2.000000_dJxy0.000000_dJz0.000000_sample1"
    assert (t["l_x"], t["l_y"], t["l_z"], t["temperature"]) == (2, 2, 2, 2.0)
    assert t["j_xy_array"] == [1.0, 1.0] and t["j_z_array"] == [0.1, 0.1]
    assert (t["sweeps"], t["thermalization"], t["binsize"], t["wolff_steps"]) == (4, 2, 2, 1)


def test_measurement_bins_mapping_and_checkpoint_round_trip(jobs, slsf):
    # a task's measurement_bins (src/model.rs:81) from its estimates: the
    # twelve per-sweep columns and the correlation columns, each with its own
    # bin length; they survive the JSON form the checkpoints keep
    rows = np.arange(3 * slsf.BIN_COLS, dtype=np.float64).reshape(3, slsf.BIN_COLS)
    corr = np.array([[0.5, 0.25], [0.75, 0.125]])
    est = {"Energy": (1.0, 0.1), "n_bins": 3, "_bins": {"binsize": 4, "rows": rows},
           "_corr_bins": {"binsize": 2, "names": ["CorrX_r1", "CorrZ_r1"], "rows": corr}}
    bins = jobs.measurement_bins(est)
    assert sorted(bins) == sorted(list(slsf.BIN_NAMES) + ["CorrX_r1", "CorrZ_r1"])
    for j, name in enumerate(slsf.BIN_NAMES):
        assert bins[name][0] == 4 and np.array_equal(bins[name][1], rows[:, j])
    assert bins["CorrZ_r1"][0] == 2 and np.array_equal(bins["CorrZ_r1"][1], corr[:, 1])
    import json

    back = jobs._est_from_json(json.loads(json.dumps(jobs._est_to_json(est))))
    assert back["Energy"] == (1.0, 0.1)
    again = jobs.measurement_bins(back)
    assert sorted(again) == sorted(bins)
    for name in bins:
        assert again[name][0] == bins[name][0] and np.array_equal(again[name][1], bins[name][1])
    # a served task without a complete bin keeps no bins
    assert jobs.measurement_bins({"_bins": {"binsize": 4, "rows": np.zeros((0, slsf.BIN_COLS))}}) == {}
