"""Job files for the B200 path: the reference's TOML job schema, its task
expansion, and a runner that feeds the tasks to the batched kernels.

The reference reads a job file into a `ThetaJobConfig` (src/model.rs:159-213
for the schema, :552-637 for defaults and key aliases, :1033-1060 for
durations) and expands it with `make_theta_tasks` (src/model.rs:697-810):
every lattice shape x delta J_xy x delta J_z x temperature x sample becomes
one task with disorder seed `base_seed + sample - 1`, its run seed from the
seed formula and two-point layer couplings drawn J_xy first, then J_z, from
FastRng(disorder_seed).  This module restates those steps; the seed formula
and the disorder draw are the host library's (slsf_task_seed,
slsf_task_couplings).

`run_job` runs a rank's share of the tasks (task index modulo world size,
ThetaJob::selected_tasks, src/model.rs:60-68):

* tasks without correlation measurements go to the continuous-batching
  server (batched persistent launches, bins kept on the device);
* tasks that measure correlations (the reference's default: r_max = L/2) run
  as groups through the batched kernels too (ThetaModel::measure,
  src/model.rs:402-442), binned on the device: replicas that fit the
  one-CTA kernel measure them inside the sweeps (slsf_task_corr_fuse);
  other groups stop every `correlation_interval` measurements for one
  batched correlation launch.  The trajectories are the ones the single-task
  path produces.

The result has the reference's ThetaJobResult layout (src/model.rs:72-106:
job_name, rank, world_size, tasks[] with task, observables{name: {mean,
error}}, acceptance, measurements) and is written to
`<output_dir>/<job file stem>.rank<r>.results.json`.

    python slsf-rs_b200/jobs.py job.toml [--output-dir DIR] [--rank R --world-size N]
"""
from __future__ import annotations

import dataclasses
import importlib.util
import json
import math
import os
import re
import sys
from collections.abc import Mapping
from typing import Optional

import numpy as np


def _package():
    """The package this file belongs to (importable by path: its directory
    name is not a Python identifier)."""
    if __package__:
        return sys.modules[__package__]
    name = "slsf_rs_b200"
    if name in sys.modules:
        return sys.modules[name]
    here = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location(name, os.path.join(here, "__init__.py"),
                                                  submodule_search_locations=[here])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


class JobError(ValueError):
    """A job file or configuration the reference rejects (with its message)."""


@dataclasses.dataclass
class JobConfig:
    """ThetaJobConfig with the reference's defaults (src/model.rs:519-546)."""

    l: list = dataclasses.field(default_factory=lambda: list(range(4, 21)))
    l_x: Optional[list] = None
    l_y: Optional[list] = None
    l_z: Optional[list] = None
    temperatures: list = dataclasses.field(default_factory=lambda: [2.8, 2.9, 3.0, 3.1, 3.2, 3.3])
    delta_j_z: list = dataclasses.field(default_factory=lambda: [0.0])
    delta_j_xy: list = dataclasses.field(default_factory=lambda: [0.0])
    samples: int = 16
    base_seed: int = 20260414
    j_xy: float = 1.0
    j_z_mean: float = 0.1
    sweeps: int = 20_000
    thermalization: int = 5_000
    binsize: int = 50
    proposal_width: float = math.pi
    wolff_steps: int = 1
    correlation_rmax: Optional[list] = None
    correlation_rmax_xy: Optional[list] = None
    correlation_rmax_z: Optional[list] = None
    correlation_interval: int = 1
    run_time_s: int = 12 * 60 * 60
    checkpoint_time_s: int = 30 * 60
    job_name: str = "xy_theta_rust"
    output_dir: Optional[str] = None
    checkpoint: bool = False


def _u64(text: str, what: str, value: str) -> int:
    """str::parse::<u64> (an optional '+', then decimal digits), with Rust's messages."""
    if text == "":
        raise JobError(f"failed to parse duration {what} in {value}: cannot parse integer from empty string")
    if not re.fullmatch(r"\+?[0-9]+", text):
        raise JobError(f"failed to parse duration {what} in {value}: invalid digit found in string")
    return int(text)


def parse_duration(value: str) -> int:
    """`[D-][[HH:]MM:]SS` to seconds (parse_duration, src/model.rs:1033-1060)."""
    days, rest = value.split("-", 1) if "-" in value else ("0", value)
    d = _u64(days, "days", value)
    parts = rest.split(":")
    if len(parts) > 3:
        raise JobError(f"{value} does not match [[HH:]MM:]SS")
    nums = [_u64(p, "component", value) for p in parts]
    h, m, s = ([0, 0] + nums)[-3:]
    return d * 86400 + h * 3600 + m * 60 + s


def _check_types(section: str, table: dict, kinds: dict):
    """serde's type checks for the keys this schema knows (unknown keys are
    ignored, as serde does without deny_unknown_fields)."""
    for key, kind in kinds.items():
        if key not in table:
            continue
        v = table[key]
        if kind == "usize_list":
            ok = isinstance(v, list) and all(isinstance(x, int) and not isinstance(x, bool) and x >= 0 for x in v)
        elif kind == "f64_list":
            ok = isinstance(v, list) and all(isinstance(x, (int, float)) and not isinstance(x, bool) for x in v)
        elif kind == "usize":
            ok = isinstance(v, int) and not isinstance(v, bool) and v >= 0
        elif kind == "f64":
            ok = isinstance(v, (int, float)) and not isinstance(v, bool)
        elif kind == "bool":
            ok = isinstance(v, bool)
        else:
            ok = isinstance(v, str)
        if not ok:
            raise JobError(f"invalid type for `{section}{key}`: expected {kind.replace('_list', ' list')}")


_TOP = {"name": "str", "output_dir": "str", "output_file": "str", "merged_output_file": "str",
        "measurement_dir": "str", "checkpoint_dir": "str", "scheduler_dir": "str", "checkpoint": "bool",
        "run_time": "str", "checkpoint_time": "str"}
_MODEL = {"l": "usize_list", "L": "usize_list", "l_x": "usize_list", "l_y": "usize_list", "l_z": "usize_list",
          "temperatures": "f64_list", "T": "f64_list", "t": "f64_list", "delta_j_z": "f64_list", "djz": "f64_list",
          "samples": "usize", "base_seed": "usize", "j_xy": "f64", "delta_j_xy": "f64_list", "djxy": "f64_list",
          "j_z_mean": "f64", "j_z": "f64"}
_RUN = {"sweeps": "usize", "thermalization": "usize", "binsize": "usize", "proposal_width": "f64",
        "wolff_steps": "usize"}
_MEASURE = {"corr_rmax": "usize_list", "corr_rmax_xy": "usize_list", "corr_rmax_z": "usize_list",
            "corr_interval": "usize", "correlation_interval": "usize"}


def config_from_toml(text: str) -> JobConfig:
    """ThetaJobConfig::try_from_toml_spec (src/model.rs:568-637) with the
    schema's aliases: L for l, T for temperatures, then t; djz, djxy and
    j_z as fallbacks of delta_j_z, delta_j_xy and j_z_mean; corr_interval
    for correlation_interval; corr_rmax as the default of corr_rmax_xy and
    corr_rmax_z."""
    import tomllib

    try:
        spec = tomllib.loads(text)
    except tomllib.TOMLDecodeError as e:
        raise JobError(str(e)) from None
    _check_types("", spec, _TOP)
    model, run, measure = spec.get("model"), spec.get("run"), spec.get("measure")
    for name, table, kinds in (("model", model, _MODEL), ("run", run, _RUN), ("measure", measure, _MEASURE)):
        if table is not None:
            if not isinstance(table, dict):
                raise JobError(f"invalid type for `{name}`: expected a table")
            _check_types(name + ".", table, kinds)
    for a, b in (("l", "L"), ("temperatures", "T")):
        if model and a in model and b in model:
            raise JobError(f"duplicate field `{a}`")
    cfg = JobConfig()
    if "name" in spec:
        cfg.job_name = spec["name"]
    cfg.output_dir = spec.get("output_dir")
    cfg.checkpoint = bool(spec.get("checkpoint", False))
    if "run_time" in spec:
        try:
            cfg.run_time_s = parse_duration(spec["run_time"])
        except JobError as e:
            raise JobError(f"invalid run_time: {e}") from None
    if "checkpoint_time" in spec:
        try:
            cfg.checkpoint_time_s = parse_duration(spec["checkpoint_time"])
        except JobError as e:
            raise JobError(f"invalid checkpoint_time: {e}") from None

    def first(d, *keys):
        for k in keys:
            if k in d:
                return d[k]
        return None

    if model is not None:
        if (v := first(model, "l", "L")) is not None:
            cfg.l = list(v)
        cfg.l_x, cfg.l_y, cfg.l_z = model.get("l_x"), model.get("l_y"), model.get("l_z")
        if (v := first(model, "temperatures", "T", "t")) is not None:
            cfg.temperatures = [float(x) for x in v]
        if (v := first(model, "delta_j_z", "djz")) is not None:
            cfg.delta_j_z = [float(x) for x in v]
        if (v := first(model, "delta_j_xy", "djxy")) is not None:
            cfg.delta_j_xy = [float(x) for x in v]
        if "samples" in model:
            cfg.samples = model["samples"]
        if "base_seed" in model:
            cfg.base_seed = model["base_seed"]
        if "j_xy" in model:
            cfg.j_xy = float(model["j_xy"])
        if (v := first(model, "j_z_mean", "j_z")) is not None:
            cfg.j_z_mean = float(v)
    if run is not None:
        for key in ("sweeps", "thermalization", "binsize", "wolff_steps"):
            if key in run:
                setattr(cfg, key, run[key])
        if "proposal_width" in run:
            cfg.proposal_width = float(run["proposal_width"])
    if measure is not None:
        cfg.correlation_rmax = measure.get("corr_rmax")
        cfg.correlation_rmax_xy = measure.get("corr_rmax_xy", cfg.correlation_rmax)
        cfg.correlation_rmax_z = measure.get("corr_rmax_z", cfg.correlation_rmax)
        if (v := first(measure, "correlation_interval", "corr_interval")) is not None:
            cfg.correlation_interval = v
    return cfg


def load_job(path: str) -> JobConfig:
    with open(path, encoding="utf-8") as f:
        return config_from_toml(f.read())


def lattice_specs(cfg: JobConfig):
    """(l_x, l_y, l_z, l) per lattice (ThetaJobConfig::lattice_specs,
    src/model.rs:812-828): cubic from `l`, else the product of the per-axis
    lists (an absent list falls back to `l`) with l = l_z."""
    if cfg.l_x is None and cfg.l_y is None and cfg.l_z is None:
        return [(l, l, l, l) for l in cfg.l]
    xs = cfg.l_x if cfg.l_x is not None else cfg.l
    ys = cfg.l_y if cfg.l_y is not None else cfg.l
    zs = cfg.l_z if cfg.l_z is not None else cfg.l
    return [(x, y, z, z) for x in xs for y in ys for z in zs]


def make_tasks(cfg: JobConfig):
    """make_theta_tasks (src/model.rs:697-810): the ThetaTask records, in the
    reference's order, with its validation messages."""
    pkg = _package()
    specs = lattice_specs(cfg)
    if not specs:
        raise JobError("at least one lattice size must be configured")
    for name, values in (("corr_rmax", cfg.correlation_rmax), ("corr_rmax_xy", cfg.correlation_rmax_xy),
                         ("corr_rmax_z", cfg.correlation_rmax_z)):
        if values is not None and len(values) != len(specs):
            raise JobError(f"{name} must contain exactly one value per lattice size: expected {len(specs)}, "
                           f"got {len(values)}")
    if not cfg.temperatures:
        raise JobError("at least one temperature must be configured")
    if not cfg.delta_j_xy or not cfg.delta_j_z:
        raise JobError("delta_j_xy and delta_j_z must not be empty")
    if cfg.samples == 0:
        raise JobError("samples must be positive")
    if cfg.binsize == 0:
        raise JobError("binsize must be positive")
    if cfg.correlation_interval == 0:
        raise JobError("correlation_interval must be positive")
    if cfg.sweeps < cfg.binsize:
        raise JobError("sweeps must be at least binsize")
    host = pkg.load_host()
    tasks = []
    for li, (lx, ly, lz, l) in enumerate(specs):
        for djxy in cfg.delta_j_xy:
            for djz in cfg.delta_j_z:
                for T in cfg.temperatures:
                    for sample in range(1, cfg.samples + 1):
                        dseed = cfg.base_seed + sample - 1
                        seed = int(host.slsf_task_seed(cfg.base_seed, lz, sample, T, djxy, djz))
                        desc = pkg.theta_task((lx, ly, lz), T, cfg.sweeps, cfg.thermalization, cfg.binsize, seed,
                                              disorder_seed=dseed, j_xy=cfg.j_xy, delta_j_xy=djxy,
                                              j_z_mean=cfg.j_z_mean, delta_j_z=djz)
                        try:
                            jx, jz = pkg.task_couplings(desc)
                        except pkg.SlsfError as e:
                            raise JobError(str(e)) from None
                        tasks.append({
                            "name": f"L{lx}x{ly}x{lz}_T{T:.6f}_dJxy{djxy:.6f}_dJz{djz:.6f}_sample{sample}",
                            "l": l, "l_x": lx, "l_y": ly, "l_z": lz, "temperature": T, "j_xy": cfg.j_xy,
                            "delta_j_xy": djxy, "j_z_mean": cfg.j_z_mean, "delta_j_z": djz,
                            "disorder_seed": dseed, "seed": seed, "sample": sample, "sweeps": cfg.sweeps,
                            "thermalization": cfg.thermalization, "binsize": cfg.binsize,
                            "proposal_width": cfg.proposal_width, "wolff_steps": cfg.wolff_steps,
                            "correlation_rmax": (cfg.correlation_rmax[li] if cfg.correlation_rmax is not None
                                                 else lz // 2),
                            "correlation_rmax_xy": (cfg.correlation_rmax_xy[li]
                                                    if cfg.correlation_rmax_xy is not None else min(lx, ly) // 2),
                            "correlation_rmax_z": (cfg.correlation_rmax_z[li] if cfg.correlation_rmax_z is not None
                                                   else lz // 2),
                            "correlation_interval": cfg.correlation_interval,
                            "j_xy_array": jx.tolist(), "j_z_array": jz.tolist(),
                        })
    return tasks


def selected(n_tasks: int, rank: int, world_size: int):
    """Task indices of one rank (ThetaJob::selected_tasks, src/model.rs:60-68)."""
    return [k for k in range(n_tasks) if world_size == 1 or k % world_size == rank]


def measures_correlations(task) -> bool:
    """ThetaModel::measure's condition (src/model.rs:410)."""
    return task["correlation_rmax_xy"] > 0 or task["correlation_rmax_z"] > 0


def corr_names(lz, rxy, rz):
    """Observable names of one correlation measurement, in ThetaModel::measure's
    order (src/model.rs:420-437); r counts from 1, z from 0."""
    names = [f"CorrX_r{r}" for r in range(1, rxy + 1)] + [f"CorrY_r{r}" for r in range(1, rxy + 1)]
    names += [f"CorrXY_r{r}" for r in range(1, rxy + 1)]
    names += [f"CorrXY_z{z}_r{r}" for z in range(lz) for r in range(1, rxy + 1)]
    names += [f"CorrZ_r{r}" for r in range(1, rz + 1)]
    return names


def _observables(est: dict, corr: Optional[dict] = None):
    out = {k: {"mean": v[0], "error": v[1]} for k, v in est.items() if isinstance(v, tuple)}
    for name, (mean, err) in (corr or {}).items():
        out[name] = {"mean": mean, "error": err}
    return dict(sorted(out.items()))


class Stopped(Exception):
    """The run time ran out; the checkpoint holds the unfinished work."""


class Checkpoints:
    """carlo-mc's run-time and checkpoint-time schedule (ThetaJobConfig
    run_time / checkpoint_time, src/model.rs:140-156) over a checkpoint
    directory: a checkpoint every `every_s` seconds, and at `run_time_s` a
    last one and a stop.  With restart, work saved in the directory is
    resumed instead of started again."""

    def __init__(self, directory, restart=False, run_time_s=None, every_s=None):
        import time

        self.dir = str(directory)
        self.restart = restart
        self.t0 = self.last = time.monotonic()
        self.run_time_s = float("inf") if run_time_s is None else float(run_time_s)
        self.every_s = float("inf") if every_s is None else float(every_s)
        os.makedirs(self.dir, exist_ok=True)

    def wait_s(self):
        import time

        now = time.monotonic()
        return min(365 * 86400.0, max(0.01, min(self.last + self.every_s, self.t0 + self.run_time_s) - now))

    def due(self):
        """None, "checkpoint" or "stop"."""
        import time

        now = time.monotonic()
        if now >= self.t0 + self.run_time_s:
            return "stop"
        if now >= self.last + self.every_s:
            return "checkpoint"
        return None

    def saved(self):
        import time

        self.last = time.monotonic()

    def path(self, *parts):
        return os.path.join(self.dir, *parts)


def _swap_dir(new, old):
    """Replaces directory `old` by `new` (a checkpoint is whole or absent)."""
    import shutil

    if os.path.isdir(old):
        shutil.rmtree(old)
    os.replace(new, old)


def _jsonable(v):
    if isinstance(v, np.ndarray):
        return v.tolist()
    if isinstance(v, dict):
        return {k: _jsonable(x) for k, x in v.items()}
    return v


def _est_to_json(est):
    return {k: (list(v) if isinstance(v, tuple) else _jsonable(v)) for k, v in est.items()}


def _est_from_json(d):
    return {k: (tuple(v) if isinstance(v, list) else v) for k, v in d.items()}


def _run_served(pkg, ctx, tasks, epoch_sweeps, ck: Optional[Checkpoints] = None):
    """Tasks without correlations through the server: {task index: estimates}.
    With checkpoints the server is stopped at each one, its finished results
    kept in served/finished.json and its unfinished requests written by
    slsf_server_checkpoint to served/; a restart restores both."""
    names = {k: t["name"] for k, t in tasks}
    binsizes = {k: t["binsize"] for k, t in tasks}
    srv = pkg.Server(ctx, epoch_sweeps=epoch_sweeps, keep_bins=True)
    out = {}

    def collect():
        for r in srv.poll(len(tasks) + 16):
            if r["status"] != pkg.OK:
                raise pkg.SlsfError(r["status"], f"task {names[r['tag']]}: {r['message']}")
            est = r["est"]
            rows = srv.take_bins(r["tag"]) if est["n_bins"] else np.zeros((0, pkg.BIN_COLS))  # none kept
            est["_bins"] = {"binsize": binsizes[r["tag"]], "rows": rows}
            out[r["tag"]] = est

    try:
        sdir = ck.path("served") if ck else None
        if ck and ck.restart and os.path.isdir(sdir):
            with open(os.path.join(sdir, "finished.json"), encoding="utf-8") as f:
                out.update({int(k): _est_from_json(v) for k, v in json.load(f).items()})
            srv.restore(sdir)
        else:
            for k, t in tasks:
                srv.submit(k, (t["l_x"], t["l_y"], t["l_z"]), t["temperature"], t["seed"], t["j_xy_array"],
                           t["j_z_array"], t["thermalization"] + t["sweeps"], thermalization=t["thermalization"],
                           proposal_width=t["proposal_width"], wolff_steps=t["wolff_steps"], binsize=t["binsize"])
        srv.start()
        while True:
            try:
                srv.wait_idle(ck.wait_s() if ck else 365 * 86400.0)
                break
            except pkg.SlsfError as e:
                if e.code != pkg.ERR_TIMEOUT or ck is None:
                    raise
            due = ck.due()
            if due is None:
                continue
            srv.stop()
            collect()
            tmp = sdir + ".new"
            os.makedirs(tmp, exist_ok=True)
            with open(os.path.join(tmp, "finished.json"), "w", encoding="utf-8") as f:
                json.dump({str(k): _est_to_json(v) for k, v in out.items()}, f)
            srv.checkpoint(tmp)
            _swap_dir(tmp, sdir)
            ck.saved()
            if due == "stop":
                raise Stopped(out)
            srv.start()
        srv.stop()
        collect()
        if ck:
            # all finished: the checkpoint keeps the results and no requests
            tmp = sdir + ".new"
            os.makedirs(tmp, exist_ok=True)
            with open(os.path.join(tmp, "finished.json"), "w", encoding="utf-8") as f:
                json.dump({str(k): _est_to_json(v) for k, v in out.items()}, f)
            _swap_dir(tmp, sdir)
    finally:
        srv.close()
    return out


def _run_correlated(pkg, ctx, group, ck: Optional[Checkpoints] = None, gdir: Optional[str] = None):
    """One group of tasks sharing (thermalization, sweeps, correlation_interval)
    through the batched kernels: thermalization, then per correlation
    measurement m (m % interval == 0) the sweeps up to it and one batched
    correlation launch that adds every task's values into its correlation bins
    on the device.  A correlation series is binned with the task's bin size
    (BinnedEstimate::from_samples); a series shorter than one bin forms one
    bin.  When every replica fits the one-CTA kernel the measurements happen
    inside the sweeps instead (slsf_task_corr_fuse) and the run is plain
    batched sweeps.  With checkpoints, every task's device state (slsf_task_state_save,
    the acceptance count riding in its caller words) goes to `gdir` between
    measurements when one is due; a restart loads them and continues."""
    import ctypes as C

    if ck and ck.restart and os.path.exists(os.path.join(gdir, "finished.json")):
        with open(os.path.join(gdir, "finished.json"), encoding="utf-8") as f:
            saved = json.load(f)
        return [(_est_from_json(e), {k: tuple(v) for k, v in c.items()}) for e, c in saved]
    t0 = group[0][1]
    therm, sweeps, interval = t0["thermalization"], t0["sweeps"], t0["correlation_interval"]
    n_corr = (sweeps + interval - 1) // interval
    objs, radii = [], []
    session = None
    try:
        for _, t in group:
            o = pkg.Task(ctx, (t["l_x"], t["l_y"], t["l_z"]), t["j_xy_array"], t["j_z_array"], t["temperature"],
                         proposal_width=t["proposal_width"], wolff_steps=t["wolff_steps"], seed=t["seed"],
                         thermalization=therm, binsize=t["binsize"], n_bins=t["sweeps"] // t["binsize"])
            objs.append(o)
            radii.append((min(t["correlation_rmax_xy"], t["l_x"] // 2, t["l_y"] // 2),
                          min(t["correlation_rmax_z"], t["l_z"] // 2)))
            cb = min(t["binsize"], n_corr)
            o.corr_setup(*radii[-1], cb, n_corr // cb)
        accepted = np.zeros(len(objs), dtype=np.uint64)
        resumed = ck and ck.restart and os.path.isdir(gdir)
        for i, o in enumerate(objs):
            if resumed:
                with open(os.path.join(gdir, f"task_{group[i][0]}.state"), "rb") as f:
                    accepted[i] = o.load_state(f.read())[0]
            else:
                o.init_random()
        handles = ctx.handle_array(objs)
        measured = [o for o in objs if o.corr_n_values]
        corr_handles = ctx.handle_array(measured)
        pos = objs[0].counters[0]
        corr_done = measured[0].corr_bins(0)[1] if measured else 0

        def advance(n):
            # sweeps outside whole measurement cycles (thermalization, the
            # first measurement's sweep, the tail): one batched call
            nonlocal pos, session
            if not n:
                return
            if session:
                session.close()
                session = False
            for i, st in enumerate(ctx.batch_run(objs, n, handles)):
                accepted[i] += st["accepted"]
            pos += n

        def save(due):
            if due == "stop" and session:
                session.close()
            tmp = gdir + ".new"
            os.makedirs(tmp, exist_ok=True)
            for i, o in enumerate(objs):
                with open(os.path.join(tmp, f"task_{group[i][0]}.state"), "wb") as f:
                    f.write(o.save_state(user=(int(accepted[i]), 0, 0, 0)))
            _swap_dir(tmp, gdir)
            ck.saved()
            if due == "stop":
                raise Stopped()

        # Replicas that fit the one-CTA kernel measure their correlations
        # inside the sweeps (slsf_task_corr_fuse): the whole run is then
        # batched sweeps, 100 per CUDA-graph replay, checkpoint checks between.
        fused = len(measured) == len(objs)
        if fused:
            try:
                for o in objs:
                    o.corr_fuse(interval)
            except pkg.SlsfError as e:
                if e.code != pkg.ERR_INVALID:
                    raise
                for o in objs:
                    o.corr_fuse(0)
                fused = False
        chunk = 100
        while fused and pos < therm + sweeps:
            n = min(chunk, therm + sweeps - pos)
            if n == chunk and session is not False:
                if session is None:
                    try:
                        session = ctx.session(objs, chunk)
                    except pkg.SlsfError as e:
                        if e.code != pkg.ERR_INVALID:
                            raise
                        session = False
                        continue
                for i, st in enumerate(session.step()):
                    accepted[i] += st["accepted"]
                pos += n
            else:
                advance(n)
            if ck and (due := ck.due()):
                save(due)
        if pos < therm:
            advance(therm - pos)
        m_idx = n_corr if fused else corr_done
        while m_idx < n_corr:
            n = therm + m_idx * interval + 1 - pos
            if n == interval and len(measured) == len(objs) and session is not False:
                # whole cycles (interval sweeps + a correlation measurement)
                # run in the library, up to 64 between checkpoint checks
                if session is None:
                    try:
                        session = ctx.session(objs, interval)
                    except pkg.SlsfError as e:
                        if e.code != pkg.ERR_INVALID:
                            raise
                        session = False
                        continue
                k = min(64, n_corr - m_idx)
                accepted += session.step_correlations(k)[:, 1]
                pos += k * interval
                m_idx += k
            else:
                advance(n)
                if measured:
                    ctx.batch_correlations(measured, corr_handles)
                m_idx += 1
            if ck and (due := ck.due()):
                save(due)
        advance(therm + sweeps - pos)
        if session:
            session.close()
        host = pkg.load_host()
        out = []
        for i, ((_, t), o) in enumerate(zip(group, objs)):
            volume = float(t["l_x"] * t["l_y"] * t["l_z"])
            bins, meas = o.bins()
            b = np.ascontiguousarray(bins)
            e = pkg.Estimates()
            pkg.host_check(host.slsf_estimates_from_bins(b.ctypes.data_as(C.POINTER(C.c_double)), len(b), volume,
                                                         1.0 / t["temperature"], C.byref(e)))
            est = e.as_dict()
            est["measurements"] = meas
            est["acceptance"] = float(accepted[i]) / (volume * (therm + sweeps))
            est["_bins"] = {"binsize": t["binsize"], "rows": b}
            corr = {}
            if o.corr_n_values:
                means, count = o.corr_bins()
                assert count == n_corr
                names = corr_names(t["l_z"], *radii[i])
                for j, name in enumerate(names):
                    # bins of one mean each: the mean of the bin means and their standard error
                    r = pkg.binned_estimate(means[:, j], 1)
                    corr[name] = (r["mean"], r["stderr"])
                est["_corr_bins"] = {"binsize": min(t["binsize"], n_corr), "names": names, "rows": means}
            out.append((est, corr))
        if ck:
            tmp = gdir + ".new"
            os.makedirs(tmp, exist_ok=True)
            with open(os.path.join(tmp, "finished.json"), "w", encoding="utf-8") as f:
                json.dump([[_est_to_json(e), {k: list(v) for k, v in c.items()}] for e, c in out], f)
            _swap_dir(tmp, gdir)
        return out
    finally:
        if session:
            session.close()
        for o in objs:
            o.close()


def measurement_bins(est: dict) -> dict:
    """A task's measurement_bins (ThetaTaskResult, src/model.rs:81) from its
    estimates: {observable: (internal bin length, bin means)} for the twelve
    per-sweep observables and, when measured, every correlation observable.
    The reference's two per-sweep timing series (_ll_sweep_time,
    _ll_measure_time, src/model.rs:438-439) have no counterpart in batched
    sweeps and are left out."""
    out = {}
    b = est.get("_bins")
    if b is not None and len(b["rows"]):
        cols = np.asarray(b["rows"], dtype=np.float64).T
        out.update(zip(_package().BIN_NAMES, ((b["binsize"], col) for col in cols)))
    c = est.get("_corr_bins")
    if c is not None and len(c["rows"]):
        cols = np.asarray(c["rows"], dtype=np.float64).T
        out.update(zip(c["names"], ((c["binsize"], col) for col in cols)))
    return out


class _TaskBins(Mapping):
    """{task index: measurement_bins} over a run's estimates, built when read."""

    def __init__(self, estimates):
        self._est = estimates

    def __getitem__(self, k):
        return measurement_bins(self._est[k])

    def __iter__(self):
        return iter(self._est)

    def __len__(self):
        return len(self._est)


def run_job_checkpointed(ctx, cfg: JobConfig, rank: int = 0, world_size: int = 1, epoch_sweeps: int = 100,
                         tasks=None, group_size: int = 1024, ck: Optional[Checkpoints] = None):
    """A rank's share of the job; returns (ThetaJobResult record, summary).
    Without `ck` every task runs to the end.  With it, the run stops once
    its run time is spent, after a last checkpoint; the record then holds
    the finished tasks only and the summary says stopped_early (JobRunSummary,
    src/model.rs:108-115)."""
    import time

    pkg = _package()
    started = time.monotonic()
    tasks = tasks if tasks is not None else make_tasks(cfg)
    mine = [(k, tasks[k]) for k in selected(len(tasks), rank, world_size)]
    served = [(k, t) for k, t in mine if not measures_correlations(t)]
    est, corr = {}, {}
    stopped = False
    try:
        if served:
            est.update(_run_served(pkg, ctx, served, epoch_sweeps, ck))
        groups = {}
        for k, t in mine:
            if measures_correlations(t):
                groups.setdefault((t["thermalization"], t["sweeps"], t["correlation_interval"]), []).append((k, t))
        for (therm, sweeps, interval), members in groups.items():
            for lo in range(0, len(members), group_size):
                chunk = members[lo: lo + group_size]
                gdir = ck.path(f"group_{therm}_{sweeps}_{interval}_{lo // group_size}") if ck else None
                for (k, _), (e, c) in zip(chunk, _run_correlated(pkg, ctx, chunk, ck, gdir)):
                    est[k], corr[k] = e, c
    except Stopped as s:
        stopped = True
        if s.args:
            est.update(s.args[0])
    out = []
    for k, t in mine:
        if k not in est:
            continue
        e = est[k]
        rec = {"task": t}
        if k:
            rec["task_index"] = k  # omitted when zero, as the reference's serializer does
        rec.update(observables=_observables(e, corr.get(k)), acceptance=e["acceptance"],
                   measurements=int(e["measurements"]))
        out.append(rec)
    result = {"job_name": cfg.job_name, "rank": rank, "world_size": world_size, "tasks": out}
    summary = {"task_count": len(out), "elapsed_seconds": time.monotonic() - started, "stopped_early": stopped,
               "checkpoint_dir": ck.dir if ck else None,
               "measurement_bins": _TaskBins({k: est[k] for k, _ in mine if k in est})}
    return result, summary


def run_job(ctx, cfg: JobConfig, rank: int = 0, world_size: int = 1, epoch_sweeps: int = 100, tasks=None,
            group_size: int = 1024):
    """A rank's share of the job, run to the end; returns the ThetaJobResult record."""
    return run_job_checkpointed(ctx, cfg, rank, world_size, epoch_sweeps, tasks, group_size)[0]


def merge_results(results):
    """merge_theta_job_results (src/results.rs:246-273): one record of all
    ranks' tasks, sorted by task name, rank 0."""
    if not results:
        raise JobError("at least one rank result is required for merge")
    first = results[0]
    tasks = list(first["tasks"])
    for r in results[1:]:
        if r["job_name"] != first["job_name"]:
            raise JobError("cannot merge results from different jobs")
        if r["world_size"] != first["world_size"]:
            raise JobError("cannot merge results with different world sizes")
        tasks.extend(r["tasks"])
    tasks.sort(key=lambda t: t["task"]["name"])
    merged = []
    for i, t in enumerate(tasks):
        t = dict(t)
        if t.get("task_index", 0) == 0 and i:
            t["task_index"] = i
        merged.append(t)
    return {"job_name": first["job_name"], "rank": 0, "world_size": first["world_size"], "tasks": merged}


def result_path(cfg: JobConfig, rank: int, output_dir: Optional[str] = None) -> str:
    """`<dir>/<file name of job_name>.rank<r>.results.json`
    (rank_result_path_with_options, src/model.rs:948-959): the directory is
    the given one, else the job file's output_dir, else $XY_OUTPUT_DIR, else
    the job name's parent directory, else results/."""
    d = output_dir or cfg.output_dir or os.environ.get("XY_OUTPUT_DIR")
    if not d:
        d = os.path.dirname(cfg.job_name) or "results"
    return os.path.join(d, f"{os.path.basename(cfg.job_name) or cfg.job_name}.rank{rank}.results.json")


def measurement_dir(cfg: JobConfig, output_dir: Optional[str] = None) -> str:
    """`<dir>/<file name of job_name>.data` (default_measurement_dir_with_options,
    src/model.rs:970-980), the directory of the per-task .meas.h5 files."""
    return result_path(cfg, 0, output_dir).replace(".rank0.results.json", ".data")


def merged_path(cfg: JobConfig, output_dir: Optional[str] = None) -> str:
    """`<dir>/<file name of job_name>.results.json` (merged_result_path_with_options,
    src/model.rs:960-967)."""
    return result_path(cfg, 0, output_dir).replace(".rank0.results.json", ".results.json")


def checkpoint_dir(cfg: JobConfig, output_dir: Optional[str] = None) -> str:
    """`<dir>/<file name of job_name>.data/checkpoints`, beside the
    measurement directory of default_measurement_dir_with_options
    (src/model.rs:969-980)."""
    return result_path(cfg, 0, output_dir).replace(".rank0.results.json", ".data/checkpoints")


def status(cfg: JobConfig, world_size: int = 1, output_dir: Optional[str] = None) -> str:
    """theta_job_status_with_carlo (src/results.rs:377-395)."""
    completed = files = 0
    for rank in range(world_size):
        path = result_path(cfg, rank, output_dir)
        if os.path.exists(path):
            files += 1
            try:
                with open(path, encoding="utf-8") as f:
                    completed += len(json.load(f)["tasks"])
            except (OSError, ValueError, KeyError):
                pass
    return f"{completed} theta task(s) completed; {files} of {world_size} rank result file(s) present"


def write_result(result: dict, path: str) -> str:
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "w", encoding="utf-8") as f:
        json.dump(result, f, indent=2)
    return path


def main(argv=None):
    import argparse

    p = argparse.ArgumentParser(description="Run a theta job file (the reference's TOML schema) on the B200 path.")
    p.add_argument("job", help="TOML job file")
    p.add_argument("command", nargs="?", default="run", choices=("run", "merge", "status"))
    p.add_argument("--output-dir")
    p.add_argument("--rank", type=int, default=int(os.environ.get("RANK", 0)))
    p.add_argument("--world-size", type=int, default=int(os.environ.get("WORLD_SIZE", 1)))
    p.add_argument("--device", type=int, default=int(os.environ.get("LOCAL_RANK", 0)))
    p.add_argument("--epoch-sweeps", type=int, default=100)
    p.add_argument("--checkpoint-dir", help="checkpoint here (default with `checkpoint = true`: "
                                             "<output>/<job>.data/checkpoints)")
    p.add_argument("--restart", action="store_true", help="resume from the checkpoint directory")
    p.add_argument("--measurement-dir", help="per-task .meas.h5 files here (default <output>/<job>.data)")
    args = p.parse_args(argv)
    cfg = load_job(args.job)
    if args.command == "status":
        print(status(cfg, args.world_size, args.output_dir))
        return 0
    if args.command == "merge":
        paths = [result_path(cfg, r, args.output_dir) for r in range(args.world_size)]
        results = []
        for path in paths:
            with open(path, encoding="utf-8") as f:
                results.append(json.load(f))
        out = write_result(merge_results(results), merged_path(cfg, args.output_dir))
        print(f"merged {len(paths)} rank file(s) -> {out}")
        return 0
    pkg = _package()
    ck = None
    cdir = args.checkpoint_dir or (checkpoint_dir(cfg, args.output_dir) if cfg.checkpoint or args.restart else None)
    if cdir:
        ck = Checkpoints(os.path.join(cdir, f"rank{args.rank}"), args.restart, cfg.run_time_s, cfg.checkpoint_time_s)
    with pkg.Context(args.device) as ctx:
        res, summary = run_job_checkpointed(ctx, cfg, args.rank, args.world_size, args.epoch_sweeps, ck=ck)
    # finish_theta_job_run (src/results.rs:130-150): measurement files, then the result record
    meas_h5 = importlib.import_module(_package().__name__ + ".meas_h5")
    meas_h5.write_job_measurements(res["tasks"], summary["measurement_bins"],
                                   args.measurement_dir or measurement_dir(cfg, args.output_dir))
    path = write_result(res, result_path(cfg, args.rank, args.output_dir))
    note = "; stopped early: restart with --restart" if summary["stopped_early"] else ""
    print(f"{len(res['tasks'])} tasks -> {path} ({summary['elapsed_seconds']:.1f} s){note}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
