"""The device against the committed golden fixtures (marked gpu).

Each trajectory of tests/golden/keyed_trajectories.json (chosen free of
FP32 tie-band decisions) is replayed from its seed through the single-task
entry points (one `slsf_task_sweep` per sweep) and through the batched
kernels, under the default kernel choice and under every other choice the
shape admits.  Final angles, accepted sites per sweep and Wolff cluster sites
must equal the fixture bit for bit; observables agree within the parity
tolerances (FP64 sums of FP32 terms in another order).
"""
import base64
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLDEN, "keyed_trajectories.json")) as _f:
    CASES = json.load(_f)["cases"]
IDS = ["x".join(map(str, c["dims"])) for c in CASES]


def angles(case):
    return np.frombuffer(base64.b64decode(case["theta_f32_base64"]), dtype=np.float32)


def make(slsf, ctx, case):
    t = slsf.Task(ctx, tuple(case["dims"]), np.array(case["j_xy"]), np.array(case["j_z"]), case["temperature"],
                  proposal_width=case["proposal_width"], wolff_steps=case["wolff_steps"], seed=case["seed"])
    t.init_random()
    return t


def cluster_sites_per_sweep(case):
    k = case["wolff_steps"]
    c = case["cluster_sizes"]
    return [sum(c[m * k:(m + 1) * k]) for m in range(case["sweeps"])]


@pytest.fixture(scope="module")
def ctx(slsf):
    slsf.build()
    c = slsf.Context()
    yield c
    c.close()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_single_task_path_reproduces_golden(slsf, ctx, case):
    t = make(slsf, ctx, case)
    accepted, sites = [], []
    for _ in range(case["sweeps"]):
        st = t.sweep(1)
        accepted.append(st["accepted"])
        sites.append(st["wolff_cluster_sites"])
    assert np.array_equal(t.theta.view(np.uint32), angles(case).view(np.uint32))
    assert accepted == case["accepted_per_sweep"]
    assert sites == cluster_sites_per_sweep(case)
    assert t.counters == (case["sweeps"], case["sweeps"] * case["wolff_steps"])
    got, ref, v = t.measure(), case["observables"], t.volume
    assert abs(got["energy"] - ref["energy"]) < 2e-5
    assert abs(got["magnetization_squared"] - ref["magnetization_squared"]) < 1e-5
    for k in ("cos_x", "cos_y", "cos_z", "sin_x", "sin_y", "sin_z"):
        assert abs(got[k] - ref[k]) < 2e-5 * v + 1e-5, k
    t.close()


CHOICES = [None, ("resident", 1, 128), ("resident", 1, 1024), ("cluster", 1, 512), ("cluster", 2, 512),
           ("cluster", 4, 1024)]


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_batched_kernels_reproduce_golden(slsf, case):
    dims = tuple(case["dims"])
    ran = 0
    for choice in CHOICES:
        with slsf.Context() as c:
            if choice is not None:
                try:
                    c.tune_set(dims, *choice)
                except slsf.SlsfError:
                    continue  # not a feasible choice for this shape
            t = make(slsf, c, case)
            [st] = c.batch_run([t], case["sweeps"])
            assert np.array_equal(t.theta.view(np.uint32), angles(case).view(np.uint32)), choice
            assert st["accepted"] == sum(case["accepted_per_sweep"]), choice
            assert st["wolff_cluster_sites"] == sum(case["cluster_sizes"]), choice
            t.close()
            ran += 1
    assert ran >= 2
