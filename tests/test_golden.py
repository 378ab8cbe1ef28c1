"""The oracle against the committed golden fixtures (no GPU).

tests/golden/keyed_trajectories.json holds whole trajectories of the
counter-keyed update path on small lattices (final FP32 angles, accepted
sites per sweep, Wolff cluster sizes, observables); the oracle must reproduce
them exactly, so any change to the keyed streams or to the update steps shows
here before a GPU run.  tests/golden/make_golden.py wrote them.
"""
import base64
import importlib.util
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def angles(case):
    return np.frombuffer(base64.b64decode(case["theta_f32_base64"]), dtype=np.float32)


def generator():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


CASES = load("keyed_trajectories.json")["cases"]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c["dims"])))
def test_oracle_reproduces_keyed_trajectory(orc, case):
    dims = tuple(case["dims"])
    jxy, jz = np.array(case["j_xy"]), np.array(case["j_z"])
    assert np.array_equal(jz, orc.uniform_disorder(dims[2], 0.5, 1.5, case["disorder_seed"]))
    got = generator().trajectory(dims, case["temperature"], case["proposal_width"], case["wolff_steps"],
                                 case["sweeps"], case["seed"], jxy, jz)
    assert got is not None, "the recorded seed has a tie-free trajectory"
    th, accepted, clusters = got
    assert np.array_equal(th.view(np.uint32), angles(case).view(np.uint32))
    assert accepted == case["accepted_per_sweep"] and clusters == case["cluster_sizes"]
    assert orc.measure_f32(dims, th, jxy.astype(np.float32), jz.astype(np.float32)) == case["observables"]


def test_published_vectors(orc):
    v = load("published_vectors.json")
    sm = v["splitmix64"]
    r = orc.FastRng(sm["seed"])
    assert [r.next_u64() for _ in sm["outputs"]] == sm["outputs"]
    for kat in v["philox4x32_10"]["vectors"]:
        assert orc.philox4x32_10(tuple(kat["ctr"]), tuple(kat["key"])) == tuple(kat["out"])
