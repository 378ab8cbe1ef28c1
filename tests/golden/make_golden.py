"""Writes the golden fixtures of this directory from the oracle.

keyed_trajectories.json: whole trajectories of the counter-keyed update path
(the one the device kernels take) on small lattices, chained from the
oracle's keyed steps in the device's order:

  angles  = INIT stream of the seed
  sweep m = Metropolis colour 0 then colour 1 (counter m), then wolff_steps
            Wolff steps (counters m * wolff_steps + k)

A case is kept only when no Metropolis decision and no Wolff bond of its
trajectory lies in the FP32 tie band (|u - p| below the device's error bound),
so the device, whose FP32 fast trig differs from the oracle's libm by less
than that band, must reproduce the final angles bit for bit.  When a seed's
trajectory has a tie, the next seed is tried; the seed kept is recorded.

published_vectors.json: Vigna's SplitMix64 vector and the Random123
philox4x32_10 known-answer vectors (the generators the oracle and the device
use), with their sources.

Run from the repository root:  python tests/golden/make_golden.py
"""
import base64
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402  (test infrastructure: the fixtures' checker)

EPS_METRO = 2e-4  # the tie bands of the device parity bars
EPS_WOLFF = 1e-4

# (dims, temperature, proposal width, wolff steps, sweeps, first seed, J_z disorder seed)
CASES = [
    ((4, 4, 4), 1.1, math.pi, 1, 6, 101, 11),
    ((6, 4, 8), 0.9, math.pi, 2, 5, 202, 12),
    ((8, 8, 8), 1.5, math.pi, 1, 4, 303, 13),
    ((10, 6, 4), 2.5, 1.0, 1, 4, 404, 14),
    ((12, 12, 12), 1.2, math.pi, 1, 3, 505, 15),
]


def encode_f32(a):
    return base64.b64encode(np.ascontiguousarray(a, np.float32).tobytes()).decode()


def trajectory(dims, temperature, width, wolff_steps, sweeps, seed, jxy, jz):
    """The keyed trajectory, or None when a decision lies in a tie band."""
    beta = np.float32(1.0 / temperature)
    jx32, jz32 = jxy.astype(np.float32), jz.astype(np.float32)
    th = oracle.keyed_init_angles(int(np.prod(dims)), seed)
    accepted, clusters = [], []
    for m in range(sweeps):
        acc = 0
        for colour in (0, 1):
            r = oracle.keyed_metro_half(dims, th, jx32, jz32, beta, np.float32(width), seed, m, colour, EPS_METRO)
            if r["tie"].any():
                return None
            th, acc = r["theta"], acc + int(r["accepted"])
        accepted.append(acc)
        for k in range(wolff_steps):
            r = oracle.keyed_wolff(dims, th, jx32, jz32, beta, seed, m * wolff_steps + k, 0, EPS_WOLFF)
            if ((r["bonds"] >> 3) & 7).any():
                return None
            th = r["theta"]
            clusters.append(int(r["size"]))
    return th, accepted, clusters


def keyed_trajectories():
    cases = []
    for dims, temperature, width, wolff_steps, sweeps, seed, dseed in CASES:
        jxy = np.full(dims[2], 1.2)
        jz = oracle.uniform_disorder(dims[2], 0.5, 1.5, dseed)
        for s in range(seed, seed + 64):
            got = trajectory(dims, temperature, width, wolff_steps, sweeps, s, jxy, jz)
            if got is not None:
                break
        else:
            raise RuntimeError(f"no tie-free seed for {dims}")
        th, accepted, clusters = got
        obs = oracle.measure_f32(dims, th, jxy.astype(np.float32), jz.astype(np.float32))
        cases.append({
            "dims": list(dims), "temperature": temperature, "proposal_width": width, "wolff_steps": wolff_steps,
            "sweeps": sweeps, "seed": s, "disorder_seed": dseed, "j_xy": jxy.tolist(), "j_z": jz.tolist(),
            "accepted_per_sweep": accepted, "cluster_sizes": clusters,
            "theta_f32_base64": encode_f32(th), "observables": obs,
        })
    return {"generator": "tests/golden/make_golden.py", "eps_metro": EPS_METRO, "eps_wolff": EPS_WOLFF,
            "cases": cases}


def published_vectors():
    return {
        "splitmix64": {
            "source": "S. Vigna, splitmix64.c, first outputs for seed 1234567",
            "seed": 1234567,
            "outputs": [6457827717110365317, 3203168211198807973, 9817491932198370423, 4593380528125082431,
                        16408922859458223821],
        },
        "philox4x32_10": {
            "source": "Random123 known-answer vectors (kat_vectors, philox4x32_10)",
            "vectors": [
                {"ctr": [0, 0, 0, 0], "key": [0, 0], "out": [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]},
                {"ctr": [0xFFFFFFFF] * 4, "key": [0xFFFFFFFF] * 2,
                 "out": [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]},
                {"ctr": [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], "key": [0xA4093822, 0x299F31D0],
                 "out": [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]},
            ],
        },
    }


def main():
    oracle.lib()
    with open(os.path.join(HERE, "keyed_trajectories.json"), "w") as f:
        json.dump(keyed_trajectories(), f, indent=1)
        f.write("\n")
    with open(os.path.join(HERE, "published_vectors.json"), "w") as f:
        json.dump(published_vectors(), f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
