"""The C ABI from plain C (tests/c/abi_client.c): both headers compile as
C99 with -pedantic -Werror, the program links against the in-tree libraries
by name, and runs.  Without a GPU it must fail loudly (exit 3 with the
library's message); on a B200 (marked gpu) its result equals the Python
binding's for the same task."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def client(slsf, tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("gcc is not installed")
    slsf.build()
    slsf.load_host()
    libdir = os.path.dirname(slsf.LIB_PATH)
    exe = str(tmp_path_factory.mktemp("c") / "abi_client")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "abi_client.c"), "-o", exe, "-L", libdir, "-lslsf_host",
                    "-lslsf_b200", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def run(exe, *args):
    return subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=300)


def test_c_client_builds_and_fails_loudly_without_a_device(slsf, client):
    r = run(client, 8, 1.1, 7, 10)
    assert r.returncode in (0, 3), r.stderr
    assert r.stdout.startswith("version slsf-b200")
    assert f"run seed of task 1 at L=8: {slsf.task_seed(7, 8, 1, 1.1, 0.0, 0.0)}" in r.stdout
    if r.returncode == 3:
        assert "no CUDA device is available" in r.stderr


@pytest.mark.gpu
def test_c_client_equals_python_binding(slsf, client):
    r = run(client, 8, 1.1, 7, 10)
    assert r.returncode == 0, r.stderr
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("energy ")][0].split()
    energy, m2, accepted = float(line[1]), float(line[3]), int(line[5])
    L = 8
    with slsf.Context() as ctx:
        t = slsf.Task(ctx, (L, L, L), np.full(L, 1.2), 0.5 + np.arange(L) / L, 1.1, wolff_steps=1, seed=7)
        t.init_random()
        st = t.sweep(10)
        o = t.measure()
        t.close()
    assert (energy, m2, accepted) == (o["energy"], o["magnetization_squared"], st["accepted"])
