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


RUST_SIZES = {"u8": 1, "u32": 4, "i32": 4, "f32": 4, "u64": 8, "f64": 8, "usize": 8, "*const f64": 8}
RUST_STRUCTS = {"SlsfTaskDesc": "slsf_task_desc", "SlsfObservables": "slsf_observables",
                "SlsfSweepStats": "slsf_sweep_stats", "SlsfKernelChoice": "slsf_kernel_choice"}


def c_layouts(tmp_path):
    exe = str(tmp_path / "abi_layout")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "abi_layout.c"), "-o", exe], check=True)
    out = {}
    for line in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.splitlines():
        name, size, *fields = line.split()
        out[name] = (int(size), [(f.split(":")[0], int(f.split(":")[1])) for f in fields])
    return out


def rust_layouts():
    """#[repr(C)] layouts of the Rust binding's structs in INTEGRATION.md (C rules: each field at its
    natural alignment, the size rounded up to the largest alignment)."""
    import re

    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    out = {}
    for m in re.finditer(r"pub struct (\w+) \{\n(.*?)\n\}", text, re.S):
        name, body = m.group(1), m.group(2)
        if name not in RUST_STRUCTS:
            continue
        off, align, fields = 0, 1, []
        for f, ty in re.findall(r"pub (\w+): ([^,\n]+)", body):
            size = RUST_SIZES[ty.strip()]
            off = (off + size - 1) // size * size
            fields.append((f, off))
            off += size
            align = max(align, size)
        out[RUST_STRUCTS[name]] = ((off + align - 1) // align * align, fields)
    return out


def test_abi_struct_layouts_agree(slsf, tmp_path):
    # The C compiler's layout of every struct of include/slsf_gpu.h equals the
    # ctypes structs of the Python binding and the Rust binding of INTEGRATION.md.
    import ctypes

    if shutil.which("gcc") is None:
        pytest.skip("gcc is not installed")
    c = c_layouts(tmp_path)
    py = {"slsf_task_desc": slsf.TaskDesc, "slsf_observables": slsf.Observables, "slsf_sweep_stats": slsf.SweepStats,
          "slsf_kernel_choice": slsf.KernelChoice}
    for name, cls in py.items():
        size, fields = c[name]
        assert ctypes.sizeof(cls) == size, name
        assert [(f, getattr(cls, f).offset) for f, _ in cls._fields_] == fields, name
    rust = rust_layouts()
    assert set(rust) == set(py)
    for name, layout in rust.items():
        assert layout == c[name], (name, layout, c[name])
