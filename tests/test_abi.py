"""The C-ABI library builds, loads and exports every symbol the header declares.

These run without a GPU: nothing here launches a kernel.
"""
import ctypes
import os

import pytest

from conftest import PKG_DIR, ROOT


def test_library_builds_and_loads(slsf):
    path = slsf.build()
    assert os.path.exists(path)
    slsf.load()
    assert slsf.load().slsf_version().decode().startswith("slsf-b200")


def test_every_declared_symbol_is_exported(slsf):
    slsf.build()
    declared = slsf.exported_symbols()
    assert len(declared) >= 24
    lib = ctypes.CDLL(slsf.LIB_PATH)
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, missing
    # and the Python binding covers every declared function
    assert sorted(slsf.SIGNATURES) == declared


def test_no_device_fails_loudly(slsf):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(slsf.SlsfError) as e:
        slsf.Context()
    assert e.value.code == slsf.ERR_CUDA
    assert "no CUDA device" in str(e.value)


def test_product_does_not_load_oracle():
    # The product sources never include, link, load or import the oracle.
    banned = ("oracle.h", "liboracle", "import oracle", "from oracle", "or_model", "or_keyed")
    for dirpath, _, files in os.walk(PKG_DIR):
        for f in files:
            if f.endswith((".cu", ".cuh", ".h", ".cpp", ".hpp", ".py")) or f == "Makefile":
                text = open(os.path.join(dirpath, f), encoding="utf-8").read()
                for b in banned:
                    assert b not in text, (f, b)


def test_task_bytes_counts_state(slsf):
    lib = slsf.load()
    b = lib.slsf_task_bytes(32, 32, 32, 0)
    assert b >= 32 ** 3 * 9  # theta (4 B) + bonds (1 B) + parent (4 B)
    assert lib.slsf_task_bytes(32, 32, 32, 64) - b >= 64 * 12 * 8
