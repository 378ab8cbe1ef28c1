"""The .meas.h5 writer (slsf_rs_b200.meas_h5, write_theta_task_measurements
of src/results.rs:38-105) read back by a reader written from the HDF5 file
format specification (tests/h5read.py); the reader is first checked on a file
that libhdf5 wrote (no HDF5 library exists in this image)."""
import importlib
import importlib.util
import os

import numpy as np
import pytest

import h5read


def libhdf5_file():
    spec = importlib.util.find_spec("scipy")
    if spec is None or not spec.origin:
        return None
    path = os.path.join(os.path.dirname(spec.origin), "io", "matlab", "tests", "data", "testhdf5_7.4_GLNX86.mat")
    return path if os.path.exists(path) else None


def test_reader_on_a_libhdf5_file():
    # a MATLAB 7.3 file: an HDF5 file behind a 512-byte user block, holding
    # testdouble = 0:pi/4:2*pi with the attribute MATLAB_class = "double"
    path = libhdf5_file()
    if path is None:
        pytest.skip("scipy's libhdf5-written test file is not installed")
    r = h5read.read(path)
    assert sorted(r) == ["/", "/testdouble"]
    d = r["/testdouble"]
    assert d.shape == (9, 1) and d.layout == "contiguous" and d.dtype == np.dtype("<f8")
    assert np.allclose(d.value.ravel(), np.arange(9) * np.pi / 4, rtol=0, atol=1e-15)
    assert d.attrs == {"MATLAB_class": "double"}


@pytest.fixture(scope="module")
def meas(slsf):
    return importlib.import_module("slsf_rs_b200.meas_h5")


def sample_bins(slsf, n_corr_z=4):
    rng = np.random.default_rng(7)
    bins = {name: (5, rng.standard_normal(8)) for name in slsf.BIN_NAMES}
    for z in range(n_corr_z):
        bins[f"CorrXY_z{z}_r1"] = (3, rng.standard_normal(2))
    bins["CorrZ_r2"] = (1, np.array([0.25]))
    return bins


def check(r, bins):
    assert sorted(k for k in r if k.count("/") == 2 and k.startswith("/observables/")) == \
        sorted(f"/observables/{n}" for n in bins)
    for name, (bin_len, samples) in bins.items():
        bl, sm = r[f"/observables/{name}/bin_length"], r[f"/observables/{name}/samples"]
        assert bl.shape == () and bl.dtype == np.dtype("<i8") and int(bl.value) == bin_len, name
        assert sm.shape == (len(samples),) and sm.dtype == np.dtype("<f8"), name
        assert np.array_equal(sm.value.view(np.uint64), np.asarray(samples, np.float64).view(np.uint64)), name


def test_round_trip(slsf, meas, tmp_path, monkeypatch):
    monkeypatch.delenv("XY_CARLO_VERSION", raising=False)
    monkeypatch.setenv("XY_MC_VERSION", "9.8.7")
    bins = sample_bins(slsf)
    path = meas.write_meas_h5(tmp_path / "task0001" / "run0001.meas.h5", bins)
    assert not os.path.exists(path + ".tmp")
    r = h5read.read(path)
    check(r, bins)
    assert r["/version/carlo_version"].value == "0.3.4"
    assert r["/version/mc_package"].value == "SLSF.XYCarlo"
    assert r["/version/mc_version"].value == "9.8.7"
    assert r["/version/mc_package"].dtype == ("string", len("SLSF.XYCarlo"), 0, 0)
    data = open(path, "rb").read()
    f = h5read._File(data)
    assert (f.base, f.leaf_k, f.internal_k, f.eof) == (0, 4, 16, len(data))


@pytest.mark.parametrize("n_corr_z", [700, 8460])
def test_large_groups_take_more_btree_levels(slsf, meas, tmp_path, n_corr_z):
    # L = 64 with r_max = 32 measures over 2000 correlation observables (two
    # B-tree levels), L = 128 with r_max = 64 over 8400 (three)
    bins = sample_bins(slsf, n_corr_z=n_corr_z)
    path = meas.write_meas_h5(tmp_path / "big.meas.h5", bins)
    check(h5read.read(path), bins)


def test_reference_errors(slsf, meas, tmp_path):
    with pytest.raises(meas.MeasH5Error, match="^theta task result does not contain measurement bins$"):
        meas.write_meas_h5(tmp_path / "a.h5", {})
    with pytest.raises(meas.MeasH5Error, match="^Energy: internal bin length must be positive$"):
        meas.write_meas_h5(tmp_path / "a.h5", {"Energy": (0, [1.0])})
    with pytest.raises(meas.MeasH5Error, match="^Energy: no complete measurement bins to write$"):
        meas.write_meas_h5(tmp_path / "a.h5", {"Energy": (2, [])})
    rec = {"observables": {"Energy": {"mean": 0.0, "error": 0.0}}}
    with pytest.raises(meas.MeasH5Error, match="^missing observable estimate for CorrZ_r1$"):
        meas.write_job_measurements([rec], {0: {"Energy": (1, [1.0]), "CorrZ_r1": (1, [1.0])}}, tmp_path)
    with pytest.raises(meas.MeasH5Error, match="^theta task result does not contain measurement bins$"):
        meas.write_job_measurements([rec], {}, tmp_path)


def test_job_measurement_paths(meas, tmp_path):
    # task<index + 1>/run0001.meas.h5 (src/results.rs:38-53); index 0 has no task_index key
    obs = {"Energy": {"mean": 0.0, "error": 0.0}}
    recs = [{"observables": obs}, {"task_index": 2, "observables": obs}]
    bins = {0: {"Energy": (1, [1.0, 2.0])}, 2: {"Energy": (1, [3.0])}}
    paths = meas.write_job_measurements(recs, bins, tmp_path / "job.data")
    assert paths == [str(tmp_path / "job.data" / "task0001" / "run0001.meas.h5"),
                     str(tmp_path / "job.data" / "task0003" / "run0001.meas.h5")]
    assert list(h5read.read(paths[1])["/observables/Energy/samples"].value) == [3.0]
