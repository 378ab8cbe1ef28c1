"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle restates SLSF-rs's update-and-measure path in FP64 C++ (see
oracle/oracle.h for the reference lines each function follows).  It is the
checker for the CUDA library and the benchmark's CPU baseline; the product
library never loads it.  `build()` compiles it with the Makefile beside this
file into oracle/_build/liboracle.so.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

OBS_FIELDS = ("energy", "magnetization_squared", "cos_x", "cos_y", "cos_z", "sin_x", "sin_y", "sin_z")
SERIES_COLS = 12  # Energy, EnergySquared, MagnetizationSquared, cos xyz, sin xyz, sin2 xyz
DERIVED = ("Magnetization", "Chi", "SpecificHeat", "RhoXY", "RhoZ")


class Rng(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("state", C.c_uint64), ("draws", C.c_uint64)]


class Obs(C.Structure):
    _fields_ = [(n, C.c_double) for n in OBS_FIELDS]

    def as_dict(self):
        return {n: getattr(self, n) for n in OBS_FIELDS}


class SimOptions(C.Structure):
    _fields_ = [
        ("thermal_sweeps", C.c_size_t),
        ("measure_sweeps", C.c_size_t),
        ("measure_interval", C.c_size_t),
        ("proposal_width", C.c_double),
        ("wolff_steps", C.c_size_t),
        ("correlation_interval", C.c_size_t),
        ("correlation_rmax", C.c_long),
        ("correlation_rmax_xy", C.c_long),
        ("correlation_rmax_z", C.c_long),
        ("init_cold", C.c_int),
    ]


class SimResult(C.Structure):
    _fields_ = [
        ("energy", C.c_double),
        ("rho_sx", C.c_double),
        ("rho_sy", C.c_double),
        ("rho_sz", C.c_double),
        ("std_rho_sx", C.c_double),
        ("std_rho_sy", C.c_double),
        ("std_rho_sz", C.c_double),
        ("magnetization_squared", C.c_double),
        ("chi", C.c_double),
        ("acceptance", C.c_double),
        ("num_measurements", C.c_size_t),
        ("num_correlation_measurements", C.c_size_t),
        ("n_corr_xy", C.c_size_t),
        ("n_corr_z", C.c_size_t),
    ]


class OracleError(RuntimeError):
    pass


def build(force: bool = False) -> str:
    if force or not all(os.path.exists(os.path.join(HERE, "_build", n))
                        for n in ("liboracle.so", "libbaseline_v4.so", "libbaseline_v3.so")):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_U8 = C.POINTER(C.c_uint8)
_I8 = C.POINTER(C.c_int8)
_U32 = C.POINTER(C.c_uint32)
_U64 = C.POINTER(C.c_uint64)
_SZ = C.c_size_t


def lib():
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = C.CDLL(LIB_PATH)
    sig = {
        "or_rng_seed": (None, [C.POINTER(Rng), C.c_uint64]),
        "or_rng_set_position": (None, [C.POINTER(Rng), C.c_uint64]),
        "or_rng_next_u64": (C.c_uint64, [C.POINTER(Rng)]),
        "or_rng_f64": (C.c_double, [C.POINTER(Rng)]),
        "or_rng_bool": (C.c_int, [C.POINTER(Rng)]),
        "or_rng_range": (C.c_uint64, [C.POINTER(Rng), C.c_uint64]),
        "or_last_error": (C.c_char_p, []),
        "or_wrap_angle": (C.c_double, [C.c_double]),
        "or_wolff_add_probability": (C.c_double, [C.c_double] * 4),
        "or_wolff_reflect_angle": (C.c_double, [C.c_double, C.c_double]),
        "or_validate_temperature": (C.c_int, [C.c_double]),
        "or_validate_proposal_width": (C.c_int, [C.c_double]),
        "or_two_point_disorder": (C.c_int, [_D, _SZ, C.c_double, C.c_double, C.POINTER(Rng), C.c_char_p]),
        "or_uniform_disorder": (None, [_D, _SZ, C.c_double, C.c_double, C.c_uint64]),
        "or_init_angles": (None, [_D, _SZ, C.c_int, C.POINTER(Rng)]),
        "or_measure_energy": (C.c_double, [_SZ, _SZ, _SZ, _D, _D, _D]),
        "or_magnetization_squared": (C.c_double, [_SZ, _D]),
        "or_helicity_sums": (None, [_SZ, _SZ, _SZ, _D, _D, _D, _D]),
        "or_helicity_modulus": (C.c_int, [_SZ, _SZ, _SZ, _D, _D, _D, C.c_double, _D]),
        "or_measure_observables": (None, [_SZ, _SZ, _SZ, _D, _D, _D, C.POINTER(Obs)]),
        "or_measure_correlations": (None, [_SZ, _SZ, _SZ, _D, C.c_long, C.c_long, C.c_long, _D, _D, _D, _D, _D, C.POINTER(_SZ)]),
        "or_model_new": (C.c_int, [_SZ, _SZ, _SZ, _D, _SZ, _D, _SZ, C.c_double, C.c_double, _SZ, C.c_uint64, C.POINTER(C.c_void_p)]),
        "or_model_free": (None, [C.c_void_p]),
        "or_model_init": (None, [C.c_void_p, C.c_int]),
        "or_model_set_theta": (None, [C.c_void_p, _D]),
        "or_model_get_theta": (None, [C.c_void_p, _D]),
        "or_model_rng_position": (C.c_uint64, [C.c_void_p]),
        "or_model_metropolis_sweep": (C.c_int, [C.c_void_p, C.c_int, _D]),
        "or_model_local_metropolis_step": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_int)]),
        "or_model_wolff_step": (C.c_int, [C.c_void_p, C.POINTER(_SZ)]),
        "or_model_sweep": (C.c_int, [C.c_void_p, C.c_int]),
        "or_model_measure": (None, [C.c_void_p, C.POINTER(Obs)]),
        "or_model_run_series": (C.c_int, [C.c_void_p, _SZ, _SZ, C.c_int, _D, _D]),
        "or_blocking_stderr": (C.c_double, [_D, _SZ]),
        "or_run_theta_simulation": (C.c_int, [_SZ, _SZ, _SZ, _D, _D, _D, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.POINTER(SimOptions), C.POINTER(Rng), C.POINTER(SimResult), _D, _D, _D, _D, _D]),
        "or_binned_estimate": (C.c_int, [_D, _SZ, _SZ, _D, _D, _D, C.POINTER(_SZ)]),
        "or_evaluate_derived": (C.c_int, [_D, _SZ, C.c_double, C.c_double, _D]),
        "or_philox4x32_10": (None, [_U32, _U32, _U32]),
        "or_keyed_init_angles": (None, [_SZ, C.c_uint64, _F]),
        "or_keyed_metro_half": (_SZ, [_SZ, _SZ, _SZ, _F, _F, _F, C.c_float, C.c_float, C.c_uint64, C.c_uint64, C.c_int,
                                      C.c_double, _F, _I8, _U8, _D]),
        "or_keyed_wolff_pick": (None, [_SZ, _SZ, _SZ, C.c_uint64, C.c_uint64, C.c_uint32, _F, _U32]),
        "or_keyed_wolff": (_SZ, [_SZ, _SZ, _SZ, _F, _F, _F, C.c_float, C.c_uint64, C.c_uint64, C.c_uint32, C.c_double,
                                 _U8, _U8, _F]),
        "or_cluster_from_bonds": (_SZ, [_SZ, _SZ, _SZ, _U8, _SZ, _U8]),
        "or_measure_f32": (None, [_SZ, _SZ, _SZ, _F, _F, _F, C.POINTER(Obs)]),
        "or_correlations_f32": (None, [_SZ, _SZ, _SZ, _F, _SZ, _SZ, _D, _D, _D, _D]),
        "or_bench_tasks": (C.c_int, [_SZ, _SZ, _SZ, _SZ, _D, _D, _D, C.c_double, _SZ, _U64, _SZ, C.c_int, _D, _D]),
        "or_series_tasks": (C.c_int, [_SZ, _SZ, _SZ, _SZ, _D, _D, _D, C.c_double, _SZ, _U64, _SZ, _SZ, _SZ, C.c_int,
                                      _D]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return lib().or_last_error().decode("utf-8")


def _check(code):
    if code != 0:
        raise OracleError(last_error())


def ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def dptr(a):
    return ptr(a, C.c_double)


def fptr(a):
    return ptr(a, C.c_float)


# ---------------------------------------------------------------- FastRng
class FastRng:
    """SplitMix64 stream with rand-style sampling (src/types.rs:9-82)."""

    def __init__(self, seed: int):
        self.s = Rng()
        lib().or_rng_seed(C.byref(self.s), C.c_uint64(seed))

    def next_u64(self):
        return lib().or_rng_next_u64(C.byref(self.s))

    def f64(self):
        return lib().or_rng_f64(C.byref(self.s))

    def bool(self):
        return bool(lib().or_rng_bool(C.byref(self.s)))

    def range(self, n):
        return lib().or_rng_range(C.byref(self.s), n)

    def set_position(self, pos):
        lib().or_rng_set_position(C.byref(self.s), pos)

    @property
    def draws(self):
        return self.s.draws


# ---------------------------------------------------------------- model
class Model:
    """ThetaModel restated (src/model.rs:254-442) with explicit J arrays."""

    def __init__(self, lx, ly, lz, j_xy, j_z, temperature, proposal_width=np.pi, wolff_steps=1, seed=0):
        self.dims = (lx, ly, lz)
        jx = np.ascontiguousarray(j_xy, dtype=np.float64)
        jz = np.ascontiguousarray(j_z, dtype=np.float64)
        h = C.c_void_p()
        _check(lib().or_model_new(lx, ly, lz, dptr(jx), jx.size, dptr(jz), jz.size, temperature, proposal_width,
                                  wolff_steps, C.c_uint64(seed), C.byref(h)))
        self.h = h
        self.volume = lx * ly * lz

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_model_free(self.h)
            self.h = None

    def init(self, cold=False):
        lib().or_model_init(self.h, int(cold))

    @property
    def theta(self):
        out = np.empty(self.volume, dtype=np.float64)
        lib().or_model_get_theta(self.h, dptr(out))
        return out

    @theta.setter
    def theta(self, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        assert v.size == self.volume
        lib().or_model_set_theta(self.h, dptr(v))

    def metropolis_sweep(self, batch8=True):
        acc = C.c_double()
        _check(lib().or_model_metropolis_sweep(self.h, int(batch8), C.byref(acc)))
        return acc.value

    def local_metropolis_step(self, width):
        acc = C.c_int()
        _check(lib().or_model_local_metropolis_step(self.h, width, C.byref(acc)))
        return bool(acc.value)

    def wolff_step(self):
        size = C.c_size_t()
        _check(lib().or_model_wolff_step(self.h, C.byref(size)))
        return size.value

    def sweep(self, batch8=True):
        _check(lib().or_model_sweep(self.h, int(batch8)))

    def measure(self):
        o = Obs()
        lib().or_model_measure(self.h, C.byref(o))
        return o.as_dict()

    def run_series(self, thermalization, sweeps, batch8=True):
        series = np.zeros((sweeps, SERIES_COLS), dtype=np.float64)
        acc = C.c_double()
        _check(lib().or_model_run_series(self.h, thermalization, sweeps, int(batch8), dptr(series), C.byref(acc)))
        return series, acc.value


# ---------------------------------------------------------------- stateless helpers
def measure_observables(dims, theta, jxy, jz):
    lx, ly, lz = dims
    o = Obs()
    t = np.ascontiguousarray(theta, np.float64)
    a = np.ascontiguousarray(jxy, np.float64)
    b = np.ascontiguousarray(jz, np.float64)
    lib().or_measure_observables(lx, ly, lz, dptr(t), dptr(a), dptr(b), C.byref(o))
    return o.as_dict()


def measure_energy(dims, theta, jxy, jz):
    lx, ly, lz = dims
    t = np.ascontiguousarray(theta, np.float64)
    a = np.ascontiguousarray(jxy, np.float64)
    b = np.ascontiguousarray(jz, np.float64)
    return lib().or_measure_energy(lx, ly, lz, dptr(t), dptr(a), dptr(b))


def helicity_sums(dims, theta, jxy, jz):
    lx, ly, lz = dims
    out = np.zeros(6)
    t = np.ascontiguousarray(theta, np.float64)
    a = np.ascontiguousarray(jxy, np.float64)
    b = np.ascontiguousarray(jz, np.float64)
    lib().or_helicity_sums(lx, ly, lz, dptr(t), dptr(a), dptr(b), dptr(out))
    return out


def helicity_modulus(dims, theta, jxy, jz, temperature):
    lx, ly, lz = dims
    out = np.zeros(3)
    t = np.ascontiguousarray(theta, np.float64)
    a = np.ascontiguousarray(jxy, np.float64)
    b = np.ascontiguousarray(jz, np.float64)
    _check(lib().or_helicity_modulus(lx, ly, lz, dptr(t), dptr(a), dptr(b), temperature, dptr(out)))
    return out


def magnetization_squared(theta):
    t = np.ascontiguousarray(theta, np.float64)
    return lib().or_magnetization_squared(t.size, dptr(t))


def measure_correlations(dims, theta, rmax=None, rmax_xy=None, rmax_z=None):
    lx, ly, lz = dims
    t = np.ascontiguousarray(theta, np.float64)
    n = max(lx, ly, lz) + 1
    cx, cy, cxy, cz = (np.zeros(n) for _ in range(4))
    cbz = np.zeros(lz * n)
    eff = (C.c_size_t * 2)()
    conv = lambda v: -1 if v is None else int(v)
    lib().or_measure_correlations(lx, ly, lz, dptr(t), conv(rmax), conv(rmax_xy), conv(rmax_z), dptr(cx), dptr(cy),
                                  dptr(cxy), dptr(cbz), dptr(cz), eff)
    rxy, rz = eff[0], eff[1]
    return {
        "r_xy": list(range(1, rxy + 1)),
        "r_z": list(range(1, rz + 1)),
        "corr_x": cx[:rxy].copy(),
        "corr_y": cy[:rxy].copy(),
        "corr_xy": cxy[:rxy].copy(),
        "corr_xy_by_z": cbz[: lz * rxy].reshape(lz, rxy).copy(),
        "corr_z": cz[:rz].copy(),
    }


def two_point_disorder(n, mean, delta, rng: FastRng, name="J_z"):
    out = np.zeros(n)
    _check(lib().or_two_point_disorder(dptr(out), n, mean, delta, C.byref(rng.s), name.encode()))
    return out


def uniform_disorder(n, lo, hi, seed):
    out = np.zeros(n)
    lib().or_uniform_disorder(dptr(out), n, lo, hi, C.c_uint64(seed))
    return out


def init_angles(n, rng: FastRng, cold=False):
    out = np.zeros(n)
    lib().or_init_angles(dptr(out), n, int(cold), C.byref(rng.s))
    return out


def run_theta_simulation(dims, j_xy, j_z_mean, delta_j_z, temperature, rng: FastRng, **opts):
    """run_theta_simulation (src/simulation.rs:13-195); defaults of ThetaSimulationOptions (types.rs:292-307)."""
    lx, ly, lz = dims
    o = SimOptions(
        thermal_sweeps=opts.get("thermal_sweeps", 1000),
        measure_sweeps=opts.get("measure_sweeps", 5000),
        measure_interval=opts.get("measure_interval", 10),
        proposal_width=opts.get("proposal_width", np.pi),
        wolff_steps=opts.get("wolff_steps", 1),
        correlation_interval=opts.get("correlation_interval", 1),
        correlation_rmax=-1 if opts.get("correlation_rmax") is None else opts["correlation_rmax"],
        correlation_rmax_xy=-1 if opts.get("correlation_rmax_xy") is None else opts["correlation_rmax_xy"],
        correlation_rmax_z=-1 if opts.get("correlation_rmax_z") is None else opts["correlation_rmax_z"],
        init_cold=int(opts.get("init_cold", False)),
    )
    theta = np.zeros(lx * ly * lz)
    jxy = np.zeros(lz)
    jz = np.zeros(lz)
    n = max(lx, ly, lz) + 1
    cx, cy, cxy, cz = (np.zeros(n) for _ in range(4))
    cbz = np.zeros(lz * n)
    res = SimResult()
    _check(lib().or_run_theta_simulation(lx, ly, lz, dptr(theta), dptr(jxy), dptr(jz), j_xy, j_z_mean, delta_j_z,
                                         temperature, C.byref(o), C.byref(rng.s), C.byref(res), dptr(cx), dptr(cy),
                                         dptr(cxy), dptr(cbz), dptr(cz)))
    out = {f[0]: getattr(res, f[0]) for f in SimResult._fields_}
    rxy, rz = res.n_corr_xy, res.n_corr_z
    out.update(corr_x=cx[:rxy].copy(), corr_y=cy[:rxy].copy(), corr_xy=cxy[:rxy].copy(),
               corr_xy_by_z=cbz[: lz * rxy].reshape(lz, rxy).copy(), corr_z=cz[:rz].copy(), theta=theta, jxy=jxy,
               jz=jz)
    return out


def blocking_stderr(x):
    a = np.ascontiguousarray(x, np.float64)
    return lib().or_blocking_stderr(dptr(a), a.size)


def binned_estimate(samples, binsize):
    a = np.ascontiguousarray(samples, np.float64)
    bins = np.zeros(max(1, a.size))
    mean, err, nb = C.c_double(), C.c_double(), C.c_size_t()
    _check(lib().or_binned_estimate(dptr(a), a.size, binsize, C.byref(mean), C.byref(err), dptr(bins), C.byref(nb)))
    return {"mean": mean.value, "stderr": err.value, "bins": bins[: nb.value].copy()}


def evaluate_derived(bin_means, volume, beta):
    bm = np.ascontiguousarray(bin_means, np.float64)
    assert bm.ndim == 2 and bm.shape[1] == SERIES_COLS
    out = np.zeros((5, 2))
    _check(lib().or_evaluate_derived(dptr(bm), bm.shape[0], volume, beta, dptr(out)))
    return {name: (out[i, 0], out[i, 1]) for i, name in enumerate(DERIVED)}


# ---------------------------------------------------------------- counter-based forms
def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    out = (C.c_uint32 * 4)()
    lib().or_philox4x32_10(c, k, out)
    return tuple(out)


def keyed_init_angles(n, seed):
    out = np.zeros(n, dtype=np.float32)
    lib().or_keyed_init_angles(n, C.c_uint64(seed), fptr(out))
    return out


def keyed_metro_half(dims, theta, jxy, jz, beta, width, seed, sweep, color, eps_tie):
    lx, ly, lz = dims
    th = np.ascontiguousarray(theta, np.float32)
    a = np.ascontiguousarray(jxy, np.float32)
    b = np.ascontiguousarray(jz, np.float32)
    out = np.empty_like(th)
    dec = np.zeros(th.size, dtype=np.int8)
    tie = np.zeros(th.size, dtype=np.uint8)
    prob = np.zeros(th.size, dtype=np.float64)
    n = lib().or_keyed_metro_half(lx, ly, lz, fptr(th), fptr(a), fptr(b), C.c_float(beta), C.c_float(width),
                                  C.c_uint64(seed), C.c_uint64(sweep), color, eps_tie, fptr(out), ptr(dec, C.c_int8),
                                  ptr(tie, C.c_uint8), dptr(prob))
    return {"theta": out, "decision": dec, "tie": tie, "prob": prob, "accepted": n}


def keyed_wolff_pick(dims, seed, sweep, step):
    lx, ly, lz = dims
    phi = C.c_float()
    site = (C.c_uint32 * 3)()
    lib().or_keyed_wolff_pick(lx, ly, lz, C.c_uint64(seed), C.c_uint64(sweep), step, C.byref(phi), site)
    return phi.value, (site[0], site[1], site[2])


def keyed_wolff(dims, theta, jxy, jz, beta, seed, sweep, step, eps_tie):
    lx, ly, lz = dims
    th = np.ascontiguousarray(theta, np.float32)
    a = np.ascontiguousarray(jxy, np.float32)
    b = np.ascontiguousarray(jz, np.float32)
    bonds = np.zeros(th.size, dtype=np.uint8)
    cluster = np.zeros(th.size, dtype=np.uint8)
    out = np.empty_like(th)
    size = lib().or_keyed_wolff(lx, ly, lz, fptr(th), fptr(a), fptr(b), C.c_float(beta), C.c_uint64(seed),
                                C.c_uint64(sweep), step, eps_tie, ptr(bonds, C.c_uint8), ptr(cluster, C.c_uint8),
                                fptr(out))
    return {"bonds": bonds, "cluster": cluster, "theta": out, "size": size}


def cluster_from_bonds(dims, bonds, seed_idx):
    lx, ly, lz = dims
    b = np.ascontiguousarray(bonds, np.uint8)
    cl = np.zeros(b.size, dtype=np.uint8)
    size = lib().or_cluster_from_bonds(lx, ly, lz, ptr(b, C.c_uint8), seed_idx, ptr(cl, C.c_uint8))
    return cl, size


def measure_f32(dims, theta, jxy, jz):
    lx, ly, lz = dims
    th = np.ascontiguousarray(theta, np.float32)
    a = np.ascontiguousarray(jxy, np.float32)
    b = np.ascontiguousarray(jz, np.float32)
    o = Obs()
    lib().or_measure_f32(lx, ly, lz, fptr(th), fptr(a), fptr(b), C.byref(o))
    return o.as_dict()


def correlations_f32(dims, theta, rmax_xy, rmax_z):
    lx, ly, lz = dims
    th = np.ascontiguousarray(theta, np.float32)
    cx, cy, cz = np.zeros(max(rmax_xy, 1)), np.zeros(max(rmax_xy, 1)), np.zeros(max(rmax_z, 1))
    cbz = np.zeros(max(lz * rmax_xy, 1))
    lib().or_correlations_f32(lx, ly, lz, fptr(th), rmax_xy, rmax_z, dptr(cx), dptr(cy), dptr(cbz), dptr(cz))
    return {"corr_x": cx[:rmax_xy], "corr_y": cy[:rmax_xy], "corr_xy_by_z": cbz[: lz * rmax_xy].reshape(lz, rmax_xy),
            "corr_z": cz[:rmax_z]}


def host_cpu():
    """The host CPU: model name, logical CPUs, physical cores and AVX-512F support (/proc/cpuinfo)."""
    model, flags, cores = "unknown", set(), set()
    phys = core = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                key, _, val = line.partition(":")
                key, val = key.strip(), val.strip()
                if key == "model name":
                    model = val
                elif key == "flags" and not flags:
                    flags = set(val.split())
                elif key == "physical id":
                    phys = val
                elif key == "core id":
                    core = val
                elif not key and phys is not None:
                    cores.add((phys, core))
                    phys = core = None
        if phys is not None:
            cores.add((phys, core))
    except OSError:
        pass
    logical = os.cpu_count() or 1
    return {"model": model, "logical_cpus": logical, "physical_cores": len(cores) or logical,
            "avx512f": "avx512f" in flags}


_baseline = None


def baseline_lib():
    """The timed CPU baseline (baseline_simd.cpp): the AVX-512 build on hosts with AVX-512F, else the AVX2 build."""
    global _baseline
    if _baseline is not None:
        return _baseline
    build()
    name = "libbaseline_v4.so" if host_cpu()["avx512f"] else "libbaseline_v3.so"
    L = C.CDLL(os.path.join(HERE, "_build", name))
    L.or_bench_tasks.restype = C.c_int
    L.or_bench_tasks.argtypes = [_SZ, _SZ, _SZ, _SZ, _D, _D, _D, C.c_double, _SZ, _U64, _SZ, C.c_int, _D, _D]
    L.or_series_tasks.restype = C.c_int
    L.or_series_tasks.argtypes = [_SZ, _SZ, _SZ, _SZ, _D, _D, _D, C.c_double, _SZ, _U64, _SZ, _SZ, _SZ, C.c_int, _D]
    L.or_last_error.restype = C.c_char_p
    L.or_last_error.argtypes = []
    L.name = name
    _baseline = L
    return L


def _check_lib(L, code):
    if code != 0:
        raise OracleError(L.or_last_error().decode("utf-8"))


def bench_tasks(dims, jxy, jz, temperatures, width, wolff_steps, seeds, sweeps, threads, simd=False):
    """Time independent tasks on `threads` host threads (the CPU baseline).  simd=True runs the
    SIMD build (the reference's vectorised Metropolis batches), else the scalar oracle."""
    lx, ly, lz = dims
    n = len(temperatures)
    a = np.ascontiguousarray(jxy, np.float64).reshape(n, lz)
    b = np.ascontiguousarray(jz, np.float64).reshape(n, lz)
    t = np.ascontiguousarray(temperatures, np.float64)
    s = np.ascontiguousarray(seeds, np.uint64)
    sec, chk = C.c_double(), C.c_double()
    L = baseline_lib() if simd else lib()
    _check_lib(L, L.or_bench_tasks(n, lx, ly, lz, dptr(a), dptr(b), dptr(t), width, wolff_steps,
                                   ptr(s, C.c_uint64), sweeps, threads, C.byref(sec), C.byref(chk)))
    return sec.value, chk.value


def series_tasks(dims, jxy, jz, temperatures, seeds, thermalization, sweeps, n_bins, width=np.pi, wolff_steps=1,
                 threads=None, simd=False):
    """Independent reference-order tasks (FastRng streams) on host threads;
    returns bin means [n_tasks][n_bins][SERIES_COLS] of each task's measured
    series (`sweeps` a multiple of `n_bins`).  jxy/jz are [n_tasks][lz]."""
    lx, ly, lz = dims
    n = len(temperatures)
    a = np.ascontiguousarray(jxy, np.float64).reshape(n, lz)
    b = np.ascontiguousarray(jz, np.float64).reshape(n, lz)
    t = np.ascontiguousarray(temperatures, np.float64)
    s = np.ascontiguousarray(seeds, np.uint64)
    out = np.zeros((n, n_bins, SERIES_COLS))
    threads = threads or os.cpu_count() or 1
    L = baseline_lib() if simd else lib()
    _check_lib(L, L.or_series_tasks(n, lx, ly, lz, dptr(a), dptr(b), dptr(t), width, wolff_steps,
                                    ptr(s, C.c_uint64), thermalization, sweeps, n_bins, threads, dptr(out)))
    return out
