"""Python binding of the slsf-b200 C ABI (include/slsf_gpu.h).

The CUDA library `libslsf_b200.so` is built in-tree by `build()` (nvcc,
sm_100a).  This module only marshals arguments; every computation runs in the
library on the GPU.  There is no CPU fallback: loading fails loudly when the
library is missing, and context creation fails when there is no CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libslsf_b200.so")
HEADER = os.path.join(ROOT, "include", "slsf_gpu.h")

OK, ERR_INVALID, ERR_CUDA, ERR_BUDGET, ERR_TIMEOUT, ERR_STATE = range(6)
OBS_FIELDS = ("energy", "magnetization_squared", "cos_x", "cos_y", "cos_z", "sin_x", "sin_y", "sin_z")
BIN_COLS = 12
BIN_NAMES = ("Energy", "EnergySquared", "MagnetizationSquared", "_helicity_cos_x", "_helicity_cos_y",
             "_helicity_cos_z", "_helicity_sin_x", "_helicity_sin_y", "_helicity_sin_z", "_helicity_sin2_x",
             "_helicity_sin2_y", "_helicity_sin2_z")


class SlsfError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class TaskDesc(C.Structure):
    _fields_ = [
        ("lx", C.c_uint32), ("ly", C.c_uint32), ("lz", C.c_uint32),
        ("temperature", C.c_double), ("proposal_width", C.c_double),
        ("wolff_steps", C.c_uint32), ("seed", C.c_uint64),
        ("j_xy", C.POINTER(C.c_double)), ("n_j_xy", C.c_size_t),
        ("j_z", C.POINTER(C.c_double)), ("n_j_z", C.c_size_t),
        ("thermalization", C.c_uint32), ("binsize", C.c_uint32), ("n_bins", C.c_uint32),
    ]


class Observables(C.Structure):
    _fields_ = [(n, C.c_double) for n in OBS_FIELDS]

    def as_dict(self):
        return {n: getattr(self, n) for n in OBS_FIELDS}


class SweepStats(C.Structure):
    _fields_ = [("sweeps", C.c_uint64), ("accepted", C.c_uint64), ("wolff_clusters", C.c_uint64),
                ("wolff_cluster_sites", C.c_uint64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


KERNEL_KINDS = ("resident", "cluster", "grid")


class KernelChoice(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("cluster", C.c_uint32), ("threads", C.c_uint32)]

    def as_dict(self):
        return {"kind": KERNEL_KINDS[self.kind], "cluster": self.cluster, "threads": self.threads}


def build(force: bool = False) -> str:
    """Compile the library with nvcc for sm_100a (works without a GPU)."""
    if force:
        subprocess.run(["make", "-s", "-C", HERE, "clean"], check=True)
    subprocess.run(["make", "-s", "-j8", "-C", HERE], check=True)
    return LIB_PATH


_P = C.c_void_p
_U8P = C.POINTER(C.c_uint8)
_F32P = C.POINTER(C.c_float)
_F64P = C.POINTER(C.c_double)
_U32P = C.POINTER(C.c_uint32)
_U64P = C.POINTER(C.c_uint64)

SIGNATURES = {
    "slsf_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "slsf_version": (C.c_char_p, []),
    "slsf_ctx_create": (C.c_int, [C.c_int, C.c_uint64, C.c_uint32, C.POINTER(_P)]),
    "slsf_ctx_destroy": (C.c_int, [_P]),
    "slsf_ctx_memory": (C.c_int, [_P, _U64P, _U64P]),
    "slsf_task_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]),
    "slsf_task_create": (C.c_int, [_P, C.POINTER(TaskDesc), C.POINTER(_P)]),
    "slsf_task_destroy": (C.c_int, [_P]),
    "slsf_task_init_random": (C.c_int, [_P]),
    "slsf_task_init_cold": (C.c_int, [_P]),
    "slsf_task_set_angles": (C.c_int, [_P, _F32P, C.c_size_t]),
    "slsf_task_get_angles": (C.c_int, [_P, _F32P, C.c_size_t]),
    "slsf_task_get_counters": (C.c_int, [_P, _U64P, _U64P]),
    "slsf_task_set_counters": (C.c_int, [_P, C.c_uint64, C.c_uint64]),
    "slsf_task_sweep": (C.c_int, [_P, C.c_uint32, C.POINTER(SweepStats)]),
    "slsf_task_metropolis_sweep": (C.c_int, [_P, _F64P]),
    "slsf_task_metropolis_color": (C.c_int, [_P, C.c_uint32, _U8P, _U64P]),
    "slsf_task_wolff_step": (C.c_int, [_P, _U64P]),
    "slsf_task_wolff_step_debug": (C.c_int, [_P, _U8P, _U8P, _F32P, _U32P, _U64P]),
    "slsf_task_measure": (C.c_int, [_P, C.POINTER(Observables)]),
    "slsf_task_correlations": (C.c_int, [_P, C.c_uint32, C.c_uint32, _F64P, _F64P, _F64P, _F64P, _F64P]),
    "slsf_task_get_bins": (C.c_int, [_P, _F64P, C.c_size_t, _U64P]),
    "slsf_task_corr_setup": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_size_t)]),
    "slsf_task_corr_bins": (C.c_int, [_P, _F64P, C.c_size_t, _U64P]),
    "slsf_task_corr_fuse": (C.c_int, [_P, C.c_uint32]),
    "slsf_batch_correlations": (C.c_int, [_P, C.POINTER(_P), C.c_size_t]),
    "slsf_task_state_size": (C.c_int, [_P, C.POINTER(C.c_size_t)]),
    "slsf_task_state_save": (C.c_int, [_P, _U64P, _P, C.c_size_t]),
    "slsf_task_state_load": (C.c_int, [_P, _P, C.c_size_t, _U64P]),
    "slsf_task_reset_bins": (C.c_int, [_P]),
    "slsf_batch_run": (C.c_int, [_P, C.POINTER(_P), C.c_size_t, C.c_uint32, C.POINTER(SweepStats)]),
    "slsf_batch_get_bins": (C.c_int, [_P, C.POINTER(_P), C.c_size_t, C.c_size_t, _F64P, _U64P]),
    "slsf_batch_run_v": (C.c_int, [_P, C.POINTER(_P), C.c_size_t, _U32P, C.POINTER(SweepStats)]),
    "slsf_ctx_set_stream": (C.c_int, [_P, _P]),
    "slsf_ctx_launch_count": (C.c_int, [_P, _U64P]),
    "slsf_ctx_set_loop_limit": (C.c_int, [_P, C.c_uint32]),
    "slsf_batch_open": (C.c_int, [_P, C.POINTER(_P), C.c_size_t, C.c_uint32, C.POINTER(_P)]),
    "slsf_batch_step": (C.c_int, [_P, C.POINTER(SweepStats)]),
    "slsf_batch_close": (C.c_int, [_P]),
    "slsf_batch_step_correlations": (C.c_int, [_P, C.c_uint32, C.POINTER(SweepStats)]),
    "slsf_tune_get": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(KernelChoice)]),
    "slsf_tune_set": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(KernelChoice)]),
    "slsf_autotune": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(KernelChoice),
                                C.POINTER(C.c_double)]),
    "slsf_tune_save": (C.c_int, [_P, C.c_char_p]),
    "slsf_tune_load": (C.c_int, [_P, C.c_char_p]),
    "slsf_measure_noalloc": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_uint32, C.c_uint32, _P,
                                       C.POINTER(Observables)]),
}

_lib = None


def load():
    """Load the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run build() (nvcc, sm_100a) first")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().slsf_last_error(buf, len(buf))
    return buf.value.decode("utf-8")


def check(code):
    if code != OK:
        raise SlsfError(code, last_error())


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class Context:
    """A device context (slsf_ctx_create)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0):
        import weakref

        h = _P()
        check(load().slsf_ctx_create(device, budget_bytes, 0, C.byref(h)))
        self.h = h
        self._tasks = weakref.WeakSet()
        self._servers = weakref.WeakSet()
        self._sessions = weakref.WeakSet()

    def close(self):
        """Destroy every live server and task of this context, then the context."""
        if getattr(self, "h", None):
            for srv in list(self._servers):
                srv.close()
            for ses in list(self._sessions):
                ses.close()
            for t in list(self._tasks):
                t.close()
            check(load().slsf_ctx_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_loop_limit(self, limit):
        """Bound of every device loop of later launches (0: defaults)."""
        check(load().slsf_ctx_set_loop_limit(self.h, limit))

    def tune_get(self, dims):
        c = KernelChoice()
        check(load().slsf_tune_get(self.h, *dims, C.byref(c)))
        return c.as_dict()

    def tune_set(self, dims, kind, cluster=1, threads=1024):
        c = KernelChoice(KERNEL_KINDS.index(kind), cluster, threads)
        check(load().slsf_tune_set(self.h, *dims, C.byref(c)))

    def autotune(self, dims, sweeps=0):
        """Times every feasible kernel choice for the shape; keeps and returns the fastest."""
        c, r = KernelChoice(), C.c_double()
        check(load().slsf_autotune(self.h, *dims, sweeps, C.byref(c), C.byref(r)))
        return dict(c.as_dict(), site_updates_per_s=r.value)

    def tune_save(self, path):
        check(load().slsf_tune_save(self.h, str(path).encode()))

    def tune_load(self, path):
        check(load().slsf_tune_load(self.h, str(path).encode()))

    def memory(self):
        used, budget = C.c_uint64(), C.c_uint64()
        check(load().slsf_ctx_memory(self.h, C.byref(used), C.byref(budget)))
        return used.value, budget.value

    def batch_run(self, tasks, n_sweeps, handles=None):
        """Run n_sweeps sweeps of every task in one persistent launch.

        `handles` may be a prepared ctypes array of the task handles (see
        `handle_array`) to avoid rebuilding it on every call."""
        arr = handles if handles is not None else self.handle_array(tasks)
        stats = (SweepStats * len(tasks))()
        check(load().slsf_batch_run(self.h, arr, len(tasks), n_sweeps, stats))
        return [s.as_dict() for s in stats]

    def batch_correlations(self, tasks, handles=None):
        """One correlation measurement of every task into its device bins
        (queued on the context's stream; returns without waiting)."""
        arr = handles if handles is not None else self.handle_array(tasks)
        check(load().slsf_batch_correlations(self.h, arr, len(tasks)))

    def session(self, tasks, n_sweeps):
        """A batch session: one captured step of n_sweeps sweeps, replayed by step()."""
        return BatchSession(self, tasks, n_sweeps)

    @staticmethod
    def handle_array(tasks):
        return (_P * len(tasks))(*[t.h for t in tasks])

    def batch_bins(self, tasks, n_rows, out=None, handles=None):
        """Bin means of every task: array [n_tasks, n_rows, 12] (one gather, one copy)."""
        arr = handles if handles is not None else self.handle_array(tasks)
        if out is None:
            out = np.zeros((len(tasks), n_rows, BIN_COLS))
        meas = np.zeros(len(tasks), dtype=np.uint64)
        check(load().slsf_batch_get_bins(self.h, arr, len(tasks), n_rows, _ptr(out, C.c_double),
                                         _ptr(meas, C.c_uint64)))
        return out, meas

    def set_stream(self, stream_handle):
        """Run the context's work on a cudaStream_t (an int handle; 0 = own stream)."""
        check(load().slsf_ctx_set_stream(self.h, C.c_void_p(stream_handle or None)))

    @property
    def launches(self):
        n = C.c_uint64()
        check(load().slsf_ctx_launch_count(self.h, C.byref(n)))
        return n.value


class BatchSession:
    """slsf_batch_open / slsf_batch_step / slsf_batch_close: one batched step
    captured in a CUDA graph and replayed."""

    def __init__(self, ctx, tasks, n_sweeps):
        h = _P()
        arr = ctx.handle_array(tasks)
        check(load().slsf_batch_open(ctx.h, arr, len(tasks), n_sweeps, C.byref(h)))
        self.h = h
        self.n = len(tasks)
        self.ctx = ctx
        ctx._sessions.add(self)

    def step(self):
        st = (SweepStats * self.n)()
        check(load().slsf_batch_step(self.h, st))
        return [x.as_dict() for x in st]

    def step_correlations(self, n_cycles, raw=None):
        """n_cycles x (step + one correlation measurement of every task)
        (slsf_batch_step_correlations).  Returns the summed stats as a
        uint64 array [n_tasks, 4] (sweeps, accepted, wolff_clusters,
        wolff_cluster_sites)."""
        st = raw if raw is not None else (SweepStats * self.n)()
        check(load().slsf_batch_step_correlations(self.h, n_cycles, st))
        return np.ctypeslib.as_array(st).view(np.uint64).reshape(self.n, 4)

    def close(self):
        if getattr(self, "h", None):
            load().slsf_batch_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Task:
    """One task (slsf_task_create): the device state of a ThetaModel."""

    def __init__(self, ctx: Context, dims, j_xy, j_z, temperature, proposal_width=np.pi, wolff_steps=1, seed=0,
                 thermalization=0, binsize=1, n_bins=0):
        lx, ly, lz = dims
        self.dims = (lx, ly, lz)
        self.volume = lx * ly * lz
        self._jxy = np.ascontiguousarray(j_xy, dtype=np.float64)
        self._jz = np.ascontiguousarray(j_z, dtype=np.float64)
        d = TaskDesc(lx=lx, ly=ly, lz=lz, temperature=temperature, proposal_width=proposal_width,
                     wolff_steps=wolff_steps, seed=seed, j_xy=_ptr(self._jxy, C.c_double), n_j_xy=self._jxy.size,
                     j_z=_ptr(self._jz, C.c_double), n_j_z=self._jz.size, thermalization=thermalization,
                     binsize=binsize, n_bins=n_bins)
        if not getattr(ctx, "h", None):
            raise SlsfError(ERR_STATE, "context is closed")
        h = _P()
        check(load().slsf_task_create(ctx.h, C.byref(d), C.byref(h)))
        self.h = h
        self.ctx = ctx
        self.n_bins = n_bins
        self.corr_n_values = self.corr_n_bins = 0
        ctx._tasks.add(self)

    def close(self):
        if getattr(self, "h", None):
            load().slsf_task_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_random(self):
        check(load().slsf_task_init_random(self.h))

    def init_cold(self):
        check(load().slsf_task_init_cold(self.h))

    @property
    def theta(self):
        out = np.empty(self.volume, dtype=np.float32)
        check(load().slsf_task_get_angles(self.h, _ptr(out, C.c_float), out.size))
        return out

    @theta.setter
    def theta(self, values):
        v = np.ascontiguousarray(values, dtype=np.float32)
        check(load().slsf_task_set_angles(self.h, _ptr(v, C.c_float), v.size))

    @property
    def counters(self):
        a, b = C.c_uint64(), C.c_uint64()
        check(load().slsf_task_get_counters(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    @counters.setter
    def counters(self, value):
        check(load().slsf_task_set_counters(self.h, value[0], value[1]))

    def sweep(self, n=1):
        st = SweepStats()
        check(load().slsf_task_sweep(self.h, n, C.byref(st)))
        return st.as_dict()

    def metropolis_sweep(self):
        acc = C.c_double()
        check(load().slsf_task_metropolis_sweep(self.h, C.byref(acc)))
        return acc.value

    def metropolis_color(self, colour, record=True):
        acc = C.c_uint64()
        mask = np.zeros(self.volume, dtype=np.uint8) if record else None
        check(load().slsf_task_metropolis_color(self.h, colour, _ptr(mask, C.c_uint8) if record else None,
                                                C.byref(acc)))
        return acc.value, mask

    def wolff_step(self):
        n = C.c_uint64()
        check(load().slsf_task_wolff_step(self.h, C.byref(n)))
        return n.value

    def wolff_step_debug(self):
        bonds = np.zeros(self.volume, dtype=np.uint8)
        cluster = np.zeros(self.volume, dtype=np.uint8)
        phi = C.c_float()
        site = (C.c_uint32 * 3)()
        n = C.c_uint64()
        check(load().slsf_task_wolff_step_debug(self.h, _ptr(bonds, C.c_uint8), _ptr(cluster, C.c_uint8),
                                                C.byref(phi), site, C.byref(n)))
        return {"bonds": bonds, "cluster": cluster, "phi": phi.value, "seed_site": tuple(site), "size": n.value}

    def measure(self):
        o = Observables()
        check(load().slsf_task_measure(self.h, C.byref(o)))
        return o.as_dict()

    def correlations(self, rmax_xy, rmax_z):
        lx, ly, lz = self.dims
        rxy = min(rmax_xy, lx // 2, ly // 2)
        rz = min(rmax_z, lz // 2)
        cx, cy, cxy = np.zeros(max(rxy, 1)), np.zeros(max(rxy, 1)), np.zeros(max(rxy, 1))
        cbz, cz = np.zeros(max(lz * rxy, 1)), np.zeros(max(rz, 1))
        f = lambda a: _ptr(a, C.c_double)
        check(load().slsf_task_correlations(self.h, rmax_xy, rmax_z, f(cx), f(cy), f(cxy), f(cbz), f(cz)))
        return {"corr_x": cx[:rxy], "corr_y": cy[:rxy], "corr_xy": cxy[:rxy],
                "corr_xy_by_z": cbz[: lz * rxy].reshape(lz, rxy), "corr_z": cz[:rz]}

    def corr_setup(self, rmax_xy, rmax_z, binsize, n_bins):
        """Correlation bins on the device (slsf_task_corr_setup); returns the
        number of values one correlation measurement produces."""
        nv = C.c_size_t()
        check(load().slsf_task_corr_setup(self.h, rmax_xy, rmax_z, binsize, n_bins, C.byref(nv)))
        self.corr_n_values, self.corr_n_bins = nv.value, n_bins
        return nv.value

    def corr_fuse(self, interval):
        """Measure the correlations inside the batched sweeps every `interval`
        measurements (slsf_task_corr_fuse; 0: off)."""
        check(load().slsf_task_corr_fuse(self.h, interval))

    def corr_bins(self, n_rows=None):
        """(bin means [n_rows][values], correlation measurements so far)."""
        n_rows = self.corr_n_bins if n_rows is None else n_rows
        out = np.zeros((max(n_rows, 1), max(self.corr_n_values, 1)))
        m = C.c_uint64()
        check(load().slsf_task_corr_bins(self.h, _ptr(out, C.c_double), n_rows, C.byref(m)))
        return out[:n_rows, : self.corr_n_values], m.value

    def save_state(self, user=(0, 0, 0, 0)) -> bytes:
        """The task's device state (slsf_task_state_save) with four caller words."""
        n = C.c_size_t()
        check(load().slsf_task_state_size(self.h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        words = (C.c_uint64 * 4)(*user)
        check(load().slsf_task_state_save(self.h, words, buf, n.value))
        return buf.raw

    def load_state(self, blob: bytes):
        """Restores a saved state; returns its four caller words."""
        words = (C.c_uint64 * 4)()
        buf = C.create_string_buffer(blob, len(blob))
        check(load().slsf_task_state_load(self.h, buf, len(blob), words))
        return tuple(words)

    def bins(self):
        out = np.zeros((max(self.n_bins, 1), BIN_COLS))
        m = C.c_uint64()
        check(load().slsf_task_get_bins(self.h, _ptr(out, C.c_double), self.n_bins, C.byref(m)))
        return out[: self.n_bins], m.value

    def reset_bins(self):
        check(load().slsf_task_reset_bins(self.h))


_MASK64 = (1 << 64) - 1


def splitmix64_uniforms(seed: int, n: int):
    """n uniforms in [0, 1) from FastRng(seed) (src/types.rs:18-24): SplitMix64
    words, top 53 bits times 2^-53 (rand's f64 sampling)."""
    out = []
    state = seed & _MASK64
    for _ in range(n):
        state = (state + 0x9E3779B97F4A7C15) & _MASK64
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK64
        z ^= z >> 31
        out.append((z >> 11) * (1.0 / 9007199254740992.0))
    return np.array(out)


def uniform_layer_disorder(lz: int, lo: float, hi: float, seed: int):
    """Per-layer couplings lo + (hi - lo) u_z, u_z from FastRng(seed) in layer
    order: the "J_z(z) uniform [0.5, 1.5] per layer from seed" workloads."""
    return lo + (hi - lo) * splitmix64_uniforms(seed, lz)


def _round_as_u64(x: float) -> int:
    """`x.round() as u64`: halves round away from zero, then the cast
    saturates (NaN and negatives to 0, past the range to 2^64 - 1)."""
    import math

    if math.isnan(x) or x <= 0.0:
        return 0
    if math.isinf(x):
        return _MASK64
    f = math.floor(x)
    return min(int(f) + (1 if x - f >= 0.5 else 0), _MASK64)


def task_seed(base_seed: int, l_z: int, sample: int, temperature: float, delta_j_xy: float = 0.0,
              delta_j_z: float = 0.0) -> int:
    """Run seed of a task (ThetaJobConfig::make_theta_tasks, src/model.rs:741-747);
    the sums wrap modulo 2^64."""
    return (base_seed + 100_000 * l_z + 1_000 * sample + _round_as_u64(100.0 * temperature)
            + _round_as_u64(1_000.0 * delta_j_xy) * 10_000 + _round_as_u64(1_000.0 * delta_j_z)) & _MASK64


def exported_symbols():
    """Function names declared in include/slsf_gpu.h."""
    import re

    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(slsf_[a-z_0-9]+)\s*\(", text)))


# ---------------------------------------------------------------- host layer (include/slsf_host.h)
HOST_LIB_PATH = os.path.join(HERE, "libslsf_host.so")
HOST_HEADER = os.path.join(ROOT, "include", "slsf_host.h")
DERIVED = ("Magnetization", "Chi", "SpecificHeat", "RhoXY", "RhoZ")


class Estimates(C.Structure):
    _fields_ = [("measurements", C.c_uint64), ("n_bins", C.c_uint32), ("acceptance", C.c_double),
                ("mean", C.c_double * BIN_COLS), ("err", C.c_double * BIN_COLS),
                ("derived", C.c_double * 5), ("derived_err", C.c_double * 5)]

    def as_dict(self):
        d = {"measurements": self.measurements, "n_bins": self.n_bins, "acceptance": self.acceptance}
        for k, name in enumerate(BIN_NAMES):
            d[name] = (self.mean[k], self.err[k])
        for k, name in enumerate(DERIVED):
            d[name] = (self.derived[k], self.derived_err[k])
        return d


class ThetaTaskDesc(C.Structure):
    _fields_ = [("lx", C.c_uint32), ("ly", C.c_uint32), ("lz", C.c_uint32), ("temperature", C.c_double),
                ("j_xy", C.c_double), ("delta_j_xy", C.c_double), ("j_z_mean", C.c_double),
                ("delta_j_z", C.c_double), ("disorder_seed", C.c_uint64), ("seed", C.c_uint64),
                ("sweeps", C.c_uint32), ("thermalization", C.c_uint32), ("binsize", C.c_uint32),
                ("proposal_width", C.c_double), ("wolff_steps", C.c_uint32),
                ("j_xy_array", C.POINTER(C.c_double)), ("j_z_array", C.POINTER(C.c_double))]


class ServerConfig(C.Structure):
    _fields_ = [("epoch_sweeps", C.c_uint32), ("max_active", C.c_uint32), ("budget_bytes", C.c_uint64),
                ("keep_bins", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("lx", C.c_uint32), ("ly", C.c_uint32), ("lz", C.c_uint32),
                ("temperature", C.c_double), ("proposal_width", C.c_double), ("wolff_steps", C.c_uint32),
                ("seed", C.c_uint64), ("j_xy", C.POINTER(C.c_double)), ("j_z", C.POINTER(C.c_double)),
                ("sweeps", C.c_uint32), ("thermalization", C.c_uint32), ("n_bins", C.c_uint32),
                ("binsize", C.c_uint32)]


class Result(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("status", C.c_int), ("message", C.c_char * 160), ("submit_s", C.c_double),
                ("admit_s", C.c_double), ("finish_s", C.c_double), ("sweeps", C.c_uint64),
                ("accepted", C.c_uint64), ("cluster_sites", C.c_uint64), ("est", Estimates)]

    def as_dict(self):
        return {"tag": self.tag, "status": self.status, "message": self.message.decode(), "submit_s": self.submit_s,
                "admit_s": self.admit_s, "finish_s": self.finish_s, "sweeps": self.sweeps,
                "accepted": self.accepted, "cluster_sites": self.cluster_sites, "est": self.est.as_dict()}


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("cancelled", C.c_uint64), ("epochs", C.c_uint64), ("launches", C.c_uint64),
                ("site_updates", C.c_uint64), ("busy_s", C.c_double), ("peak_active", C.c_uint64),
                ("peak_bytes", C.c_uint64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


HOST_SIGNATURES = {
    "slsf_host_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "slsf_binned_estimate": (C.c_int, [_F64P, C.c_size_t, C.c_size_t, _F64P, _F64P, C.POINTER(C.c_size_t)]),
    "slsf_estimates_from_bins": (C.c_int, [_F64P, C.c_size_t, C.c_double, C.c_double, C.POINTER(Estimates)]),
    "slsf_task_seed": (C.c_uint64, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double]),
    "slsf_task_couplings": (C.c_int, [C.POINTER(ThetaTaskDesc), _F64P, _F64P]),
    "slsf_model_run": (C.c_int, [_P, C.POINTER(ThetaTaskDesc), C.c_int, C.POINTER(Estimates)]),
    "slsf_server_create": (C.c_int, [_P, C.POINTER(ServerConfig), C.POINTER(_P)]),
    "slsf_server_destroy": (C.c_int, [_P]),
    "slsf_server_submit": (C.c_int, [_P, C.POINTER(Request)]),
    "slsf_server_cancel": (C.c_int, [_P, C.c_uint64]),
    "slsf_server_step": (C.c_int, [_P, _U32P, _U32P]),
    "slsf_server_start": (C.c_int, [_P]),
    "slsf_server_stop": (C.c_int, [_P]),
    "slsf_server_wait_idle": (C.c_int, [_P, C.c_double]),
    "slsf_server_poll": (C.c_int, [_P, C.POINTER(Result), C.c_size_t, C.POINTER(C.c_size_t)]),
    "slsf_server_stats_get": (C.c_int, [_P, C.POINTER(ServerStats)]),
    "slsf_server_take_bins": (C.c_int, [_P, C.c_uint64, _F64P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "slsf_server_checkpoint": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_size_t)]),
    "slsf_server_restore": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_size_t)]),
}

_host = None


def load_host():
    global _host
    if _host is not None:
        return _host
    load()
    if not os.path.exists(HOST_LIB_PATH):
        raise RuntimeError(f"{HOST_LIB_PATH} is missing: run build() first")
    lib = C.CDLL(HOST_LIB_PATH)
    for name, (res, args) in HOST_SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _host = lib
    return lib


def host_last_error() -> str:
    buf = C.create_string_buffer(1024)
    load_host().slsf_host_last_error(buf, len(buf))
    return buf.value.decode("utf-8")


def host_check(code):
    if code != OK:
        raise SlsfError(code, host_last_error())


def host_declared_symbols():
    import re

    text = re.sub(r"/\*.*?\*/", "", open(HOST_HEADER).read(), flags=re.S)
    return sorted(set(re.findall(r"\b(slsf_[a-z_0-9]+)\s*\(", text)))


def binned_estimate(samples, binsize):
    a = np.ascontiguousarray(samples, np.float64)
    mean, err, nb = C.c_double(), C.c_double(), C.c_size_t()
    host_check(load_host().slsf_binned_estimate(_ptr(a, C.c_double), a.size, binsize, C.byref(mean), C.byref(err),
                                                C.byref(nb)))
    return {"mean": mean.value, "stderr": err.value, "n_bins": nb.value}


def theta_task(dims, temperature, sweeps, thermalization, binsize, seed, disorder_seed=0, j_xy=1.0, delta_j_xy=0.0,
               j_z_mean=0.1, delta_j_z=0.0, proposal_width=np.pi, wolff_steps=1, j_xy_array=None, j_z_array=None):
    """A ThetaTask (src/model.rs:20-47); keeps the J arrays alive on the struct."""
    d = ThetaTaskDesc(lx=dims[0], ly=dims[1], lz=dims[2], temperature=temperature, j_xy=j_xy, delta_j_xy=delta_j_xy,
                      j_z_mean=j_z_mean, delta_j_z=delta_j_z, disorder_seed=disorder_seed, seed=seed, sweeps=sweeps,
                      thermalization=thermalization, binsize=binsize, proposal_width=proposal_width,
                      wolff_steps=wolff_steps)
    keep = []
    if j_xy_array is not None:
        a = np.ascontiguousarray(j_xy_array, np.float64)
        keep.append(a)
        d.j_xy_array = _ptr(a, C.c_double)
    if j_z_array is not None:
        b = np.ascontiguousarray(j_z_array, np.float64)
        keep.append(b)
        d.j_z_array = _ptr(b, C.c_double)
    d._keep = keep
    return d


def task_couplings(desc):
    jx, jz = np.zeros(desc.lz), np.zeros(desc.lz)
    host_check(load_host().slsf_task_couplings(C.byref(desc), _ptr(jx, C.c_double), _ptr(jz, C.c_double)))
    return jx, jz


def model_run(ctx, desc, batched=True):
    """ThetaModel driven the way carlo-mc drives it; returns binned estimates."""
    e = Estimates()
    host_check(load_host().slsf_model_run(ctx.h, C.byref(desc), int(batched), C.byref(e)))
    return e.as_dict()


class Server:
    """Continuous-batching server (slsf_server_*)."""

    def __init__(self, ctx, epoch_sweeps=100, max_active=0, budget_bytes=0, keep_bins=False):
        h = _P()
        cfg = ServerConfig(epoch_sweeps=epoch_sweeps, max_active=max_active, budget_bytes=budget_bytes,
                           keep_bins=int(bool(keep_bins)))
        host_check(load_host().slsf_server_create(ctx.h, C.byref(cfg), C.byref(h)))
        self.h = h
        self.ctx = ctx
        ctx._servers.add(self)

    def close(self):
        if getattr(self, "h", None):
            load_host().slsf_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, tag, dims, temperature, seed, j_xy, j_z, sweeps, thermalization=0, n_bins=1,
               proposal_width=np.pi, wolff_steps=1, binsize=0):
        """Queues a request; `sweeps` counts the thermalization sweeps too."""
        jx = np.ascontiguousarray(j_xy, np.float64)
        jz = np.ascontiguousarray(j_z, np.float64)
        r = Request(tag=tag, lx=dims[0], ly=dims[1], lz=dims[2], temperature=temperature,
                    proposal_width=proposal_width, wolff_steps=wolff_steps, seed=seed, j_xy=_ptr(jx, C.c_double),
                    j_z=_ptr(jz, C.c_double), sweeps=sweeps, thermalization=thermalization, n_bins=n_bins,
                    binsize=binsize)
        host_check(load_host().slsf_server_submit(self.h, C.byref(r)))

    def cancel(self, tag):
        host_check(load_host().slsf_server_cancel(self.h, tag))

    def step(self):
        a, p = C.c_uint32(), C.c_uint32()
        host_check(load_host().slsf_server_step(self.h, C.byref(a), C.byref(p)))
        return a.value, p.value

    def start(self):
        host_check(load_host().slsf_server_start(self.h))

    def stop(self):
        host_check(load_host().slsf_server_stop(self.h))

    def wait_idle(self, timeout_s=600.0):
        host_check(load_host().slsf_server_wait_idle(self.h, timeout_s))

    def poll(self, max_results=4096):
        buf = (Result * max_results)()
        n = C.c_size_t()
        host_check(load_host().slsf_server_poll(self.h, buf, max_results, C.byref(n)))
        return [buf[i].as_dict() for i in range(n.value)]

    def take_bins(self, tag):
        """Bin means [n_rows, BIN_COLS] of a finished request (server created with keep_bins)."""
        n = C.c_size_t()
        host_check(load_host().slsf_server_take_bins(self.h, tag, None, 0, C.byref(n)))
        out = np.empty((n.value, BIN_COLS), dtype=np.float64)
        host_check(load_host().slsf_server_take_bins(self.h, tag, _ptr(out, C.c_double), n.value, C.byref(n)))
        return out

    def checkpoint(self, directory):
        """Writes every unfinished request to `directory` (worker stopped); returns the count."""
        n = C.c_size_t()
        host_check(load_host().slsf_server_checkpoint(self.h, str(directory).encode(), C.byref(n)))
        return n.value

    def restore(self, directory):
        """Queues the requests saved in `directory`; returns the count."""
        n = C.c_size_t()
        host_check(load_host().slsf_server_restore(self.h, str(directory).encode(), C.byref(n)))
        return n.value

    def stats(self):
        st = ServerStats()
        host_check(load_host().slsf_server_stats_get(self.h, C.byref(st)))
        return st.as_dict()
