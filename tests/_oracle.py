"""ctypes binding of the CPU checker (oracle/liboracle.so) — test infrastructure.

OracleContext offers the same methods as cbm_b200.Context so that a test can
run one scenario through both and compare.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None


def load_oracle(abi):
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(ORACLE_DIR, "cbm_oracle.cpp")
    if (not os.path.exists(ORACLE_LIB)
            or os.path.getmtime(ORACLE_LIB) < os.path.getmtime(src)):
        subprocess.run(["sh", os.path.join(ORACLE_DIR, "build.sh")], check=True)
    lib = C.CDLL(ORACLE_LIB)
    vp, i32, i64, dbl, u32, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_uint32, C.c_uint64
    sig = {
        "oracle_set_threads": (None, [C.c_int]),
        "oracle_max_threads": (C.c_int, []),
        "oracle_create": (vp, [C.POINTER(abi.CbmConfig)]),
        "oracle_destroy": (None, [vp]),
        "oracle_upload": (C.c_int, [vp, C.POINTER(abi.CbmStateView)]),
        "oracle_download": (C.c_int, [vp, C.POINTER(abi.CbmStateView), C.c_int]),
        "oracle_stage": (C.c_int, [vp, C.c_int]),
        "oracle_step": (C.c_int, [vp, C.c_int]),
        "oracle_step_noise": (C.c_int, [vp, vp]),
        "oracle_take_error": (C.c_int, [vp]),
        "oracle_get_counters": (C.c_int, [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64),
                                          C.POINTER(i64), C.POINTER(i32), C.POINTER(i64)]),
        "oracle_grid_shape": (C.c_int, [vp, C.POINTER(i32)]),
        "oracle_get_grid": (C.c_int, [vp, vp, vp, vp, vp]),
        "oracle_get_neighbors": (C.c_int, [vp, vp, vp, i64]),
        "oracle_count_neighbors": (C.c_int, [vp, dbl, vp]),
        "oracle_rng_fill": (C.c_int, [C.c_int, u64, u32, C.c_int, dbl, dbl, i64, i64, vp]),
        "oracle_log_f64": (dbl, [dbl]),
        "oracle_log_f32": (C.c_float, [C.c_float]),
        "oracle_cossin_f64": (None, [dbl, C.POINTER(dbl), C.POINTER(dbl)]),
        "oracle_cossin_f32": (None, [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "oracle_philox": (None, [u32, u32, u32, u32, u32, u32, C.POINTER(u32)]),
        "oracle_normals": (None, [C.c_int, u64, i64, u32, u32, u32, C.c_int, vp]),
        "oracle_medium_create": (vp, [C.POINTER(abi.CbmMediumConfig)]),
        "oracle_medium_destroy": (None, [vp]),
        "oracle_medium_upload": (C.c_int, [vp, vp, vp]),
        "oracle_medium_step": (C.c_int, [vp, C.c_int]),
        "oracle_medium_download": (C.c_int, [vp, vp, C.POINTER(dbl)]),
        "oracle_rods_create": (vp, [C.POINTER(abi.CbmRodsConfig)]),
        "oracle_rods_destroy": (None, [vp]),
        "oracle_rods_upload": (C.c_int, [vp, C.c_int64, C.POINTER(vp)]),
        "oracle_rods_step": (C.c_int, [vp, C.c_int]),
        "oracle_rods_download": (C.c_int, [vp, C.POINTER(vp)]),
        "oracle_rod_pair_f64": (C.c_int, [C.POINTER(dbl)] * 4),
        "oracle_rods_count": (i64, [vp, C.POINTER(C.c_int)]),
        "oracle_uniform_f64": (dbl, [u64, i64, u32, u32, u32]),
        "oracle_uniform_f32": (C.c_float, [u64, i64, u32, u32, u32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


STAGE_ID = {"agent_rule": 0, "agent_de": 1, "medium_rule": 2, "medium_de": 3, "update": 4,
            "neighbors": 5}


class OracleContext:
    def __init__(self, abi, cfg, threads=1):
        self.abi = abi
        self.lib = load_oracle(abi)
        self.cfg = cfg
        self.lib.oracle_set_threads(threads)
        self.h = self.lib.oracle_create(C.byref(cfg))
        if not self.h:
            raise ValueError("oracle_create rejected the configuration")
        self.n_nodes = (int(np.prod([cfg.n_medium[d] for d in range(cfg.dims)]))
                        if cfg.medium else 0)

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, state, t=0.0, step=0, id_max=0):
        buf, N, present = self.abi.state_from_dict(self.cfg, state, n_nodes=self.n_nodes)
        view = buf.view(N=N, t=t, step=step, id_max=id_max, fields=present)
        rc = self.lib.oracle_upload(self.h, C.byref(view))
        assert rc == 0, rc

    def download(self, which=0, capacity=None):
        cap = capacity or max(int(self.cfg.n_max), 1)
        buf = self.abi.StateBuffers(self.cfg, cap, self.n_nodes)
        view = buf.view()
        rc = self.lib.oracle_download(self.h, C.byref(view), which)
        assert rc == 0, rc
        N = view.N
        out = {k: v[:N].copy() for k, v in buf.arrays.items()
               if k not in self.abi.StateBuffers.MEDIUM}
        if self.n_nodes:
            for k in self.abi.StateBuffers.MEDIUM:
                out[k] = buf.arrays[k][: self.n_nodes].copy()
        out.update(N=N, t=view.t, step=view.step, id_max=view.id_max)
        return out

    def step(self, n=1, flags=0):
        self.lib.oracle_step(self.h, n)
        return self.take_error()

    def step_noise(self, noise):
        """One step whose EM increments are `noise` (N x dims, index order)."""
        dt = np.float64 if self.cfg.precision == self.abi.F64 else np.float32
        buf = np.ascontiguousarray(noise, dtype=dt)
        self.lib.oracle_step_noise(self.h, buf.ctypes.data)
        return self.take_error()

    def take_error(self):
        return self.lib.oracle_take_error(self.h)

    def stage(self, name):
        rc = self.lib.oracle_stage(self.h, STAGE_ID[name])
        assert rc == 0

    def counters(self):
        v = [C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32(), C.c_int64()]
        self.lib.oracle_get_counters(self.h, *[C.byref(x) for x in v])
        return dict(N=v[0].value, n_add=v[1].value, n_remove=v[2].value, id_max=v[3].value,
                    flag=v[4].value, step=v[5].value)

    def grid(self):
        n3 = (C.c_int32 * 3)()
        self.lib.oracle_grid_shape(self.h, n3)
        nc = int(n3[0]) * int(n3[1]) * int(n3[2])
        N = self.counters()["N"]
        agent_cell = np.zeros(max(N, 1), np.int32)
        agents = np.zeros(max(N, 1), np.int32)
        start = np.zeros(nc, np.int32)
        count = np.zeros(nc, np.int32)
        self.lib.oracle_get_grid(self.h, agent_cell.ctypes.data, start.ctypes.data,
                                 count.ctypes.data, agents.ctypes.data)
        return dict(shape=tuple(int(v) for v in n3), agent_cell=agent_cell[:N], cell_start=start,
                    cell_count=count, cell_agents=agents[:N])

    def neighbors(self):
        N = self.counters()["N"]
        M = int(self.cfg.n_max_neighbors)
        counts = np.zeros(max(N, 1), np.int32)
        lst = np.zeros(max(N * M, 1), np.int32)
        rc = self.lib.oracle_get_neighbors(self.h, counts.ctypes.data, lst.ctypes.data, lst.size)
        assert rc == 0
        return counts[:N], lst[: N * M].reshape(N, M)

    def count_neighbors(self, radius):
        N = self.counters()["N"]
        out = np.zeros(max(N, 1), np.int32)
        self.lib.oracle_count_neighbors(self.h, float(radius), out.ctypes.data)
        return out[:N]

    def rng_fill(self, kind, a, b, n, step=0):
        dt = np.float64 if self.cfg.precision == self.abi.F64 else np.float32
        out = np.zeros(max(n, 1), dt)
        self.lib.oracle_rng_fill(self.cfg.precision, self.cfg.seed, self.cfg.community, kind,
                                 float(a), float(b), n, step, out.ctypes.data)
        return out[:n]


def oracle_adjoint_dual(abi, cfg, x0, target, nsteps, seeds=(), threads=None):
    """Forward-mode dual numbers of the Euler trajectory: (loss, dL/dtheta, dL/dx0[seeds]).
    Agents are evaluated on `threads` host threads (all cores by default); the
    result does not depend on the count."""
    lib = load_oracle(abi)
    lib.oracle_set_threads(int(threads or os.cpu_count()))
    f = lib.oracle_adjoint_dual
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.CbmConfig), C.c_int64, C.POINTER(C.c_void_p), C.c_int,
                  C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    xs = [np.ascontiguousarray(a, dtype=np.float64) for a in x0]
    ts = [np.ascontiguousarray(a, dtype=np.float64) for a in target]
    xp = (C.c_void_p * 3)(*[a.ctypes.data for a in xs])
    tp = (C.c_void_p * 3)(*[a.ctypes.data for a in ts])
    ns = len(seeds)
    sa = (C.c_int64 * max(ns, 1))(*[s[0] for s in seeds])
    sx = (C.c_int32 * max(ns, 1))(*[s[1] for s in seeds])
    loss = C.c_double()
    g = (C.c_double * 3)()
    dx = (C.c_double * max(ns, 1))()
    rc = f(C.byref(cfg), len(xs[0]), xp, nsteps, tp, ns, sa, sx, C.byref(loss), g, dx)
    assert rc == 0
    return loss.value, np.array(list(g)), np.array(list(dx)[:ns])


class OracleMedium:
    """The DGADI medium of the checker, with cbm_b200.Medium's methods."""

    def __init__(self, abi, cfg):
        self.lib = load_oracle(abi)
        self.h = self.lib.oracle_medium_create(C.byref(cfg))
        if not self.h:
            raise ValueError("invalid medium configuration")
        self.dtype = np.float64 if cfg.precision == abi.F64 else np.float32
        self.shape = (cfg.n_fields,) + tuple(int(cfg.n[d]) for d in reversed(range(cfg.dims)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle_medium_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, fields, source=None):
        f = np.ascontiguousarray(fields, dtype=self.dtype).reshape(self.shape)
        s = None if source is None else np.ascontiguousarray(source, dtype=self.dtype)
        self.lib.oracle_medium_upload(self.h, f.ctypes.data, None if s is None else s.ctypes.data)

    def step(self, n):
        self.lib.oracle_medium_step(self.h, n)

    def download(self):
        out = np.zeros(self.shape, self.dtype)
        t = C.c_double()
        self.lib.oracle_medium_download(self.h, out.ctypes.data, C.byref(t))
        return out, t.value


class OracleRods:
    """The rods2D Euler step of the checker, with Rods2D's methods."""

    def __init__(self, abi, cfg):
        self.abi = abi
        self.lib = load_oracle(abi)
        self.h = self.lib.oracle_rods_create(C.byref(cfg))
        self.dtype = np.float64 if cfg.precision == abi.F64 else np.float32
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle_rods_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, state):
        nf = len(self.abi.ROD_FIELDS)
        arrs = [np.ascontiguousarray(state[k], dtype=self.dtype) for k in self.abi.ROD_FIELDS[:12]]
        self.n = len(arrs[0])
        lt = np.ascontiguousarray(state.get("l_target", np.zeros(self.n)), dtype=self.dtype)
        self._keep = arrs + [lt]
        ptrs = (C.c_void_p * nf)(*([a.ctypes.data for a in arrs] + [None, lt.ctypes.data]))
        self.lib.oracle_rods_upload(self.h, self.n, ptrs)

    def step(self, n):
        self.lib.oracle_rods_step(self.h, n)

    def count(self):
        err = C.c_int()
        n = self.lib.oracle_rods_count(self.h, C.byref(err))
        return int(n), int(err.value)

    def download(self):
        nf = len(self.abi.ROD_FIELDS)
        self.n = self.count()[0]
        out = np.zeros((nf, self.n), self.dtype)
        ptrs = (C.c_void_p * nf)(*[out[q].ctypes.data for q in range(nf)])
        self.lib.oracle_rods_download(self.h, ptrs)
        return {k: out[q] for q, k in enumerate(self.abi.ROD_FIELDS)}


def oracle_rod_pair(abi, a, b, k):
    """rodForces of one pair (a, b: x, y, d, l, theta, vx, vy, m; k: kn, γn,
    γt, μcc) in Float64: (contact, [Fx, Fy, W, xi, yi, xj, yj])."""
    lib = load_oracle(abi)
    arr = [np.ascontiguousarray(v, dtype=np.float64) for v in (a, b, k)]
    out = np.zeros(7)
    dp = C.POINTER(C.c_double)
    c = lib.oracle_rod_pair_f64(*(v.ctypes.data_as(dp) for v in arr), out.ctypes.data_as(dp))
    return bool(c), out
