"""ctypes binding of include/cbm_b200.h (libcbm_b200.so).

The structures mirror the C declarations field by field; `Context` wraps one
cbm_ctx.  There is no fallback: if the shared library or a CUDA device is
missing, loading or cbm_create fails with an exception.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcbm_b200.so")

# ---- constants (include/cbm_b200.h) ------------------------------------------
CBM_OK = 0
CBM_ERR_ARG = 1
CBM_ERR_CUDA = 2
CBM_ERR_AGENT_OVERFLOW = 3
CBM_ERR_NEIGHBOR_OVERFLOW = 4
CBM_ERR_TIMEOUT = 5
CBM_ERR_STATE = 6
CBM_ERR_NOMEM = 7
ERR_NAMES = {1: "CBM_ERR_ARG", 2: "CBM_ERR_CUDA", 3: "CBM_ERR_AGENT_OVERFLOW",
             4: "CBM_ERR_NEIGHBOR_OVERFLOW", 5: "CBM_ERR_TIMEOUT", 6: "CBM_ERR_STATE",
             7: "CBM_ERR_NOMEM"}

F32, F64 = 0, 1
NEIGH_NONE, NEIGH_FULL, NEIGH_CELL_LINKED, NEIGH_VERLET_DISPLACEMENT, NEIGH_CLVD = 0, 1, 2, 3, 4
INT_EULER, INT_EM, INT_HEUN, INT_RK4, INT_EULER_HEUN = 0, 1, 2, 3, 4
FORCE_DIRECT, FORCE_LAGGED = 0, 1
ATT_FROM_REP, ATT_TO_ATT = 0, 1
WALLS_NONE, WALLS_REFLECT, WALLS_PUSH = 0, 1, 2
FATE_NONE, FATE_VOLUME, FATE_ID_PARITY = 0, 1, 2
MEDIUM_NEAREST, MEDIUM_BILINEAR = 0, 1
SYNC, NO_GRAPH = 1, 2
VIEW_COMMITTED, VIEW_NEW = 0, 1
STAGES = ("agent_rule", "agent_de", "medium_rule", "medium_de", "update", "neighbors")


class CbmConfig(C.Structure):
    _fields_ = [
        ("dims", C.c_int32), ("precision", C.c_int32), ("n_max", C.c_int64),
        ("box_lo", C.c_double * 3), ("box_hi", C.c_double * 3), ("dt", C.c_double),
        ("seed", C.c_uint64), ("community", C.c_uint32), ("neighbors", C.c_int32),
        ("n_max_neighbors", C.c_int32), ("integrator", C.c_int32),
        ("cell_edge", C.c_double), ("skin", C.c_double), ("rebuild_threshold", C.c_double),
        ("sigma", C.c_double), ("force_mode", C.c_int32), ("att_form", C.c_int32),
        ("k_rep", C.c_double), ("r_rep", C.c_double), ("k_att", C.c_double),
        ("r_att", C.c_double), ("walls", C.c_int32), ("fate", C.c_int32),
        ("wall_force", C.c_double), ("wall_range", C.c_double), ("drift_linear", C.c_double),
        ("growth", C.c_int32), ("medium", C.c_int32), ("v_div", C.c_double),
        ("div_sep", C.c_double), ("p_death", C.c_double), ("n_medium", C.c_int32 * 3),
        ("medium_sampling", C.c_int32), ("diff_D", C.c_double), ("decay", C.c_double),
        ("secretion", C.c_double), ("chemotaxis", C.c_double), ("uptake", C.c_double),
    ]


class CbmStateView(C.Structure):
    _fields_ = [
        ("N", C.c_int64), ("capacity", C.c_int64), ("t", C.c_double), ("step", C.c_int64),
        ("id_max", C.c_int64), ("pos", C.c_void_p * 3), ("v", C.c_void_p), ("g", C.c_void_p),
        ("f", C.c_void_p * 3), ("id", C.POINTER(C.c_int64)), ("parent", C.POINTER(C.c_int64)),
        ("medium_c", C.c_void_p), ("medium_grad", C.c_void_p * 3),
    ]


def make_config(**kw):
    """cbm_config with the reference's defaults; keyword names are the C field names."""
    cfg = CbmConfig()
    defaults = dict(dims=3, precision=F64, n_max=0, box_lo=(0.0, 0.0, 0.0),
                    box_hi=(1.0, 1.0, 1.0), dt=1.0, seed=0, community=0,
                    neighbors=NEIGH_NONE, n_max_neighbors=32, integrator=INT_EULER,
                    cell_edge=1.0, skin=1.0, rebuild_threshold=0.0, sigma=0.0,
                    force_mode=FORCE_DIRECT, att_form=ATT_FROM_REP, k_rep=0.0, r_rep=0.0,
                    k_att=0.0, r_att=0.0, walls=WALLS_NONE, fate=FATE_NONE, wall_force=0.0,
                    wall_range=0.0, drift_linear=0.0, growth=0, medium=0, v_div=0.0,
                    div_sep=0.0, p_death=0.0, n_medium=(1, 1, 1),
                    medium_sampling=MEDIUM_NEAREST, diff_D=0.0, decay=0.0, secretion=0.0,
                    chemotaxis=0.0, uptake=0.0)
    unknown = set(kw) - set(defaults)
    if unknown:
        raise TypeError(f"unknown cbm_config fields: {sorted(unknown)}")
    defaults.update(kw)
    for name, val in defaults.items():
        if name in ("box_lo", "box_hi"):
            v = list(val) + [0.0] * (3 - len(val))
            setattr(cfg, name, (C.c_double * 3)(*v[:3]))
        elif name == "n_medium":
            v = list(val) + [1] * (3 - len(val))
            setattr(cfg, name, (C.c_int32 * 3)(*v[:3]))
        else:
            setattr(cfg, name, val)
    return cfg


def real_dtype(cfg):
    return np.float64 if cfg.precision == F64 else np.float32


class CbmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load_library(path=LIB_PATH):
    """Loads libcbm_b200.so once.  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with build.py (nvcc, sm_100a)")
    lib = C.CDLL(path)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    sig = {
        "cbm_version": (C.c_char_p, []),
        "cbm_last_error": (C.c_char_p, [vp]),
        "cbm_create": (C.c_int, [C.POINTER(vp), C.POINTER(CbmConfig)]),
        "cbm_destroy": (None, [vp]),
        "cbm_upload": (C.c_int, [vp, C.POINTER(CbmStateView)]),
        "cbm_download": (C.c_int, [vp, C.POINTER(CbmStateView), i32]),
        "cbm_step": (C.c_int, [vp, i32, i32]),
        "cbm_step_noise": (C.c_int, [vp, vp, i32]),
        "cbm_agent_step_rule": (C.c_int, [vp]),
        "cbm_agent_step_de": (C.c_int, [vp]),
        "cbm_medium_step_rule": (C.c_int, [vp]),
        "cbm_medium_step_de": (C.c_int, [vp]),
        "cbm_update": (C.c_int, [vp]),
        "cbm_compute_neighbors": (C.c_int, [vp]),
        "cbm_sync": (C.c_int, [vp]),
        "cbm_get_counters": (C.c_int, [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64),
                                       C.POINTER(i64), C.POINTER(i32), C.POINTER(i64)]),
        "cbm_grid_shape": (C.c_int, [vp, C.POINTER(i32)]),
        "cbm_get_grid": (C.c_int, [vp, vp, vp, vp, vp]),
        "cbm_get_neighbors": (C.c_int, [vp, vp, vp, i64]),
        "cbm_count_neighbors": (C.c_int, [vp, dbl, vp]),
        "cbm_rng_fill": (C.c_int, [vp, i32, dbl, dbl, i64, i64, vp]),
        "cbm_stream": (vp, [vp]),
        "cbm_kernels_per_step": (C.c_int, [vp]),
        "cbm_profile_step": (C.c_int, [vp, i32, C.POINTER(C.c_float), C.POINTER(C.c_char_p),
                                       C.POINTER(i32)]),
        "cbm_set_kernel_timing": (C.c_int, [vp, i32]),
        "cbm_kernel_times": (C.c_int, [vp, i32, C.POINTER(C.c_float), C.POINTER(C.c_char_p),
                                       C.POINTER(i32)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a):
    return None if a is None else a.ctypes.data


class StateBuffers:
    """Host arrays of one Community plus the cbm_state_view pointing at them."""

    AGENT_REAL = ("x", "y", "z", "v", "g", "fx", "fy", "fz")
    MEDIUM = ("c", "gx", "gy", "gz")

    def __init__(self, cfg, capacity, n_nodes):
        dt = real_dtype(cfg)
        self.cfg = cfg
        self.capacity = capacity
        self.arrays = {k: np.zeros(capacity, dt) for k in self.AGENT_REAL}
        self.arrays["id"] = np.zeros(capacity, np.int64)
        self.arrays["parent"] = np.zeros(capacity, np.int64)
        for k in self.MEDIUM:
            self.arrays[k] = np.zeros(max(n_nodes, 1), dt)
        self.n_nodes = n_nodes

    def view(self, N=0, t=0.0, step=0, id_max=0, fields=None):
        a = self.arrays
        d = self.cfg.dims
        use = set(fields) if fields is not None else None

        def sel(k):
            return a[k] if (use is None or k in use) else None

        s = CbmStateView()
        s.N, s.capacity, s.t, s.step, s.id_max = N, self.capacity, t, step, id_max
        for i, k in enumerate(("x", "y", "z")):
            s.pos[i] = _ptr(sel(k)) if i < d else None
        s.v = _ptr(sel("v"))
        s.g = _ptr(sel("g"))
        for i, k in enumerate(("fx", "fy", "fz")):
            s.f[i] = _ptr(sel(k)) if i < d else None
        s.id = a["id"].ctypes.data_as(C.POINTER(C.c_int64)) if sel("id") is not None else None
        s.parent = (a["parent"].ctypes.data_as(C.POINTER(C.c_int64))
                    if sel("parent") is not None else None)
        if self.n_nodes:
            s.medium_c = _ptr(sel("c"))
            for i, k in enumerate(("gx", "gy", "gz")):
                s.medium_grad[i] = _ptr(sel(k)) if i < d else None
        return s


def state_from_dict(cfg, state, capacity=None, n_nodes=0):
    """Packs a dict of arrays (x, y, z, v, g, fx.., id, parent, c, gx..) into buffers."""
    N = int(state.get("N", len(state["x"])))
    cap = max(capacity or 0, N, 1)
    buf = StateBuffers(cfg, cap, n_nodes)
    present = []
    for k, arr in state.items():
        if k in buf.arrays and arr is not None:
            arr = np.asarray(arr)
            dst = buf.arrays[k]
            n = N if k not in StateBuffers.MEDIUM else n_nodes
            dst[:n] = arr[:n]
            present.append(k)
    return buf, N, present


class Context:
    """One cbm_ctx: a Community loaded on the B200 platform."""

    def __init__(self, cfg):
        self.lib = load_library()
        self.cfg = cfg
        h = C.c_void_p()
        rc = self.lib.cbm_create(C.byref(h), C.byref(cfg))
        if rc != CBM_OK:
            raise CbmError(rc, self.lib.cbm_last_error(None).decode())
        self.h = h
        self.n_nodes = int(np.prod([cfg.n_medium[d] for d in range(cfg.dims)])) if cfg.medium else 0

    def _check(self, rc):
        if rc != CBM_OK:
            raise CbmError(rc, self.lib.cbm_last_error(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.cbm_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, state, t=0.0, step=0, id_max=0):
        buf, N, present = state_from_dict(self.cfg, state, n_nodes=self.n_nodes)
        fields = present + [k for k in ("x", "y", "z") if k in present]
        view = buf.view(N=N, t=t, step=step, id_max=id_max, fields=fields)
        self._check(self.lib.cbm_upload(self.h, C.byref(view)))

    def download(self, which=VIEW_COMMITTED, capacity=None):
        cap = capacity or max(int(self.cfg.n_max), 1)
        buf = StateBuffers(self.cfg, cap, self.n_nodes)
        view = buf.view()
        self._check(self.lib.cbm_download(self.h, C.byref(view), which))
        N = view.N
        out = {k: v[:N].copy() for k, v in buf.arrays.items() if k not in StateBuffers.MEDIUM}
        if self.n_nodes:
            for k in StateBuffers.MEDIUM:
                out[k] = buf.arrays[k][: self.n_nodes].copy()
        out.update(N=N, t=view.t, step=view.step, id_max=view.id_max)
        return out

    def step(self, n=1, flags=SYNC):
        return self._check(self.lib.cbm_step(self.h, n, flags))

    def step_noise(self, noise, flags=SYNC):
        """One step whose EM increments are `noise` (N x dims, index order)."""
        dt = np.float64 if self.cfg.precision == F64 else np.float32
        buf = np.ascontiguousarray(noise, dtype=dt)
        return self._check(self.lib.cbm_step_noise(self.h, buf.ctypes.data, flags))

    def stage(self, name):
        fn = {"agent_rule": self.lib.cbm_agent_step_rule, "agent_de": self.lib.cbm_agent_step_de,
              "medium_rule": self.lib.cbm_medium_step_rule, "medium_de": self.lib.cbm_medium_step_de,
              "update": self.lib.cbm_update, "neighbors": self.lib.cbm_compute_neighbors}[name]
        return self._check(fn(self.h))

    def sync(self):
        return self._check(self.lib.cbm_sync(self.h))

    def counters(self):
        v = [C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32(), C.c_int64()]
        self._check(self.lib.cbm_get_counters(self.h, *[C.byref(x) for x in v]))
        return dict(N=v[0].value, n_add=v[1].value, n_remove=v[2].value, id_max=v[3].value,
                    flag=v[4].value, step=v[5].value)

    def grid(self):
        n3 = (C.c_int32 * 3)()
        self._check(self.lib.cbm_grid_shape(self.h, n3))
        nc = int(n3[0]) * int(n3[1]) * int(n3[2])
        N = self.counters()["N"]
        agent_cell = np.zeros(max(N, 1), np.int32)
        agent_list = np.zeros(max(N, 1), np.int32)
        start = np.zeros(nc, np.int32)
        count = np.zeros(nc, np.int32)
        self._check(self.lib.cbm_get_grid(self.h, _ptr(agent_cell), _ptr(start), _ptr(count),
                                          _ptr(agent_list)))
        return dict(shape=tuple(int(v) for v in n3), agent_cell=agent_cell[:N], cell_start=start,
                    cell_count=count, cell_agents=agent_list[:N])

    def neighbors(self):
        N = self.counters()["N"]
        M = int(self.cfg.n_max_neighbors)
        counts = np.zeros(max(N, 1), np.int32)
        lst = np.zeros(max(N * M, 1), np.int32)
        self._check(self.lib.cbm_get_neighbors(self.h, _ptr(counts), _ptr(lst), lst.size))
        return counts[:N], lst[: N * M].reshape(N, M)

    def count_neighbors(self, radius):
        N = self.counters()["N"]
        out = np.zeros(max(N, 1), np.int32)
        self._check(self.lib.cbm_count_neighbors(self.h, float(radius), _ptr(out)))
        return out[:N]

    def rng_fill(self, kind, a, b, n, step=0):
        out = np.zeros(max(n, 1), real_dtype(self.cfg))
        self._check(self.lib.cbm_rng_fill(self.h, kind, float(a), float(b), n, step, _ptr(out)))
        return out[:n]

    def stream(self):
        return self.lib.cbm_stream(self.h)

    def kernels_per_step(self):
        return self.lib.cbm_kernels_per_step(self.h)

    def profile_step(self):
        """One eager step with per-kernel event timing: [(kernel name, ms)]."""
        ms = (C.c_float * 64)()
        names = (C.c_char_p * 64)()
        n = C.c_int32()
        self._check(self.lib.cbm_profile_step(self.h, 64, ms, names, C.byref(n)))
        return [(names[i].decode(), ms[i]) for i in range(min(n.value, 64))]

    def set_kernel_timing(self, on=True):
        """Event records around every kernel inside the step graphs (on), or none."""
        self._check(self.lib.cbm_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_times(self):
        """[(kernel name, ms)] of the last graph-replayed step (kernel timing on)."""
        ms = (C.c_float * 64)()
        names = (C.c_char_p * 64)()
        n = C.c_int32()
        self._check(self.lib.cbm_kernel_times(self.h, 64, ms, names, C.byref(n)))
        return [(names[i].decode(), ms[i]) for i in range(min(n.value, 64))]


# ---- batched communities (cbm_batch_*) --------------------------------------
class CbmCommunityDesc(C.Structure):
    _fields_ = [("n", C.c_int64), ("box_lo", C.c_double * 3), ("box_hi", C.c_double * 3),
                ("k_rep", C.c_double), ("r_rep", C.c_double), ("k_att", C.c_double),
                ("r_att", C.c_double), ("sigma", C.c_double), ("community", C.c_uint32),
                ("pad", C.c_int32)]


class CbmBatchTuning(C.Structure):
    _fields_ = [("threads", C.c_int32), ("ctas_per_sm", C.c_int32), ("skin", C.c_double),
                ("rebuild_threshold", C.c_double), ("tile_agents", C.c_int32),
                ("lanes_per_agent", C.c_int32)]

    def as_dict(self):
        return dict(threads=self.threads, ctas_per_sm=self.ctas_per_sm, skin=self.skin,
                    rebuild_threshold=self.rebuild_threshold, tile_agents=self.tile_agents,
                    lanes_per_agent=max(self.lanes_per_agent, 1))


def _bind_batch(lib):
    if getattr(lib, "_batch_bound", False):
        return
    vp, i32 = C.c_void_p, C.c_int32
    sig = {
        "cbm_batch_create": (C.c_int, [C.POINTER(vp), C.POINTER(CbmConfig), i32,
                                       C.POINTER(CbmCommunityDesc)]),
        "cbm_batch_destroy": (None, [vp]),
        "cbm_batch_last_error": (C.c_char_p, [vp]),
        "cbm_batch_upload": (C.c_int, [vp, i32, C.POINTER(CbmStateView)]),
        "cbm_batch_download": (C.c_int, [vp, i32, C.POINTER(CbmStateView)]),
        "cbm_batch_step": (C.c_int, [vp, i32, i32]),
        "cbm_batch_set_tuning": (C.c_int, [vp, C.POINTER(CbmBatchTuning)]),
        "cbm_batch_get_tuning": (C.c_int, [vp, C.POINTER(CbmBatchTuning)]),
        "cbm_batch_autotune": (C.c_int, [vp, i32, C.POINTER(CbmBatchTuning)]),
        "cbm_batch_stream": (vp, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib._batch_bound = True


class Batch:
    """Many independent 3D communities advanced by one persistent launch."""

    def __init__(self, base_cfg, descs):
        self.lib = load_library()
        _bind_batch(self.lib)
        arr = (CbmCommunityDesc * len(descs))(*descs)
        h = C.c_void_p()
        rc = self.lib.cbm_batch_create(C.byref(h), C.byref(base_cfg), len(descs), arr)
        if rc != CBM_OK:
            raise CbmError(rc, self.lib.cbm_batch_last_error(None).decode())
        self.h = h
        self.cfg = base_cfg
        self.sizes = [int(d.n) for d in descs]

    def _check(self, rc):
        if rc != CBM_OK:
            raise CbmError(rc, self.lib.cbm_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.cbm_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, c, x, y, z, step=0):
        x, y, z = (np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, z))
        s = CbmStateView()
        s.N, s.capacity, s.step = len(x), len(x), step
        s.pos[0], s.pos[1], s.pos[2] = x.ctypes.data, y.ctypes.data, z.ctypes.data
        self._check(self.lib.cbm_batch_upload(self.h, c, C.byref(s)))

    def download(self, c):
        n = self.sizes[c]
        out = {k: np.zeros(max(n, 1), np.float32) for k in "xyz"}
        s = CbmStateView()
        s.capacity = n
        s.pos[0], s.pos[1], s.pos[2] = (out[k].ctypes.data for k in "xyz")
        self._check(self.lib.cbm_batch_download(self.h, c, C.byref(s)))
        return {k: v[:n] for k, v in out.items()} | {"step": s.step, "N": n}

    def step(self, n, flags=SYNC):
        self._check(self.lib.cbm_batch_step(self.h, n, flags))

    def tuning(self):
        t = CbmBatchTuning()
        self._check(self.lib.cbm_batch_get_tuning(self.h, C.byref(t)))
        return t

    def set_tuning(self, threads, ctas_per_sm, skin, rebuild_threshold=0.0, tile_agents=0,
                   lanes_per_agent=1):
        t = CbmBatchTuning(threads, ctas_per_sm, skin, rebuild_threshold, tile_agents,
                           lanes_per_agent)
        self._check(self.lib.cbm_batch_set_tuning(self.h, C.byref(t)))

    def autotune(self, trial_steps=20):
        t = CbmBatchTuning()
        self._check(self.lib.cbm_batch_autotune(self.h, trial_steps, C.byref(t)))
        return t

    def stream(self):
        return self.lib.cbm_batch_stream(self.h)


# ---- adjoint (cbm_adjoint_*) --------------------------------------------------
# ---- implicit medium (cbm_medium_*, DGADI) ----------------------------------
MEDIUM_MAX_FIELDS = 8


class CbmMediumConfig(C.Structure):
    _fields_ = [("dims", C.c_int32), ("precision", C.c_int32), ("n", C.c_int32 * 3),
                ("n_fields", C.c_int32), ("box_lo", C.c_double * 3), ("box_hi", C.c_double * 3),
                ("dt", C.c_double), ("diffusion", C.c_double * MEDIUM_MAX_FIELDS),
                ("decay", C.c_double * MEDIUM_MAX_FIELDS), ("c_max", C.c_double)]


def make_medium_config(dims, n, box_lo, box_hi, dt, diffusion, decay=None, c_max=0.0,
                       precision=F32):
    """A cbm_medium_config: `n` nodes per axis, one diffusion coefficient (and
    optional decay) per field."""
    k = CbmMediumConfig()
    k.dims, k.precision = dims, precision
    for d in range(3):
        k.n[d] = int(n[d]) if d < dims else 1
        k.box_lo[d] = float(box_lo[d]) if d < dims else 0.0
        k.box_hi[d] = float(box_hi[d]) if d < dims else 1.0
    k.n_fields = len(diffusion)
    k.dt, k.c_max = float(dt), float(c_max)
    for f, D in enumerate(diffusion):
        k.diffusion[f] = float(D)
        k.decay[f] = float(decay[f]) if decay is not None else 0.0
    return k


def _bind_medium(lib):
    if getattr(lib, "_medium_bound", False):
        return
    vp, i32 = C.c_void_p, C.c_int32
    sig = {
        "cbm_medium_create": (C.c_int, [C.POINTER(vp), C.POINTER(CbmMediumConfig)]),
        "cbm_medium_destroy": (None, [vp]),
        "cbm_medium_last_error": (C.c_char_p, [vp]),
        "cbm_medium_upload": (C.c_int, [vp, vp, vp]),
        "cbm_medium_step": (C.c_int, [vp, i32, i32]),
        "cbm_medium_download": (C.c_int, [vp, vp, C.POINTER(C.c_double)]),
        "cbm_medium_stream": (vp, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib._medium_bound = True


class DGADIMedium:
    """A medium advanced by the implicit Douglas–Gunn ADI step (DGADI).
    Fields are arrays of shape (n_fields, [n2, [n1,]] n0), x fastest."""

    def __init__(self, cfg):
        self.lib = load_library()
        _bind_medium(self.lib)
        h = C.c_void_p()
        rc = self.lib.cbm_medium_create(C.byref(h), C.byref(cfg))
        if rc != CBM_OK:
            raise CbmError(rc, self.lib.cbm_medium_last_error(None).decode())
        self.h = h
        self.cfg = cfg
        self.dtype = np.float64 if cfg.precision == F64 else np.float32
        self.shape = (cfg.n_fields,) + tuple(int(cfg.n[d]) for d in reversed(range(cfg.dims)))

    def _check(self, rc):
        if rc != CBM_OK:
            raise CbmError(rc, self.lib.cbm_medium_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.cbm_medium_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, fields, source=None):
        f = np.ascontiguousarray(fields, dtype=self.dtype).reshape(self.shape)
        s = None if source is None else np.ascontiguousarray(source, dtype=self.dtype)
        self._check(self.lib.cbm_medium_upload(self.h, f.ctypes.data,
                                               None if s is None else s.ctypes.data))

    def step(self, n, flags=SYNC):
        self._check(self.lib.cbm_medium_step(self.h, n, flags))

    def download(self):
        out = np.zeros(self.shape, self.dtype)
        t = C.c_double()
        self._check(self.lib.cbm_medium_download(self.h, out.ctypes.data, C.byref(t)))
        return out, t.value

    def stream(self):
        return self.lib.cbm_medium_stream(self.h)


ROD_FIELDS = ("x", "y", "vx", "vy", "theta", "omega", "d", "l", "m", "fx", "fy", "W",
              "pressure", "l_target")


class CbmRodsConfig(C.Structure):
    _fields_ = [("precision", C.c_int32), ("neighbors", C.c_int32), ("n_max", C.c_int64),
                ("box_lo", C.c_double * 2), ("box_hi", C.c_double * 2), ("cell_edge", C.c_double),
                ("dt", C.c_double), ("kn", C.c_double), ("gamma_n", C.c_double),
                ("gamma_t", C.c_double), ("mu_cc", C.c_double), ("mu_cw", C.c_double),
                ("beta", C.c_double), ("beta_w", C.c_double), ("growth_model", C.c_int32),
                ("pad0", C.c_int32), ("growth", C.c_double), ("alpha", C.c_double),
                ("sigma_l_target", C.c_double), ("l_max", C.c_double), ("seed", C.c_uint64)]


def make_rods_config(n_max, box_lo, box_hi, dt, kn, gamma_n, gamma_t, mu_cc, beta, beta_w,
                     mu_cw=0.0, cell_edge=0.0, neighbors=NEIGH_CELL_LINKED, precision=F64,
                     growth=None, alpha=0.0, sigma_l_target=0.0, l_max=0.0, seed=0):
    """A cbm_rods_config: the model parameters of rods2D (kn, γn, γt, μcc, μcw,
    β, βω), its simBox and the CellLinked cell edge; with `growth` given, the
    rods2dGrowth model (growth, α, σlTarget, lMax) and the seed of its draws."""
    k = CbmRodsConfig()
    if growth is not None:
        k.growth_model, k.growth, k.alpha = 1, float(growth), float(alpha)
        k.sigma_l_target, k.l_max, k.seed = float(sigma_l_target), float(l_max), int(seed)
    k.precision, k.neighbors, k.n_max = precision, neighbors, int(n_max)
    for d in range(2):
        k.box_lo[d], k.box_hi[d] = float(box_lo[d]), float(box_hi[d])
    k.cell_edge, k.dt = float(cell_edge), float(dt)
    k.kn, k.gamma_n, k.gamma_t = float(kn), float(gamma_n), float(gamma_t)
    k.mu_cc, k.mu_cw, k.beta, k.beta_w = float(mu_cc), float(mu_cw), float(beta), float(beta_w)
    return k


class Rods2D:
    """The rods2D / rods2dGrowth model (src/models/rods.jl) stepped with Euler
    on the device.  State is a dict of ROD_FIELDS arrays; pressure is output
    only and l_target is used by rods2dGrowth only."""

    def __init__(self, cfg):
        self.lib = load_library()
        lib = self.lib
        if not getattr(lib, "_rods_bound", False):
            vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
            for name, res, args in (
                    ("cbm_rods_create", C.c_int, [C.POINTER(vp), C.POINTER(CbmRodsConfig)]),
                    ("cbm_rods_destroy", None, [vp]),
                    ("cbm_rods_last_error", C.c_char_p, [vp]),
                    ("cbm_rods_upload", C.c_int, [vp, i64, C.POINTER(vp)]),
                    ("cbm_rods_step", C.c_int, [vp, i32, i32]),
                    ("cbm_rods_download", C.c_int, [vp, C.POINTER(vp), C.POINTER(i64)]),
                    ("cbm_rods_stream", vp, [vp])):
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            lib._rods_bound = True
        h = C.c_void_p()
        rc = lib.cbm_rods_create(C.byref(h), C.byref(cfg))
        if rc != CBM_OK:
            raise CbmError(rc, lib.cbm_rods_last_error(None).decode())
        self.h = h
        self.cfg = cfg
        self.dtype = np.float64 if cfg.precision == F64 else np.float32
        self.n = 0

    def _check(self, rc):
        if rc != CBM_OK:
            raise CbmError(rc, self.lib.cbm_rods_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.cbm_rods_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, state):
        nf = len(ROD_FIELDS)
        arrs = [np.ascontiguousarray(state[k], dtype=self.dtype) for k in ROD_FIELDS[:12]]
        n = len(arrs[0]) if arrs else 0
        lt = state.get("l_target")
        lt = None if lt is None else np.ascontiguousarray(lt, dtype=self.dtype)
        ptrs = (C.c_void_p * nf)(*([a.ctypes.data for a in arrs]
                                   + [None, None if lt is None else lt.ctypes.data]))
        self._keep = arrs + [lt]
        self._check(self.lib.cbm_rods_upload(self.h, n, ptrs))
        self.n = n

    def step(self, n, flags=SYNC):
        self._check(self.lib.cbm_rods_step(self.h, n, flags))

    def download(self):
        nf = len(ROD_FIELDS)
        n = C.c_int64()
        none = (C.c_void_p * nf)()
        self._check(self.lib.cbm_rods_download(self.h, none, C.byref(n)))  # the count only
        self.n = int(n.value)
        out = np.zeros((nf, self.n), self.dtype)
        ptrs = (C.c_void_p * nf)(*[out[q].ctypes.data for q in range(nf)])
        self._check(self.lib.cbm_rods_download(self.h, ptrs, C.byref(n)))
        return {k: out[q] for q, k in enumerate(ROD_FIELDS)}

    def stream(self):
        return self.lib.cbm_rods_stream(self.h)


class Adjoint:
    """Gradients of mean((x_T - target)^2) w.r.t. (k_rep, k_att, r_rep) and x0."""

    def __init__(self, cfg):
        self.lib = load_library()
        lib = self.lib
        if not getattr(lib, "_adj_bound", False):
            vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
            for name, res, args in (
                    ("cbm_adjoint_create", C.c_int, [C.POINTER(vp), C.POINTER(CbmConfig)]),
                    ("cbm_adjoint_destroy", None, [vp]),
                    ("cbm_adjoint_last_error", C.c_char_p, [vp]),
                    ("cbm_adjoint_run", C.c_int, [vp, i64, C.POINTER(vp), i32, i32, C.POINTER(vp),
                                                  C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                  C.POINTER(vp), C.POINTER(vp)]),
                    ("cbm_adjoint_forward", C.c_int, [vp, i64, C.POINTER(vp), i32, C.POINTER(vp)]),
                    ("cbm_adjoint_stream", vp, [vp])):
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            lib._adj_bound = True
        h = C.c_void_p()
        rc = lib.cbm_adjoint_create(C.byref(h), C.byref(cfg))
        if rc != CBM_OK:
            raise CbmError(rc, lib.cbm_adjoint_last_error(None).decode())
        self.h = h
        self.cfg = cfg
        self.dtype = real_dtype(cfg)

    def close(self):
        if getattr(self, "h", None):
            self.lib.cbm_adjoint_destroy(self.h)
            self.h = None

    __del__ = close

    def _arrs(self, xyz):
        arrs = [np.ascontiguousarray(a, dtype=self.dtype) for a in xyz]
        return arrs, (C.c_void_p * 3)(*[a.ctypes.data for a in arrs])

    def run(self, x0, target, nsteps, checkpoint_every=20, want_dx0=True):
        n = len(x0[0])
        xs, xp = self._arrs(x0)
        ts, tp = self._arrs(target)
        dx = [np.zeros(n, self.dtype) for _ in range(3)]
        xT = [np.zeros(n, self.dtype) for _ in range(3)]
        dxp = (C.c_void_p * 3)(*[a.ctypes.data for a in dx]) if want_dx0 else None
        xTp = (C.c_void_p * 3)(*[a.ctypes.data for a in xT])
        loss = C.c_double()
        g = (C.c_double * 3)()
        rc = self.lib.cbm_adjoint_run(self.h, n, xp, nsteps, checkpoint_every, tp, C.byref(loss), g,
                                      dxp, xTp)
        if rc != CBM_OK:
            raise CbmError(rc, self.lib.cbm_adjoint_last_error(self.h).decode())
        return dict(loss=loss.value, dtheta=np.array(list(g)), dx0=dx if want_dx0 else None, xT=xT)

    def forward(self, x0, nsteps):
        n = len(x0[0])
        xs, xp = self._arrs(x0)
        xT = [np.zeros(n, self.dtype) for _ in range(3)]
        xTp = (C.c_void_p * 3)(*[a.ctypes.data for a in xT])
        rc = self.lib.cbm_adjoint_forward(self.h, n, xp, nsteps, xTp)
        if rc != CBM_OK:
            raise CbmError(rc, self.lib.cbm_adjoint_last_error(self.h).decode())
        return xT

    def stream(self):
        return self.lib.cbm_adjoint_stream(self.h)
