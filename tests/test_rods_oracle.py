"""The checker's rods2D restatement against a plain-Python transcription of the
reference's rod model, statement by statement:
rodForces (src/models/rods.jl:21-59), the rods2D agentODE (rods.jl:86-118)
and CBMMetrics' geometry (src/metrics.jl:137-246).

The reference ships no rod tests or fixtures, so this transcription is the pin.
The transcription follows the Julia text with this build's definitions:
cos and sin come from the shared series on theta / (2 pi) reduced to [0, 1),
and x^1.5 is x * sqrt(x).  Python floats are IEEE doubles and Python does no
contraction, so the Float64 comparisons are bit-exact.
"""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import cbm
from _oracle import OracleRods, load_oracle, oracle_rod_pair

abi = cbm._abi


def _sqrt(v):
    """sqrt in the operand's precision (np.float32 stays Float32)."""
    return np.sqrt(v) if isinstance(v, np.float32) else math.sqrt(v)


def _cossin(theta):
    lib = load_oracle(abi)
    if isinstance(theta, np.float32):
        w = theta * np.float32(0.15915494309189535)
        w = w - np.floor(w)
        if w >= 1:
            w = w - np.float32(1)
        c, s = C.c_float(), C.c_float()
        lib.oracle_cossin_f32(float(w), C.byref(c), C.byref(s))
        return np.float32(c.value), np.float32(s.value)
    w = theta * 0.15915494309189535
    w = w - math.floor(w)
    if w >= 1.0:
        w = w - 1.0
    c, s = C.c_double(), C.c_double()
    lib.oracle_cossin_f64(w, C.byref(c), C.byref(s))
    return c.value, s.value


def jl_min(a, b):
    if a != a or b != b:
        return a + b
    if a == b:
        return b if math.copysign(1.0, b) < 0 else a
    return b if b < a else a


def jl_max(a, b):
    if a != a or b != b:
        return a + b
    if a == b:
        return b if math.copysign(1.0, a) < 0 else a
    return b if b > a else a


# --- CBMMetrics (src/metrics.jl) ------------------------------------------------
def intersection2lines(x1, y1, t1, x2, y2, t2):
    c1, s1 = _cossin(t1)
    c2, s2 = _cossin(t2)
    cx = x1 - x2
    cy = y1 - y2
    norm = c1 * s2 - s1 * c2
    if abs(norm) > 0.0000001:
        scale = (-s2 * cx + c2 * cy) / norm
        return scale * c1 + x1, scale * s1 + y1
    return (x1 + x2) / 2, (y1 + y2) / 2


def point2line(x1, y1, x2, y2, t2):
    c2, s2 = _cossin(t2)
    cx = x2 - x1
    cy = y2 - y1
    return (s2 * cx - c2 * cy) * s2 + x1, -(s2 * cx - c2 * cy) * c2 + y1


def point_inside_rod(x1, y1, l1, t1, px, py, sep):
    di = jl_max(_sqrt((x1 - px) * (x1 - px) + (y1 - py) * (y1 - py)), 0.00000001)
    dxi = (px - x1) / di
    dyi = (py - y1) / di
    return sep * jl_min(di, l1 / 2) * dxi + x1, sep * jl_min(di, l1 / 2) * dyi + y1


def rod_intersection(x1, y1, l1, t1, x2, y2, l2, t2, sep=0.99):
    x1a, y1a, x2a, y2a = x1, y1, x2, y2
    px, py = intersection2lines(x1, y1, t1, x2, y2, t2)
    di = _sqrt((x1 - px) * (x1 - px) + (y1 - py) * (y1 - py))
    dj = _sqrt((x2 - px) * (x2 - px) + (y2 - py) * (y2 - py))
    c1, s1 = _cossin(t1)
    c2, s2 = _cossin(t2)
    norm = c1 * s2 - s1 * c2
    if abs(norm) < 0.000001:
        x1a, y1a = point2line(px, py, x1, y1, t1)
        x1a, y1a = point_inside_rod(x1, y1, l1, t1, x1a, y1a, sep)
        x2a, y2a = point2line(px, py, x2, y2, t2)
        x2a, y2a = point_inside_rod(x2, y2, l2, t2, x2a, y2a, sep)
    elif di <= l1 / 2 and dj <= l2 / 2:
        x1a, y1a = point_inside_rod(x1, y1, l1, t1, px, py, sep)
        x2a, y2a = point_inside_rod(x2, y2, l2, t2, px, py, sep)
    elif di <= l1 / 2 and dj > l2 / 2:
        x2a, y2a = point_inside_rod(x2, y2, l2, t2, px, py, sep)
        x1a, y1a = point2line(x2a, y2a, x1, y1, t1)
    elif di > l1 / 2 and dj <= l2 / 2:
        x1a, y1a = point_inside_rod(x1, y1, l1, t1, px, py, sep)
        x2a, y2a = point2line(x1a, y1a, x2, y2, t2)
    else:
        x2a, y2a = point_inside_rod(x2, y2, l2, t2, px, py, sep)
        x1a, y1a = point2line(x2a, y2a, x1, y1, t1)
        dj = _sqrt((x1 - x1a) * (x1 - x1a) + (y1 - y1a) * (y1 - y1a))
        if dj > l1 / 2:
            x1a, y1a = point_inside_rod(x1, y1, l1, t1, px, py, sep)
            x2b, y2b = point2line(x1a, y1a, x2, y2, t2)
            dj = _sqrt((x2 - x2b) * (x2 - x2b) + (y2 - y2b) * (y2 - y2b))
            if dj < l2 / 2:
                x2a, y2a = x2b, y2b
    return x1a, y1a, x2a, y2a


# --- rodForces (src/models/rods.jl:21-59) ----------------------------------------
def rod_forces(x, y, d, l, th, vx, vy, m, x2, y2, d2, l2, th2, vx2, vy2, kn, gn, gt, mucc,
               pow15=lambda v: v * _sqrt(v)):
    fx = fy = w = 0.0
    xi, yi, xj, yj = rod_intersection(x, y, l, th, x2, y2, l2, th2)
    rij = _sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj))
    if rij > 0.0 and rij < (d + d2) / 2:
        delta = d - rij
        me = m / 2
        nx = (xi - xj) / rij
        ny = (yi - yj) / rij
        vijx = vx - vx2
        vijy = vy - vy2
        vn = nx * vijx + ny * vijy
        fn = kn * pow15(delta) - gn * me * delta * vn
        ft = -jl_min(gt * me * _sqrt(delta), mucc * fn)
        fx = fn * nx + ft * (vijx - vn * nx)
        fy = fn * ny + ft * (vijy - vn * ny)
        w = (xi - x) * fy - (yi - y) * fx
    return fx, fy, w, (xi, yi, xj, yj)


K = dict(kn=2.0e6, gn=100.0, gt=20.0, mucc=0.1)


def _pairs(seed, n):
    """Pairs of rods at contact range in all the geometric cases: crossing,
    T-shaped, end to end, side by side, exactly and nearly parallel."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        d, l = rng.uniform(0.8, 1.2), rng.uniform(1.0, 4.0)
        # d2 <= d: with d2 > d a contact can have delta = d - rij < 0, where
        # Julia's delta^1.5 raises a DomainError
        d2, l2 = rng.uniform(0.8, 1.0) * d, rng.uniform(1.0, 4.0)
        th = rng.uniform(-7.0, 7.0)
        kind = q % 5
        if kind == 3:
            th2 = th
        elif kind == 4:
            th2 = th + rng.uniform(-1e-6, 1e-6)
        else:
            th2 = rng.uniform(-7.0, 7.0)
        r = rng.uniform(0.0, (l + l2) / 2 + 1.0)
        phi = rng.uniform(0, 2 * math.pi)
        a = [0.3, -0.2, d, l, th, rng.normal(), rng.normal(), rng.uniform(0.5, 2.0)]
        b = [0.3 + r * math.cos(phi), -0.2 + r * math.sin(phi), d2, l2, th2, rng.normal(),
             rng.normal(), rng.uniform(0.5, 2.0)]
        out.append((a, b))
    return out


def test_rod_pair_matches_transcription():
    k = [K["kn"], K["gn"], K["gt"], K["mucc"]]
    contacts = 0
    for a, b in _pairs(7, 600):
        hit, got = oracle_rod_pair(abi, a, b, k)
        fx, fy, w, pts = rod_forces(*a, *b[:7], **K)
        assert list(got[3:]) == list(pts), (a, b)
        assert (got[0], got[1], got[2]) == (fx, fy, w), (a, b)
        contacts += hit
    assert contacts > 100  # the cases reach contact


def test_pow15_definition_close_to_julia_pow():
    """x^1.5 as x*sqrt(x) differs from a correctly rounded pow by an ulp or so."""
    for a, b in _pairs(8, 300):
        f1 = rod_forces(*a, *b[:7], **K)
        f2 = rod_forces(*a, *b[:7], **K, pow15=lambda v: v ** 1.5)
        for u, v in zip(f1[:3], f2[:3]):
            assert u == pytest.approx(v, rel=1e-12, abs=1e-9)


def _colony(n, seed, box=12.0):
    rng = np.random.default_rng(seed)
    st = {k: np.zeros(n) for k in abi.ROD_FIELDS}
    st["x"] = rng.uniform(-box, box, n)
    st["y"] = rng.uniform(-box, box, n)
    st["vx"] = rng.normal(0, 0.1, n)
    st["vy"] = rng.normal(0, 0.1, n)
    st["theta"] = rng.uniform(-math.pi, math.pi, n)
    st["omega"] = rng.normal(0, 0.1, n)
    st["d"] = np.full(n, 1.0)
    st["l"] = rng.uniform(1.0, 3.0, n)
    st["m"] = rng.uniform(0.8, 1.2, n)
    return st


PARAMS = dict(dt=1e-4, kn=2.0e6, gamma_n=100.0, gamma_t=20.0, mu_cc=0.1, beta=0.8, beta_w=0.8)
BOX_LO, BOX_HI = (-14.0, -14.0), (14.0, 14.0)


def _cell_of(x, lo, hi, edge, n):
    # cellPos (src/neighbors.jl:636-638), 0-based, with Julia's float ÷
    if x > hi:
        return n - 1
    if not (x >= lo):
        return 0
    a = x - lo
    p = int(round((a - math.fmod(a, edge)) / edge)) + 1
    return min(p, n - 1)


def _py_step(st, neighbors, edge):
    """One step!: agentStepDE! (Euler over rods2D's agentODE), update!,
    with neighbors walked as @loopOverNeighbors does."""
    n = len(st["x"])
    f = {k: list(np.asarray(v)) for k, v in st.items()}
    order = list(range(n))
    if neighbors == abi.NEIGH_CELL_LINKED:
        nc = [math.ceil((BOX_HI[d] - BOX_LO[d]) / edge + 2) for d in range(2)]
        cell = [_cell_of(f["x"][i], BOX_LO[0], BOX_HI[0], edge, nc[0])
                + nc[0] * _cell_of(f["y"][i], BOX_LO[1], BOX_HI[1], edge, nc[1]) for i in range(n)]
        members = {}
        for i in range(n):
            members.setdefault(cell[i], []).append(i)
    zero = f["x"][0] * 0 if n else 0.0
    new = {k: [zero] * n for k in ("fx", "fy", "W", "pressure")}
    for i in range(n):
        if neighbors == abi.NEIGH_FULL:
            cand = order
        else:
            cx, cy = cell[i] % nc[0], cell[i] // nc[0]
            cand = []
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    qx, qy = cx + dx, cy + dy
                    if 0 <= qx < nc[0] and 0 <= qy < nc[1]:
                        cand += members.get(qx + nc[0] * qy, [])
        fx = fy = w = p = zero
        for j in cand:
            if j == i:
                continue
            a, b, c, _ = rod_forces(f["x"][i], f["y"][i], f["d"][i], f["l"][i], f["theta"][i],
                                    f["vx"][i], f["vy"][i], f["m"][i], f["x"][j], f["y"][j],
                                    f["d"][j], f["l"][j], f["theta"][j], f["vx"][j], f["vy"][j],
                                    PARAMS["kn"], PARAMS["gamma_n"], PARAMS["gamma_t"],
                                    PARAMS["mu_cc"])
            fx += a
            fy += b
            w += c
            p += _sqrt(a * a + b * b)
        new["fx"][i], new["fy"][i], new["W"][i], new["pressure"][i] = fx, fy, w, p
    dt, beta, bw = PARAMS["dt"], PARAMS["beta"], PARAMS["beta_w"]
    out = {k: list(v) for k, v in f.items()}
    for i in range(n):
        vx, vy, om = f["vx"][i], f["vy"][i], f["omega"][i]
        d, l, m = f["d"][i], f["l"][i], f["m"][i]
        out["x"][i] = f["x"][i] + vx * dt
        out["y"][i] = f["y"][i] + vy * dt
        out["vx"][i] = vx + (-beta * vx + f["fx"][i] / m) * dt
        out["vy"][i] = vy + (-beta * vy + f["fy"][i] / m) * dt
        out["theta"][i] = f["theta"][i] + om * dt
        out["omega"][i] = om + (f["W"][i] / (m * ((d + l) * (d + l)) / 12 + m * (d * d)) - bw * om) * dt
    for k in new:
        out[k] = new[k]
    return {k: np.array(v) for k, v in out.items()}


@pytest.mark.parametrize("neighbors", ["full", "cell_linked"])
def test_rods_step_f32_matches_transcription(neighbors):
    """The Float32 checker against the same transcription run on np.float32
    scalars: every operation and constant in Float32."""
    nb = abi.NEIGH_FULL if neighbors == "full" else abi.NEIGH_CELL_LINKED
    st = {k: v.astype(np.float32) for k, v in _colony(50, 4, box=5.0).items()}
    cfg = abi.make_rods_config(50, BOX_LO, BOX_HI, cell_edge=4.0, neighbors=nb,
                               precision=abi.F32, **PARAMS)
    orc = OracleRods(abi, cfg)
    orc.upload(st)
    ref = st
    for _ in range(3):
        ref = _py_step(ref, nb, 4.0)
        orc.step(1)
        got = orc.download()
        for k in abi.ROD_FIELDS[:13]:
            assert ref[k].dtype == np.float32, k
            np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert np.count_nonzero(ref["pressure"]) > 10


@pytest.mark.parametrize("neighbors", ["full", "cell_linked"])
def test_rods_step_matches_transcription(neighbors):
    nb = abi.NEIGH_FULL if neighbors == "full" else abi.NEIGH_CELL_LINKED
    edge = 4.0
    st = _colony(60, 3, box=6.0)
    cfg = abi.make_rods_config(60, BOX_LO, BOX_HI, cell_edge=edge, neighbors=nb,
                               precision=abi.F64, **PARAMS)
    orc = OracleRods(abi, cfg)
    orc.upload(st)
    ref = {k: np.asarray(v, dtype=float) for k, v in st.items()}
    for _ in range(3):
        ref = _py_step(ref, nb, edge)
        orc.step(1)
        got = orc.download()
        for k in abi.ROD_FIELDS:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert np.count_nonzero(ref["pressure"]) > 10  # rods are in contact



GROW = dict(growth=200.0, alpha=50.0, sigma_l_target=0.2, l_max=3.0, seed=77)


def _uniform(step, agent, stream, f32=False):
    lib = load_oracle(abi)
    if f32:
        return np.float32(lib.oracle_uniform_f32(GROW["seed"], step, agent, stream, 0))
    return lib.oracle_uniform_f64(GROW["seed"], step, agent, stream, 0)


def _py_grow_step(st, step, neighbors, edge, n_max):
    """One step! of rods2dGrowth (rods.jl:123-163), as the reference runs it:
    agentStepRule! (@addAgent at rows N + NAdd into the new copies, fields not
    given taken from the parent; @removeAgent), agentStepDE! (rods2D's ODE and
    dt(l) = growth/(1+α pressure), pressure committed), update! (holes filled
    from the surviving tail, update.jl:15-84) and the commit."""
    f32 = np.asarray(st["x"]).dtype == np.float32
    T = np.float32 if f32 else float
    f = {k: list(np.asarray(v)) for k, v in st.items()}
    n = len(f["x"])
    de = _py_step(st, neighbors, edge)  # rows < n: Euler and the neighbor sums
    g = {k: list(np.asarray(v)) for k, v in de.items()}
    for i in range(n):
        g["l"][i] = f["l"][i] + (T(GROW["growth"]) / (1 + T(GROW["alpha"]) * f["pressure"][i])) * \
            T(PARAMS["dt"])
    dividers = [i for i in range(n) if f["l"][i] > f["l_target"][i]]
    holes, survive = [], [True] * n_max
    lo = T(GROW["l_max"]) - T(GROW["sigma_l_target"])
    hi = T(GROW["l_max"]) + T(GROW["sigma_l_target"])
    for i in dividers:
        c, s = _cossin(f["theta"][i])
        ww = (T(0.1) - T(-0.1)) * _uniform(step, i, 5, f32) + T(-0.1)
        l, d = f["l"][i], f["d"][i]
        for h in (0, 1):
            if len(g["x"]) >= n_max:  # functionRule.jl:58-70: the birth is dropped
                continue
            for k in g:
                g[k].append(f[k][i])
            sg = (l + d) / 4 if h == 0 else -(l + d) / 4
            g["x"][-1] = sg * c + f["x"][i]
            g["y"][-1] = sg * s + f["y"][i]
            g["l"][-1] = (l - d) / 2
            g["omega"][-1] = f["omega"][i] + ww if h == 0 else f["omega"][i] - ww
            g["l_target"][-1] = (hi - lo) * _uniform(step, i, 6 + h, f32) + lo
        holes.append(i)  # @removeAgent runs whether or not the births fitted
        survive[i] = False
    repo, last = [], len(g["x"]) - 1
    while len(holes) > len(repo) and last >= 0:
        if survive[last]:
            repo.append(last)
        last -= 1
    for k in g:
        for hole, src in zip(holes, repo):
            if hole < src:
                g[k][hole] = g[k][src]
    n_new = len(g["x"]) - len(holes)
    return {k: np.array(v[:n_new]) for k, v in g.items()}


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("neighbors", ["full", "cell_linked"])
def test_rods_growth_step_matches_transcription(neighbors, prec):
    """rods2dGrowth: divisions in most steps, including rods that divide in
    the same step, against the transcription, field by field (in Float32 on
    np.float32 scalars)."""
    nb = abi.NEIGH_FULL if neighbors == "full" else abi.NEIGH_CELL_LINKED
    edge = 4.0
    st = _colony(24, 5, box=5.0)
    rng = np.random.default_rng(6)
    st["l_target"] = st["l"] + rng.uniform(-0.02, 0.06, 24)  # a third divide at once
    if prec == "f32":
        st = {k: v.astype(np.float32) for k, v in st.items()}
    cfg = abi.make_rods_config(200, BOX_LO, BOX_HI, cell_edge=edge, neighbors=nb,
                               precision=abi.F32 if prec == "f32" else abi.F64, **PARAMS, **GROW)
    orc = OracleRods(abi, cfg)
    orc.upload(st)
    ref = dict(st)
    sizes = []
    for step in range(6):
        ref = _py_grow_step(ref, step, nb, edge, 200)
        orc.step(1)
        got = orc.download()
        assert orc.count() == (len(ref["x"]), 0)
        for k in abi.ROD_FIELDS:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{k} after step {step}")
        sizes.append(len(ref["x"]))
        assert all(v.dtype == st["x"].dtype for v in ref.values())
    assert sizes[0] > 24 and sizes[-1] > sizes[0]


@pytest.mark.parametrize("n_max", [10, 11, 14, 17, 25, 30])
def test_rods_growth_overflow_matches_transcription(n_max):
    """Births beyond n_max are dropped in order and every parent is still
    removed; update! then also moves surviving old rows into the holes when
    fewer daughters than parents were born.  Capacities from no room at all
    to room for every birth."""
    st = _colony(10, 8, box=3.0)
    st["l_target"] = st["l"] + np.where(np.arange(10) % 3 == 1, 1.0, -0.5)  # 7 of 10 divide
    cfg = abi.make_rods_config(n_max, BOX_LO, BOX_HI, cell_edge=4.0, precision=abi.F64, **PARAMS,
                               **GROW)
    orc = OracleRods(abi, cfg)
    orc.upload(st)
    ref = _py_grow_step(dict(st), 0, abi.NEIGH_CELL_LINKED, 4.0, n_max)
    orc.step(1)
    got = orc.download()
    overflow = 10 + 2 * 7 > n_max
    assert orc.count() == (len(ref["x"]), abi.CBM_ERR_AGENT_OVERFLOW if overflow else 0)
    assert len(ref["x"]) == 10 + min(14, n_max - 10) - 7
    for k in abi.ROD_FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def _literal_rows(n, flags, n_max):
    """The reference's bookkeeping on labels: rows after @addAgent /
    @removeAgent and update!'s fill (update.jl:15-84)."""
    rows = [("old", i) for i in range(n)]
    survive = [True] * n_max
    holes, k = [], 0
    for i in range(n):
        if not flags[i]:
            continue
        for h in (0, 1):
            if len(rows) < n_max:
                rows.append(("new", k, h))
        holes.append(i)
        survive[i] = False
        k += 1
    repo, last = [], len(rows) - 1
    while len(holes) > len(repo) and last >= 0:
        if survive[last]:
            repo.append(last)
        last -= 1
    for hole, src in zip(holes, repo):
        if hole < src:
            rows[hole] = rows[src]
    return rows[:len(rows) - len(holes)]


def _device_rows(n, flags, n_max):
    """The closed form of k_rod_holes / k_rod_step / rod_divide
    (cellbasedmodels.jl_b200/csrc/cbm_rods.cu): every row written once, at
    its final index."""
    rank = [0] * (n + 1)
    for i in range(n):
        rank[i + 1] = rank[i] + flags[i]
    D = rank[n]
    A = min(2 * D, n_max - n)
    holes = [i for i in range(n) if flags[i]]
    out = [None] * (n + A - D)

    def put(row, label):
        assert 0 <= row < len(out) and out[row] is None, (row, label)
        out[row] = label

    for i in range(n):
        if flags[i]:
            k = rank[i]
            for h in (0, 1):
                e = 2 * k + h
                if e >= A:
                    continue
                s = n + e
                m = n + A - 1 - s
                put(holes[m] if m < D else s, ("new", k, h))
        else:
            dest = i
            if A < D:
                m = A + (n - 1 - i) - (D - rank[i + 1])
                if m < D and holes[m] < i:
                    dest = holes[m]
            put(dest, ("old", i))
    assert None not in out
    return out


def test_device_closed_form_matches_the_bookkeeping():
    """The device writes each row straight to its final index; on labels,
    that gives the reference's rows for every mix of divisions and
    capacities, overflow included."""
    rng = np.random.default_rng(12)
    cases = 0
    for _ in range(3000):
        n = int(rng.integers(0, 14))
        flags = [int(v) for v in rng.random(n) < rng.random()]
        n_max = n + int(rng.integers(0, 2 * sum(flags) + 3))
        assert _device_rows(n, flags, n_max) == _literal_rows(n, flags, n_max), (n, flags, n_max)
        cases += n_max < n + 2 * sum(flags)
    assert cases > 500  # overflow cases covered
