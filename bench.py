#!/usr/bin/env python
"""Agent-steps/s of the per-step hot path on B200.

Default workload (one GPU): the 3D growing colony as configured.  10^4 agents
uniform in a radius-20 ball centred in [0,400]^3 grow by division on the GPU
to 10^6 (1330 steps; about 4 agents per unit volume in the core, some 350
partners inside the cutoff per agent), and the timed steps run on that state.
Float32, soft-sphere repulsion/adhesion (k=10, a=1, r=1), Euler–Maruyama noise
sigma=0.05, volume growth with division at v=2 and death probability 1e-4
(divisions occur every step), CLVD neighbors with list radius 3.3 and rebuild
threshold 0.15, dt=0.005.  `--workload packed` times a synthetic snapshot of
10^6 agents at the packing density (0.15 per unit volume) instead.  A "step"
is one step! (rule, DE, update!, computeNeighbors!).

  value  : device time (CUDA events on the library's stream, CUDA-graph replay),
           inputs resident in HBM, L2 flushed between timed steps
  e2e    : loadToPlatform! + step! + bringFromPlatform! per step through the
           C ABI, from and to pinned host buffers (host copies included)
  roofline: the dominant kernel's algorithmic bytes / its event-timed duration
  cpu_baseline: the CPU checker (C++ restatement of the reference CPU path,
           CellLinked rebuilt every step, OpenMP over agents) on the same
           workload, a bounded sample of steps

--gpus N (under torchrun) runs N independent colonies, one per rank (weak
scaling, no data-path collective); the time is the max over ranks.
--impl reference times the CPU restatement of the reference path instead.
"""
import argparse
import datetime
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "agent-steps/s at 1M agents 3D; batched & adjoint vs plain, one B200"
UNIT = "agent-steps/s"


def load_package():
    import importlib.util
    if "cbm_b200" in sys.modules:
        return sys.modules["cbm_b200"]
    pkg = os.path.join(ROOT, "cellbasedmodels.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "cbm_b200", os.path.join(pkg, "__init__.py"), submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cbm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class NvmlClocks:
    """SM clock and clock-event reasons polled through NVML every ~1 ms while
    the timed region runs (a short region ends before nvidia-smi's first
    sample).  Read-only: nothing is set."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown",
                "nvmlClocksThrottleReasonHwSlowdown", 0x8),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown",
                "nvmlClocksThrottleReasonHwThermalSlowdown", 0x40),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown",
                "nvmlClocksThrottleReasonSwThermalSlowdown", 0x20),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap",
                "nvmlClocksThrottleReasonSwPowerCap", 0x4))

    def __init__(self, index):
        import threading

        import pynvml as N
        self.N = N
        N.nvmlInit()
        self.h = None
        try:
            import torch
            p = torch.cuda.get_device_properties(index)
            bus = "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            self.h = N.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            self.h = None
        if self.h is None:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [x for x in vis.split(",") if x.strip()]
            phys = int(ids[index]) if index < len(ids) and ids[index].isdigit() else index
            self.h = N.nvmlDeviceGetHandleByIndex(phys)
        self.smax = float(N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM))
        self.masks = [(n, getattr(N, a, getattr(N, b, m))) for n, a, b, m in self.REASONS]
        get = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            getattr(N, "nvmlDeviceGetCurrentClocksThrottleReasons")
        self.get_reasons = get
        self.samples = []
        self.stop_ev = threading.Event()
        self.thread = threading.Thread(target=self._run, daemon=True)

    def _sample(self):
        sm = self.N.nvmlDeviceGetClockInfo(self.h, self.N.NVML_CLOCK_SM)
        self.samples.append((float(sm), int(self.get_reasons(self.h))))

    def _run(self):
        while not self.stop_ev.is_set():
            self._sample()
            time.sleep(0.001)

    def start(self):
        self._sample()
        self.thread.start()

    def stop(self):
        self._sample()
        self.stop_ev.set()
        self.thread.join(timeout=5)
        reasons = set()
        for _, r in self.samples:
            for n, m in self.masks:
                if r & m:
                    reasons.add(n)
        out = {"sm_mhz": float(np.median([s for s, _ in self.samples])),
               "sm_max_mhz": self.smax, "reasons": sorted(reasons),
               "samples": len(self.samples), "source": "nvml, 1 ms polling"}
        try:
            self.N.nvmlShutdown()
        except Exception:
            pass
        return out


def Clocks(index):
    try:
        return NvmlClocks(index)
    except Exception:
        return SmiClocks(index)


class SmiClocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = max(smax, float(p[2]))
                except ValueError:
                    continue
                for n, v in zip(names, p[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi -lms 200"}


# Per-agent figures of one ncu capture of k_agent_de on the grown colony
# (Float32): DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) and warp
# instructions (smsp__inst_executed.sum) per agent of the launch.  They are
# read from the capture's summary under profiles/, which gives the command
# that made it; a changed kernel needs a new capture.
KERNEL_PROFILE = os.path.join(ROOT, "profiles", "k_agent_de_grown_colony_1m_f32.md")


def profile_per_agent(path=KERNEL_PROFILE):
    """{"dram_bytes_per_agent": B, "warp_inst_per_agent": I} from the lines
    `per-agent: name = value` of a profile summary (absent: {})."""
    out = {}
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("per-agent:") and "=" in line:
                    k, v = line[len("per-agent:"):].split("=", 1)
                    out[k.strip()] = float(v.strip().split()[0])
    except OSError:
        pass
    return out


def alg_bytes_per_agent(name, s, d, nbar, verlet, fate):
    """Compulsory HBM bytes per agent of one launch (neighbor-position gathers,
    which are served from L2, are not counted)."""
    if name == "k_agent_de":
        b = 2 * d * s + 2 * s + s  # positions r/w, volume r/w, growth rate
        b += (4 + 4 * nbar) if verlet else 8  # list count + entries, or own cell range
        b += d * s if verlet else 0  # displacement check against posOld
        b += 1 if fate else 0  # fate byte
        return b
    if name == "k_verlet_list":
        return d * s + 4 * nbar + 4  # positions, list entries, count
    if name == "k_cells_hist":
        return d * s + 8 + (d * s if verlet else 0)
    if name == "k_cells_scatter":
        return 12
    if name == "k_cells_stable":
        return 8
    if name == "k_agent_rule":
        return 2 * s + 1
    return None


def make_workload(abi, args, rank):
    """The synthetic snapshot (--workload packed): args.n agents at the
    packing density 0.15 in a ball, v ~ U(1,2)."""
    from scenarios import packed_colony_3d
    prec = abi.F64 if args.precision == "f64" else abi.F32
    kw, state = packed_colony_3d(abi, N=args.n, seed=2 + rank, precision=prec,
                                 density=args.density)
    return kw, state


def grow_colony(cbm, args, rank):
    """The 3D growing colony as configured: 10^4 agents uniform in a radius-20
    ball centred in [0,400]^3, v ~ U(1,2), g ~ U(0.8,1.2), grown by division on
    the GPU until N >= args.n (n_max = 1.2 args.n), 10 steps per graph replay.
    Returns (config kwargs, loaded context, growth steps).  The grown colony is
    far denser than packed spheres (about 4 agents per unit volume in its core
    at 10^6, some 350 neighbors inside the cutoff), which is the state the
    reference's own run reaches with this model."""
    from scenarios import growing_colony_3d
    abi = cbm._abi
    prec = abi.F64 if args.precision == "f64" else abi.F32
    kw, st = growing_colony_3d(abi, args.n, precision=prec, seed=2 + rank)
    ctx = cbm.Context(abi.make_config(**kw))
    ctx.upload(st)
    steps = 0
    while ctx.counters()["N"] < args.n and steps < 20000:
        ctx.step(10)
        steps += 10
    return kw, ctx, steps


def pinned_state(cbm, cfg, state, capacity):
    import torch
    dt = torch.float64 if cfg.precision == cbm._abi.F64 else torch.float32
    bufs = cbm._abi.StateBuffers(cfg, capacity, 0)
    for k in list(bufs.arrays):
        tdt = torch.int64 if k in ("id", "parent") else dt
        bufs.arrays[k] = torch.zeros(capacity, dtype=tdt, pin_memory=True).numpy()
    for k, v in state.items():
        if k in bufs.arrays:
            bufs.arrays[k][: len(v)] = v
    return bufs


def e2e_through_abi(cbm, ctx, cfg, steps):
    """loadToPlatform! + step! + bringFromPlatform! per step through the C ABI
    (cbm_upload, cbm_step, cbm_download) from and to pinned host buffers,
    starting from the context's current state.  The first of `steps` calls
    also builds the step graph of its parity and is not counted.  Returns
    (seconds, agent-steps, H2D bytes, D2H bytes) of the counted calls and the
    state before them."""
    import ctypes as C

    import torch
    abi = cbm._abi
    s = 8 if cfg.precision == abi.F64 else 4
    cap = int(cfg.n_max)
    snap = ctx.download()
    host = pinned_state(cbm, cfg, {k: snap[k] for k in ("x", "y", "z", "v", "g", "id", "parent")},
                        cap)
    lib = ctx.lib
    e2e_time, e2e_agents, h2d, d2h = 0.0, 0, 0, 0
    nstate = snap["N"]
    t_now, st_now, idm = snap["t"], snap["step"], snap["id_max"]
    per_agent = 3 * s + 2 * s + 16  # x,y,z,v,g + id,parent
    for k in range(steps):
        view = host.view(N=nstate, t=t_now, step=st_now, id_max=idm,
                         fields=("x", "y", "z", "v", "g", "id", "parent"))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx._check(lib.cbm_upload(ctx.h, C.byref(view)))
        ctx._check(lib.cbm_step(ctx.h, 1, abi.SYNC))
        view.capacity = cap
        ctx._check(lib.cbm_download(ctx.h, C.byref(view), abi.VIEW_COMMITTED))
        t1 = time.perf_counter()
        if k > 0:
            e2e_time += t1 - t0
            e2e_agents += nstate
            h2d += nstate * per_agent
            d2h += view.N * per_agent
        nstate, t_now, st_now, idm = view.N, view.t, view.step, view.id_max
    return e2e_time, e2e_agents, h2d, d2h, snap


def run_ours(args, rank, world, local_rank):
    import torch
    cbm = load_package()
    abi = cbm._abi
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    grow_steps = 0
    if args.workload == "grown":
        kw, ctx, grow_steps = grow_colony(cbm, args, rank)
        if args.timed_neighbors == "cell_linked":
            # the grown state in a CellLinked context: the same force walk
            # (every step of the colony has births, so CLVD walks the cells
            # too), without the Verlet rows' memory on the device
            snap = ctx.download()
            ctx.close()
            kw = dict(kw, neighbors=abi.NEIGH_CELL_LINKED)
            ctx = cbm.Context(abi.make_config(**kw))
            ctx.upload({k: snap[k] for k in ("x", "y", "z", "v", "g", "id", "parent")},
                       t=snap["t"], step=snap["step"], id_max=snap["id_max"])
        cfg = abi.make_config(**kw)
    else:
        kw, state = make_workload(abi, args, rank)
        cfg = abi.make_config(**kw)
        ctx = cbm.Context(cfg)
        ctx.upload(state)
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # Warm-up: the first steps build the step graphs of both parities; the
    # last k of them (k = min(5, W - 2)) carry an event pair around every
    # kernel (graphs of their own), read after each replay, for the per-kernel
    # times.  Event nodes cost a few microseconds a kernel, so the K timed
    # steps that follow carry none.
    n_kern = max(1, min(5, args.warmup - 2))
    kern = {}  # kernel -> [ms of each launch]
    kern_agent_steps = 0
    kernel_timing = "events inside the graph replays of the last warm-up steps"
    for w in range(args.warmup):
        timed_kernels = w >= args.warmup - n_kern
        if timed_kernels and w == args.warmup - n_kern:
            ctx.set_kernel_timing(True)
        n_before = ctx.counters()["N"]
        ctx.step(1, abi.SYNC)
        if timed_kernels and kernel_timing.startswith("events"):
            try:
                for name, ms in ctx.kernel_times():
                    kern.setdefault(name, []).append(ms)
                kern_agent_steps += n_before
            except cbm.CbmError as err:
                kernel_timing = f"eager steps after the timed region ({err})"
                kern = {}
        flush.zero_()
        torch.cuda.synchronize()
    ctx.set_kernel_timing(False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local_rank)
    clocks.start()
    total_ms, agent_steps = 0.0, 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for _ in range(args.steps):
        n_before = ctx.counters()["N"]
        e0.record(stream)
        ctx.step(1, 0)
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        agent_steps += n_before
        flush.zero_()  # evict L2 (256 MB > 126 MB) between timed steps
        torch.cuda.synchronize()
    ctx.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    if not kern:  # the graph's event nodes could not be read: time eager steps instead
        kern_agent_steps = 0
        for _ in range(5):
            kern_agent_steps += ctx.counters()["N"]
            for name, ms in ctx.profile_step():
                kern.setdefault(name, []).append(ms)
    if dist:
        t = torch.tensor([total_ms, float(agent_steps)], dtype=torch.float64, device="cuda")
        tmax = t.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        tsum = t.clone()
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        total_ms_job, agent_steps_job = float(tmax[0]), float(tsum[1])
    else:
        total_ms_job, agent_steps_job = total_ms, float(agent_steps)
    value = agent_steps_job / (total_ms_job / 1e3)
    ms_per_step = total_ms_job / args.steps

    # roofline of the dominant kernel: its launches were timed inside the
    # step graphs above, on the library's stream
    walked = ctx.counters()["flag"] == 1
    verlet = cfg.neighbors in (abi.NEIGH_CLVD, abi.NEIGH_VERLET_DISPLACEMENT) and not walked
    nbar = float(np.mean(ctx.neighbors()[0])) if verlet else 0.0
    s = 8 if cfg.precision == abi.F64 else 4
    stats = {k: (float(np.mean(v)), float(np.sum(v))) for k, v in kern.items()}
    top = max(stats, key=lambda k: stats[k][1])
    agents = kern_agent_steps / len(kern[top])  # agents per launch of the kernel-timed steps
    hbm, peak_kind = peaks()
    bpa = alg_bytes_per_agent(top, s, cfg.dims, nbar, verlet, cfg.fate != abi.FATE_NONE)
    roof = None
    if bpa is not None:
        avg_ms = stats[top][0]
        achieved = bpa * agents / (avg_ms / 1e3) / 1e9
        per = profile_per_agent() if (top == "k_agent_de" and s == 4 and walked
                                      and args.workload == "grown") else {}
        traffic = per.get("dram_bytes_per_agent")
        roof = {"kernel": top, "bound": "hbm", "achieved": round(achieved, 1),
                "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(achieved / hbm, 4),
                "traffic": None if traffic is None else round(traffic * agents),
                "traffic_source": os.path.relpath(KERNEL_PROFILE, ROOT) if traffic else None,
                "alg_bytes_per_agent": round(bpa, 2), "agents": round(agents), "nbar": round(nbar, 2),
                "avg_ms": round(avg_ms, 4), "launches_timed": len(kern[top]),
                "kernel_timing": kernel_timing}
        inst = per.get("warp_inst_per_agent")
        if inst and clk and clk.get("sm_mhz"):
            # issue-rate roofline: warp instructions per second against the
            # issue limit of 148 SMs x 4 schedulers x one instruction a clock
            n_sm = torch.cuda.get_device_properties(local_rank).multi_processor_count
            issue_peak = n_sm * 4 * clk["sm_mhz"] * 1e6
            issue = inst * agents / (avg_ms / 1e3)
            roof["issue"] = {"achieved": round(issue / 1e9, 2), "peak": round(issue_peak / 1e9, 2),
                             "unit": "G warp-instructions/s", "frac": round(issue / issue_peak, 4),
                             "warp_inst_per_agent": inst,
                             "source": os.path.relpath(KERNEL_PROFILE, ROOT)}
    step_share = {k: round(v[1] / sum(x[1] for x in stats.values()), 4) for k, v in stats.items()}
    kern = stats

    # end to end through the C ABI with pinned host buffers
    e2e_time, e2e_agents, h2d, d2h, snap = e2e_through_abi(cbm, ctx, cfg, args.e2e_steps)
    n_e2e = max(args.e2e_steps - 1, 1)
    if dist:
        t = torch.tensor([e2e_time, float(e2e_agents)], dtype=torch.float64, device="cuda")
        tm = t.clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        ts = t.clone()
        dist.all_reduce(ts, op=dist.ReduceOp.SUM)
        e2e_value = float(ts[1]) / float(tm[0])
    else:
        e2e_value = e2e_agents / e2e_time
    launches = ctx.kernels_per_step() * args.steps
    return dict(value=value, ms_per_step=ms_per_step, roof=roof, share=step_share, kern=kern,
                clocks=clk, e2e=dict(value=round(e2e_value, 1), unit=UNIT,
                                     h2d_bytes_per_step=int(h2d / n_e2e),
                                     d2h_bytes_per_step=int(d2h / n_e2e)),
                launches=launches, cfg=cfg, kw=kw, snap=snap, grow_steps=grow_steps)


def run_batched(args, rank=0, world=1, dist=None):
    """512 communities (N_i ~ U[500, 20000]) x 500 EM steps in one persistent
    launch per GPU, against the plain path run once per community (a sample).
    Under torchrun the communities are partitioned across ranks by agent count
    (no data-path collective; strong scaling of the fixed sweep) and the time
    is the max over ranks."""
    import torch
    from scenarios import batched_sweep, make_descs, plain_config_for
    cbm = load_package()
    abi = cbm._abi
    base, descs, states = batched_sweep(abi, n_comm=args.batched_comms)
    sb = cbm.ShardedBatch(abi.make_config(**base), make_descs(abi, descs), rank=rank, world=world)
    b = sb.batch

    def load_all():
        for c, st in enumerate(states):
            sb.upload(c, st["x"], st["y"], st["z"])

    load_all()
    tuning, tune_s = None, 0.0
    if b is not None:
        t0 = time.perf_counter()
        tuning = b.tuning() if args.batched_no_autotune else b.autotune(trial_steps=args.batched_trial)
        tune_s = time.perf_counter() - t0
        b.step(args.batched_steps)  # first replay builds the graph
    load_all()
    ms, clk = 0.0, None
    if dist:
        dist.barrier()
    if b is not None:
        stream = torch.cuda.ExternalStream(b.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        clocks = Clocks(torch.cuda.current_device())
        clocks.start()
        e0.record(stream)
        b.step(args.batched_steps, 0)
        e1.record(stream)
        e1.synchronize()
        clk = clocks.stop()
        b.step(0)  # report device flags
        ms = e0.elapsed_time(e1)
    ms_job = cbm.sweep.max_over_ranks(dist, ms)
    total = sum(d["n"] for d in descs)
    batched = total * args.batched_steps / (ms_job / 1e3)
    roof = None
    if tuning is not None:
        # compulsory bytes of a list step per agent: positions read and
        # written (2 x 3 x 4), the row count (4) and the list row (4 n_bar),
        # n_bar = density x (4/3) pi R^3 at the sweep's density (one agent
        # per 2.5^3) and the tuned list radius R = cutoff + skin
        R = 3.0 + tuning.skin
        nbar = (1.0 / 2.5 ** 3) * 4.0 / 3.0 * math.pi * R ** 3
        bpa = 2 * 3 * 4 + 4 + 4 * nbar
        hbm, peak_kind = peaks()
        achieved = bpa * batched / 1e9
        roof = {"kernel": "k_batch", "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "alg_bytes_per_agent_step": round(bpa, 1), "nbar": round(nbar, 1),
                "list_radius": R}
    out = {"communities": len(descs), "agents": int(total), "steps": args.batched_steps,
           "value": round(batched, 1), "unit": UNIT, "ms": round(ms_job, 3),
           "ranks": world, "scaling": "strong" if world > 1 else None,
           "rank0_communities": len(sb.mine), "rank0_agents": int(sb.n_agents),
           "tuning": tuning.as_dict() if tuning is not None else None,
           "autotune_s": round(tune_s, 3), "clocks": clk, "roofline": roof}
    if rank != 0 or tuning is None:
        return out
    # The plain path, one community at a time, on a sample of the communities:
    # device time of the 500 steps (graphs built beforehand by a 2-step run of
    # the same context) and end to end (upload + 500 steps + download).
    rng = np.random.default_rng(7)
    sample = sorted(rng.choice(len(descs), size=min(args.plain_sample, len(descs)), replace=False))
    agents, dev_ms, e2e_s = 0, 0.0, 0.0
    for c in sample:
        st = states[c]
        g = cbm.Context(abi.make_config(**plain_config_for(abi, base, descs[c], tuning.as_dict())))
        g.upload(st)
        g.step(2)  # builds the step graph of both parities
        stream = torch.cuda.ExternalStream(g.stream())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.upload(st)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step(args.batched_steps, 0)
        e1.record(stream)
        g.download()
        e2e_s += time.perf_counter() - t0
        dev_ms += e0.elapsed_time(e1)
        agents += descs[c]["n"] * args.batched_steps
        g.close()
    plain_dev = agents / (dev_ms / 1e3)
    out.update({"plain_value": round(plain_dev, 1), "plain_e2e_value": round(agents / e2e_s, 1),
                "plain_sample": len(sample),
                "plain_timing": "device events around the 500 graph-replayed steps of each "
                                "sampled community (graphs built beforehand); e2e adds "
                                "upload and download"})
    if world == 1:
        out["speedup_vs_plain"] = round(batched / plain_dev, 2)
    return out


def run_adjoint(args):
    """Gradient of the trajectory MSE (65536 agents, 200 Euler steps, Float64,
    checkpoint every 20) against the forward trajectory alone."""
    import torch
    from scenarios import adjoint_problem
    cbm = load_package()
    abi = cbm._abi
    kw, x0, star = adjoint_problem(abi, N=args.adjoint_n, steps=args.adjoint_steps)
    k, a, rho = star
    tgt_fw = cbm.Adjoint(abi.make_config(**dict(kw, k_rep=k, k_att=a, r_rep=rho, r_att=1.5 * rho,
                                                cell_edge=max(kw["cell_edge"], 1.5 * rho))))
    tgt = tgt_fw.forward(x0, args.adjoint_steps)
    adj = cbm.Adjoint(abi.make_config(**kw))
    adj.forward(x0, args.adjoint_steps)  # warm-up: builds the forward plan (buffers + graph)
    adj.run(x0, tgt, args.adjoint_steps, checkpoint_every=args.checkpoint_every)
    stream = torch.cuda.ExternalStream(adj.stream())

    def timed(fn, reps=5):
        out, ms = None, []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            out = fn()  # synchronous: copies in, graph replay, copies out
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return out, float(np.median(ms))

    _, fwd = timed(lambda: adj.forward(x0, args.adjoint_steps))
    res, full = timed(lambda: adj.run(x0, tgt, args.adjoint_steps,
                                      checkpoint_every=args.checkpoint_every))
    return {"agents": args.adjoint_n, "steps": args.adjoint_steps, "dtype": "f64",
            "checkpoint_every": args.checkpoint_every, "forward_ms": round(fwd, 3),
            "forward_plus_adjoint_ms": round(full, 3), "backward_ms": round(full - fwd, 3),
            "cost_ratio": round(full / fwd, 3), "loss": res["loss"],
            "dL_dtheta": [float(v) for v in res["dtheta"]],
            "timing": "CUDA events on the adjoint stream around each synchronous call "
                      "(host<->device copies included), median of 5; cost_ratio = "
                      "(forward + checkpointed backward) / forward"}


def _one_call(ctx, steps):
    """Device time (ms) of `steps` steps made by one cbm_step call (as
    evolve! over that many steps makes them), one event pair around it."""
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    ctx.step(steps, 0)
    e1.record(stream)
    e1.synchronize()
    ctx.sync()
    return e0.elapsed_time(e1)


def _device_steps(cbm, ctx, steps, flush=None):
    """Device time (ms) of `steps` graph-replayed steps, one event pair per step."""
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream())
    total = 0.0
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.step(1, 0)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
        if flush is not None:
            flush.zero_()
            torch.cuda.synchronize()
    ctx.sync()
    return total


def _rel_err(a, b):
    """max |a - b| over max |b| (positions: relative to the box scale)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if b.size else 0.0


def run_medium_3d(cbm, abi, n_medium=256, agents=200_000, steps=50):
    """The explicit medium in 3D: a 256^3 Float32 field (unit spacing, D=1,
    decay 0.01, dt 0.05) with 2x10^5 agents that secrete, take up (first
    order) and follow the gradient.  The steps are timed as one cbm_step
    call (chained step graphs), and one call a step for comparison; the
    medium kernels are then timed inside the step graph (an event pair
    around each kernel) over as many steps; their roofline is the compulsory bytes per
    node (gradient: c read, three components written, 16 B; FTCS: c read
    and written, 8 B) over their time, against the measured HBM bandwidth."""
    from scenarios import medium_colony
    kw, st = medium_colony(abi, 3, N=agents, L=float(n_medium), n_medium=n_medium)
    st["c"] = np.random.default_rng(9).uniform(0.0, 1.0, n_medium ** 3).astype(np.float32)
    g = cbm.Context(abi.make_config(**kw))
    g.upload(st)
    g.step(3)
    # the steps themselves, graph replays without timing nodes
    total = _one_call(g, steps)
    per_call = _device_steps(cbm, g, steps)
    # then the same number of steps with an event pair around every kernel
    g.set_kernel_timing(True)
    g.step(1)
    kern = {}
    for _ in range(steps):
        g.step(1, 0)
        for name, ms in g.kernel_times():
            kern.setdefault(name, []).append(ms)
    g.set_kernel_timing(False)
    g.close()
    nodes = n_medium ** 3
    hbm, peak_kind = peaks()
    roof = {}
    for name, bpn in (("k_medium_de", 8), ("k_medium_grad", 16)):
        if name in kern:
            ms = float(np.mean(kern[name]))
            gbs = bpn * nodes / (ms / 1e3) / 1e9
            roof[name] = {"avg_ms": round(ms, 4), "bytes_per_node": bpn,
                          "achieved_gbs": round(gbs, 1), "frac": round(gbs / hbm, 3)}
    return {"medium": f"{n_medium}^3 Float32", "agents": agents, "steps_timed": steps,
            "us_per_step": round(1e3 * total / steps, 2),
            "us_per_step_one_call_per_step": round(1e3 * per_call / steps, 2),
            "cell_updates_per_s": round(nodes * steps / (total / 1e3), 1),
            "kernel_avg_ms": {k: round(float(np.mean(v)), 4) for k, v in kern.items()},
            "roofline": roof, "peak": hbm, "peak_kind": peak_kind}


def run_dgadi(cpu=True):
    """The implicit medium (DGADI) lines: {name: record}."""
    import torch
    from _oracle import OracleMedium
    cbm = load_package()
    abi = cbm._abi
    out = {}
    # Implicit medium (DGADI): the two workloads of examples/Implementation.ipynb,
    # co2 and co3 (D = 1 and 2) on [0,1]^d, dt 0.01, a source of strength 1 at
    # the central node, Float32 as the reference's GPU platform runs them.
    # The notebook's @time (2.45 s for 500 2D steps, 45.67 % of it compilation;
    # 10.64 s for 200 3D steps; GPU model not stated) is wall time around the
    # loop; wall_ms here is the same loop through the C ABI, synchronised.
    for name, dims, nn, steps, cpu_steps, published in (
            ("medium_dgadi_2d_101", 2, (101, 101, 1), 500, 50, 2.45),
            ("medium_dgadi_3d_101", 3, (101, 101, 101), 200, 2, 10.64)):
        mcfg = abi.make_medium_config(dims, nn, (0.0,) * 3, (1.0,) * 3, 0.01, [1.0, 2.0],
                                      c_max=1.0, precision=abi.F32)
        nodes = int(np.prod(nn[:dims]))
        src = np.zeros(tuple(reversed(nn[:dims])), np.float32)
        src[tuple(round(k / 2) - 1 for k in reversed(nn[:dims]))] = 1.0
        u0 = np.zeros((2, nodes), np.float32)
        med = abi.DGADIMedium(mcfg)
        med.upload(u0, src.reshape(-1))
        med.step(10)
        mst = torch.cuda.ExternalStream(med.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        e0.record(mst)
        med.step(steps, 0)
        e1.record(mst)
        e1.synchronize()
        wall = time.perf_counter() - w0
        dev_ms = e0.elapsed_time(e1)
        med.close()
        cpu_ms = None
        if cpu:
            o = OracleMedium(abi, mcfg)
            o.upload(u0, src.reshape(-1))
            c0 = time.perf_counter()
            o.step(cpu_steps)
            cpu_ms = round(1e3 * (time.perf_counter() - c0) / cpu_steps, 3)
            o.close()
        out[name] = {"workload": f"examples/Implementation.ipynb {dims}D: 2 fields on "
                                 f"{'x'.join(str(k) for k in nn[:dims])} nodes, {steps} DGADI steps",
                     "dtype": "f32", "steps": steps, "device_ms": round(dev_ms, 3),
                     "wall_ms": round(wall * 1e3, 3), "us_per_step": round(1e3 * dev_ms / steps, 2),
                     "node_updates_per_s": round(2 * nodes * steps / (dev_ms / 1e3), 1),
                     "reference_published_s": published,
                     "cpu_oracle_ms_per_step": cpu_ms, "cpu_oracle_threads": 1}
    return out


def rod_disc(abi, n, seed=21):
    """n rods of d = 1, l uniform in [2, 3], uniform in a disc at about one rod
    per 3.8 units^2 (the colony's packing), small random velocities."""
    rng = np.random.default_rng(seed)
    radius = math.sqrt(n * 3.8 / math.pi)
    r = radius * np.sqrt(rng.uniform(0, 1, n))
    phi = rng.uniform(0, 2 * math.pi, n)
    st = {k: np.zeros(n) for k in abi.ROD_FIELDS}
    st["x"], st["y"] = r * np.cos(phi), r * np.sin(phi)
    st["vx"], st["vy"] = rng.normal(0, 0.01, n), rng.normal(0, 0.01, n)
    st["theta"] = rng.uniform(-math.pi, math.pi, n)
    st["omega"] = rng.normal(0, 0.01, n)
    st["d"], st["m"] = np.ones(n), np.ones(n)
    st["l"] = rng.uniform(2.0, 3.0, n)
    return st


# Model constants of examples/Bacteries.ipynb in its natural units (m = 1/100,
# g = 1/10000, d = 1): kn = 2e6 m g / d, gamma = 2.2e2 sqrt(g / d)
ROD_PARAMS = dict(dt=0.1, kn=2.0e6 * (1e-2 * 1e-4), gamma_n=2.2e2 * math.sqrt(1e-4),
                  gamma_t=2.2e2 * math.sqrt(1e-4), mu_cc=0.1, mu_cw=0.8, beta=0.8, beta_w=0.8)


def run_rods(cpu=True, n=32768, steps=200, cpu_steps=3):
    """The rods2D line: a colony of the size examples/Bacteries.ipynb times
    (about 3.2e4 rods, Float64, CellLinked cellEdge 4, simBox [-300, 300]^2),
    200 steps through the C ABI, with the CPU checker beside it."""
    import torch
    from _oracle import OracleRods
    cbm = load_package()
    abi = cbm._abi
    st = rod_disc(abi, n)
    cfg = abi.make_rods_config(n, (-300.0, -300.0), (300.0, 300.0), cell_edge=4.0,
                               neighbors=abi.NEIGH_CELL_LINKED, precision=abi.F64, **ROD_PARAMS)
    g = abi.Rods2D(cfg)
    g.upload(st)
    g.step(5)
    rst = torch.cuda.ExternalStream(g.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(rst)
    g.step(steps, 0)
    e1.record(rst)
    e1.synchronize()
    dev_ms = e0.elapsed_time(e1)
    # e2e: host state in, steps, host state out
    w0 = time.perf_counter()
    g.upload(st)
    g.step(steps, 0)
    out_state = g.download()
    wall = time.perf_counter() - w0
    g.close()
    rec = {"workload": f"rods2D colony, {n} rods (d 1, l 2-3) in a disc at one rod per 3.8 "
                       f"units^2, examples/Bacteries.ipynb constants, dt 0.1, CellLinked "
                       f"cellEdge 4, simBox [-300,300]^2",
           "dtype": "f64", "rods": n, "steps": steps, "device_ms": round(dev_ms, 3),
           "ms_per_step": round(dev_ms / steps, 4),
           "value": round(n * steps / (dev_ms / 1e3), 1), "unit": "rod-steps/s",
           "e2e_rod_steps_per_s": round(n * steps / wall, 1),
           "rods_in_contact": int(np.count_nonzero(out_state["pressure"]))}
    if cpu:
        o = OracleRods(abi, cfg)
        o.upload(st)
        c0 = time.perf_counter()
        o.step(cpu_steps)
        cpu_s = (time.perf_counter() - c0) / cpu_steps
        o.close()
        rec["cpu_oracle_ms_per_step"] = round(1e3 * cpu_s, 3)
        rec["cpu_oracle_threads"] = os.cpu_count()
        rec["cpu_value"] = round(n / cpu_s, 1)
    return rec


# rods2dGrowth constants of examples/Bacteries.ipynb: growth = 1e-6 sqrt(g d) 1e5,
# lMax 3, sigma_lTarget 0.2, alpha 50
ROD_GROWTH = dict(growth=1e-6 * math.sqrt(1e-4) * 1e5, alpha=50.0, sigma_l_target=0.2,
                  l_max=3.0, seed=2024)


def run_rods_growth(n=32768, steps=200):
    """The rods2dGrowth line: the disc of run_rods with lTarget = l + U(0, 0.02),
    so that rods divide throughout the timed steps (the notebook's scaling loop
    times 200 steps of a growing colony at about this size)."""
    import torch
    cbm = load_package()
    abi = cbm._abi
    st = rod_disc(abi, n)
    st["l_target"] = st["l"] + np.random.default_rng(5).uniform(0.0, 0.02, n)
    cfg = abi.make_rods_config(2 * n, (-300.0, -300.0), (300.0, 300.0), cell_edge=4.0,
                               neighbors=abi.NEIGH_CELL_LINKED, precision=abi.F64,
                               **ROD_PARAMS, **ROD_GROWTH)
    g = abi.Rods2D(cfg)
    g.upload(st)
    g.step(2)
    n0 = len(g.download()["x"])
    rst = torch.cuda.ExternalStream(g.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(rst)
    g.step(steps, 0)
    e1.record(rst)
    e1.synchronize()
    dev_ms = e0.elapsed_time(e1)
    n1 = len(g.download()["x"])
    g.close()
    return {"workload": f"rods2dGrowth colony, {n} rods at start (the rods2d line's disc), "
                        f"lTarget = l + U(0, 0.02), examples/Bacteries.ipynb constants, dt 0.1, "
                        f"CellLinked cellEdge 4, n_max {2 * n}",
            "dtype": "f64", "rods_start": n0, "rods_end": n1, "steps": steps,
            "device_ms": round(dev_ms, 3), "ms_per_step": round(dev_ms / steps, 4),
            "value": round(0.5 * (n0 + n1) * steps / (dev_ms / 1e3), 1), "unit": "rod-steps/s"}


def run_aggregation_2d(args, cbm, abi, cpu=True):
    """c1: the 2D aggregation, 4096 agents, Float64: the timed steps as one
    cbm_step call (one launch of the small-community kernel), one call a step
    for comparison, and the CPU checker beside it when `cpu`."""
    import torch
    from _oracle import OracleContext
    from scenarios import aggregation_2d
    threads = os.cpu_count()
    kw, st = aggregation_2d(abi)
    g = cbm.Context(abi.make_config(**kw))
    g.upload(st)
    g.step(3)
    ms = _one_call(g, args.config_steps)
    ms_graph = _device_steps(cbm, g, 20)  # one call per step, for comparison
    g.close()
    rec = {"agents": 4096, "dtype": "f64", "steps_timed": args.config_steps,
           "us_per_step": round(1e3 * ms / args.config_steps, 2),
           "value": round(4096 * args.config_steps / (ms / 1e3), 1), "unit": UNIT,
           "us_per_step_one_call_per_step": round(1e3 * ms_graph / 20, 2),
           "note": "L2-resident: the timed steps are one cbm_step call, run by one launch of "
                   "a thread-block cluster (hardware cluster barriers between the phases of a "
                   "step); us_per_step_one_call_per_step: one call (one launch) per step"}
    if cpu:
        o = OracleContext(abi, abi.make_config(**kw), threads=threads)
        o.upload(st)
        t0 = time.perf_counter()
        o.step(args.config_cpu_steps)
        cpu_s = (time.perf_counter() - t0) / args.config_cpu_steps
        o.close()
        rec.update(cpu_us_per_step=round(1e6 * cpu_s, 2), cpu_cores=threads)
    return rec


def run_chemotaxis_2d(args, cbm, abi, cpu=True):
    """c3: 2D chemotaxis, 2x10^5 agents on a 1024^2 Float32 medium: graph
    replays, eager per-kernel times, and the CPU checker beside it when `cpu`."""
    from _oracle import OracleContext
    from scenarios import chemotaxis_2d
    threads = os.cpu_count()
    kw, st = chemotaxis_2d(abi)
    g = cbm.Context(abi.make_config(**kw))
    g.upload(st)
    g.step(3)
    g.step(8)  # builds the chained graph the timed call starts with (odd step count)
    ms = _one_call(g, args.config_steps)
    ms_step = _device_steps(cbm, g, 20)  # one call per step, for comparison
    prof = {}
    for _ in range(3):
        for name, kms in g.profile_step():
            prof.setdefault(name, []).append(kms)
    g.close()
    nodes = 1024 * 1024
    rec = {"agents": 200000, "medium": "1024x1024", "dtype": "f32", "steps_timed": args.config_steps,
           "us_per_step": round(1e3 * ms / args.config_steps, 2),
           "value": round(200000 * args.config_steps / (ms / 1e3), 1), "unit": UNIT,
           "cell_updates_per_s": round(nodes * args.config_steps / (ms / 1e3), 1),
           "us_per_step_one_call_per_step": round(1e3 * ms_step / 20, 2),
           "kernel_avg_ms": {k: round(float(np.mean(v)), 4) for k, v in prof.items()},
           "note": "bilinear secretion and uptake as an ordered gather, FTCS, chemotactic drift; "
                   "the timed steps are one cbm_step call (chained step graphs); "
                   "us_per_step_one_call_per_step: one call (one graph replay) per step"}
    if cpu:
        o = OracleContext(abi, abi.make_config(**kw), threads=threads)
        o.upload(st)
        t0 = time.perf_counter()
        o.step(args.config_cpu_steps)
        cpu_s = (time.perf_counter() - t0) / args.config_cpu_steps
        o.close()
        rec.update(cpu_value=round(200000 / cpu_s, 1), cpu_cores=threads)
    return rec


def run_configs(args):
    """The other configurations of the path: the 2D aggregation (Float64,
    L2-resident, launch-bound: us/step) and 2D chemotaxis on a 1024^2 medium
    (agent-steps/s and medium cell-updates/s), each with the CPU checker
    beside it; the 3D colony in Float64; and the error of every Float32 result
    against a Float64 run of the same seeded inputs after 100 steps."""
    import torch
    from scenarios import aggregation_2d, chemotaxis_2d, colony_3d, growing_colony_3d, packed_colony_3d
    cbm = load_package()
    abi = cbm._abi
    out = {}

    out["aggregation_2d"] = run_aggregation_2d(args, cbm, abi, cpu=True)
    out["chemotaxis_2d"] = run_chemotaxis_2d(args, cbm, abi, cpu=True)

    # c2 as a whole run: 10^4 agents uniform in a radius-20 ball centred in
    # [0,400]^3, grown by division to 10^6 (n_max 1.2M), Float32, graph
    # replays in chunks of 10 steps; agent-steps counted per chunk from N at its
    # ends (trapezoid)
    kw, st = growing_colony_3d(abi, 1_000_000, seed=2)
    g = cbm.Context(abi.make_config(**kw))
    g.upload(st)
    stream = torch.cuda.ExternalStream(g.stream())
    n_prev, steps, agent_steps, dev_ms = 10_000, 0, 0.0, 0.0
    while n_prev < 1_000_000 and steps < 5000:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step(10, 0)
        e1.record(stream)
        e1.synchronize()
        dev_ms += e0.elapsed_time(e1)
        n_now = g.counters()["N"]
        agent_steps += 10 * (n_prev + n_now) / 2.0
        steps += 10
        n_prev = n_now
    g.sync()
    g.close()
    out["colony_3d_growth"] = {
        "start": "10^4 agents uniform in a radius-20 ball centred in [0,400]^3", "dtype": "f32",
        "steps_to_1e6": steps, "final_agents": int(n_prev), "device_s": round(dev_ms / 1e3, 4),
        "value": round(agent_steps / (dev_ms / 1e3), 1), "unit": UNIT}

    # c2 in Float64: the colony grown in Float64 from the same start, timed on
    # that state; and the Float32 packed snapshot (density 0.15), the light
    # synthetic stand-in this configuration used to be timed on
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    class _F64:
        n = args.n
        precision = "f64"
    kw64, g, gsteps = grow_colony(cbm, _F64, 0)
    n0 = g.counters()["N"]
    g.step(3)
    ms = _device_steps(cbm, g, args.config_f64_steps, flush=flush)
    # end to end through the C ABI in Float64, host copies included
    et, ea, eh, ed, _ = e2e_through_abi(cbm, g, abi.make_config(**kw64), args.e2e_steps)
    g.close()
    n_e2e = max(args.e2e_steps - 1, 1)
    out["colony_3d_f64"] = {"workload": "grown from 10^4 in Float64", "grow_steps": gsteps,
                            "agents": int(n0), "steps_timed": args.config_f64_steps,
                            "ms_per_step": round(ms / args.config_f64_steps, 4),
                            "value": round(n0 * args.config_f64_steps / (ms / 1e3), 1),
                            "unit": UNIT, "dtype": "f64",
                            "e2e": {"value": round(ea / et, 1), "unit": UNIT,
                                    "h2d_bytes_per_step": int(eh / n_e2e),
                                    "d2h_bytes_per_step": int(ed / n_e2e)}}
    kw, st = packed_colony_3d(abi, N=args.n)
    g = cbm.Context(abi.make_config(**kw))
    g.upload(st)
    g.step(3)
    n0 = g.counters()["N"]
    ms = _device_steps(cbm, g, args.config_f64_steps, flush=flush)
    g.close()
    del flush
    out["colony_3d_packed_f32"] = {"workload": "synthetic snapshot at density 0.15",
                                   "agents": int(n0), "steps_timed": args.config_f64_steps,
                                   "ms_per_step": round(ms / args.config_f64_steps, 4),
                                   "value": round(n0 * args.config_f64_steps / (ms / 1e3), 1),
                                   "unit": UNIT}

    out["medium_3d_ftcs"] = run_medium_3d(cbm, abi)
    out.update(run_dgadi())
    out["rods2d_colony_32k_f64"] = run_rods()
    out["rods2d_growth_32k_f64"] = run_rods_growth()

    # Error of the Float32 results against Float64 runs, 100 steps.  The noise
    # of an SDE run is drawn in the run's precision (Box-Muller in float or
    # double), so the two precisions follow different sample paths; the
    # comparison therefore runs each configuration with sigma = 0, which
    # isolates the arithmetic precision.
    def colony_nodiv(abi, precision):
        # division thresholds (v >= 2) are crossed at different steps in the two
        # precisions, which changes the agent set; growth and death are off here
        kw, st = colony_3d(abi, N=20000, precision=precision, p_death=0.0, sigma=0.0)
        return dict(kw, growth=0, fate=abi.FATE_NONE), st

    def chemo_ode(abi, precision):
        kw, st = chemotaxis_2d(abi, N=20000, L=256.0, n_medium=256, precision=precision)
        return dict(kw, sigma=0.0, integrator=abi.INT_EULER), st

    def pair(builder, keys, steps=100):
        res = []
        for prec in (abi.F32, abi.F64):
            kw, st = builder(abi, precision=prec)
            g = cbm.Context(abi.make_config(**kw))
            g.upload(st)
            g.step(steps)
            res.append(g.download())
            g.close()
        f32, f64 = res
        if f32["N"] != f64["N"]:
            return {"N_f32": int(f32["N"]), "N_f64": int(f64["N"])}
        out = {}
        for k in keys:
            a = np.asarray(f32[k], np.float64)
            b = np.asarray(f64[k], np.float64)
            scale = max(float(np.max(np.abs(b))), 1e-300)
            d = np.abs(a - b) / scale
            out[k] = {"max": float(np.max(d)), "median": float(np.median(d))}
        return out

    out["error_vs_f64_100_steps"] = {
        "aggregation_2d": pair(aggregation_2d, ("x", "y")),
        "chemotaxis_2d_sigma0": pair(chemo_ode, ("x", "y", "c")),
        "colony_3d_sigma0_no_division": pair(colony_nodiv, ("x", "y", "z")),
        "definition": "|v_f32 - v_f64| / max |v_f64| per field after 100 steps from the same "
                      "seeded inputs, max and median over agents (medium nodes for c); "
                      "Float32 and Float64 runs on the GPU, each bit-identical to the CPU "
                      "checker in its own precision"}
    return out


def cpu_baseline(args, steps, threads=None, kw=None, snap=None):
    """The CPU checker on the same workload (CellLinked, rebuilt every step),
    from the same state as the GPU run (`snap`, a download of it) when given."""
    cbm = load_package()
    abi = cbm._abi
    from _oracle import OracleContext
    up = {}
    if snap is None:
        kw, state = make_workload(abi, args, 0)
    else:
        state = {k: snap[k] for k in ("x", "y", "z", "v", "g", "id", "parent")}
        up = dict(t=snap["t"], step=snap["step"], id_max=snap["id_max"])
    kw = dict(kw, neighbors=abi.NEIGH_CELL_LINKED, precision=abi.F64)
    cfg = abi.make_config(**kw)
    threads = threads or os.cpu_count()
    o = OracleContext(abi, cfg, threads=threads)
    o.upload(state, **up)
    agent_steps, wall = 0, 0.0
    for _ in range(steps):
        n = o.counters()["N"]
        t0 = time.perf_counter()
        o.step(1)
        wall += time.perf_counter() - t0
        agent_steps += n
    return dict(value=agent_steps / wall, unit=UNIT, cores=threads, kind="port",
                sample=f"{steps} full steps of the {'grown' if snap is not None else 'packed'} "
                       f"colony ({agent_steps // steps} agents), Float64, CellLinked(3.3) rebuilt "
                       f"every step, OpenMP over agents, from the GPU run's state")


def run_reference(args, config):
    """The reference arm: the CPU restatement of the reference's CPU path (the
    oracle: Float64, CellLinked rebuilt every step, OpenMP over agents, serial
    compaction, as src/neighbors.jl:918-979 and update.jl:15-119 run it) on
    all host cores, W untimed and K timed steps.  The reference is Julia and
    cannot run here.  Its input is built without the product library: growing
    10^4 agents to 10^6 on the CPU takes hours, so for the grown workload a
    stand-in of 10^6 agents is drawn from the grown colony's measured density,
    volume and growth-rate histograms (tests/golden/), with the grown state's
    partner counts.  The CPU steps it at least as fast as the grown state
    itself, so the ratio to this arm understates the speed-up, if anything."""
    cbm = load_package()  # the ctypes structures only: libcbm_b200.so is not loaded
    abi = cbm._abi
    from _oracle import OracleContext
    if args.workload == "grown":
        from scenarios import grown_colony_stand_in
        kw, state = grown_colony_stand_in(abi, precision=abi.F64)
        sample = ("the 10^6-agent grown-colony stand-in (density, volume and growth-rate "
                  "histograms of the colony grown on the device, numbered in cell order)")
    else:
        kw, state = make_workload(abi, args, 0)
        sample = f"the packed snapshot at density {args.density}"
    kw = dict(kw, neighbors=abi.NEIGH_CELL_LINKED, precision=abi.F64)
    threads = os.cpu_count()
    o = OracleContext(abi, abi.make_config(**kw), threads=threads)
    o.upload(state)
    for _ in range(args.warmup):
        o.step(1)
    wall, agent_steps = 0.0, 0
    for _ in range(args.steps):
        n = o.counters()["N"]
        t0 = time.perf_counter()
        o.step(1)
        wall += time.perf_counter() - t0
        agent_steps += n
    o.close()
    value = agent_steps / wall
    cb = {"value": round(value, 1), "unit": UNIT, "cores": threads, "kind": "port",
          "sample": f"{args.steps} timed steps (after {args.warmup} untimed) of {sample}, "
                    f"{agent_steps // max(args.steps, 1)} agents per step, Float64, "
                    f"CellLinked(3.3) rebuilt every step, OpenMP over agents"}
    return {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * wall / max(args.steps, 1), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config, "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference is Julia and cannot run here; this times its C++ restatement "
                    "(the CPU checker) on the host cores"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--density", type=float, default=0.15,
                    help="agents per unit volume of the --workload packed snapshot (the grown "
                         "colony reaches about 4 in its core)")
    ap.add_argument("--workload", default="grown", choices=["grown", "packed"],
                    help="grown: the colony grown from 10^4 to n (the configured run); "
                         "packed: a synthetic snapshot at packing density")
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--timed-neighbors", default="clvd", choices=["clvd", "cell_linked"],
                    help="cell_linked: time the grown state in a CellLinked context (the same "
                         "force walk without the Verlet rows' memory; for profiler captures)")
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-comms", type=int, default=512)
    ap.add_argument("--batched-steps", type=int, default=500)
    ap.add_argument("--batched-trial", type=int, default=20)
    ap.add_argument("--plain-sample", type=int, default=32)
    ap.add_argument("--batched-no-autotune", action="store_true",
                    help="keep the default tuning (for profiling one known launch)")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    ap.add_argument("--dgadi-only", action="store_true",
                    help="print only the implicit-medium (DGADI) lines, without the CPU checker")
    ap.add_argument("--rods-only", action="store_true",
                    help="print only the rods2D line, without the CPU checker")
    ap.add_argument("--config-only", choices=["aggregation_2d", "chemotaxis_2d"],
                    help="print only that configuration's line, without the CPU checker")
    ap.add_argument("--medium-only", action="store_true",
                    help="print only the 3D explicit-medium line")
    ap.add_argument("--medium-n", type=int, default=256, help="nodes per axis of the 3D medium")
    ap.add_argument("--medium-agents", type=int, default=200_000)
    ap.add_argument("--medium-steps", type=int, default=50)
    ap.add_argument("--config-steps", type=int, default=200)
    ap.add_argument("--config-cpu-steps", type=int, default=5)
    ap.add_argument("--config-f64-steps", type=int, default=10)
    ap.add_argument("--adjoint-n", type=int, default=65536)
    ap.add_argument("--adjoint-steps", type=int, default=200)
    ap.add_argument("--checkpoint-every", type=int, default=20)
    args = ap.parse_args()
    if args.dgadi_only:
        print(json.dumps({"dgadi": run_dgadi(cpu=False)}))
        return
    if args.rods_only:
        print(json.dumps({"rods": run_rods(cpu=False), "rods_growth": run_rods_growth()}))
        return
    if args.config_only:
        cbm = load_package()
        fn = {"aggregation_2d": run_aggregation_2d, "chemotaxis_2d": run_chemotaxis_2d}
        print(json.dumps({args.config_only: fn[args.config_only](args, cbm, cbm._abi, cpu=False)}))
        return
    if args.medium_only:
        cbm = load_package()
        print(json.dumps({"medium_3d_ftcs": run_medium_3d(
            cbm, cbm._abi, n_medium=args.medium_n, agents=args.medium_agents,
            steps=args.medium_steps)}))
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.workload == "grown":
        workload = (f"3D growing colony: 10^4 agents uniform in a radius-20 ball centred in "
                    f"[0,400]^3 grown by division to {args.n} (n_max {int(1.2 * args.n)}), then "
                    f"timed; {args.precision}, EM sigma 0.05, division at v=2 + death 1e-4, "
                    f"CLVD R_list 3.3 rebuild 0.15, dt 0.005")
    else:
        workload = (f"3D colony snapshot, {args.n} agents at density {args.density} in a ball in "
                    f"[0,400]^3, {args.precision}, EM sigma 0.05, division at v=2 + death 1e-4 "
                    f"every step, CLVD R_list 3.3 rebuild 0.15, dt 0.005")
    config = {"workload": workload, "n_agents": args.n, "n_max": int(1.2 * args.n),
              "neighbors": "CLVD", "l2": "flushed between timed steps (256 MB write)",
              "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single GPU"}

    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(run_reference(args, config)), flush=True)
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    r = run_ours(args, rank, world, local_rank)
    cb = batched = adjoint = None
    if not args.no_batched:
        batched = run_batched(args, rank, world, dist if world > 1 else None)
    configs = None
    if rank == 0 and world == 1:
        if not args.no_configs:
            configs = run_configs(args)
        if not args.no_adjoint:
            adjoint = run_adjoint(args)
        if not args.no_cpu_baseline:
            cb = cpu_baseline(args, args.cpu_steps, kw=r["kw"], snap=r["snap"])
    if rank == 0:
        line = {"metric": METRIC, "value": round(r["value"], 1), "unit": UNIT,
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(r["ms_per_step"], 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
                "data": "synthetic", "config": config,
                "state": {"grow_steps": r["grow_steps"], "agents_after_timing": r["snap"]["N"]},
                "roofline": r["roof"],
                "cpu_baseline": cb, "e2e": r["e2e"], "gpu_launches": r["launches"],
                "clocks": r["clocks"], "kernel_share": r["share"],
                "kernel_avg_ms": {k: round(v[0], 4) for k, v in r["kern"].items()},
                "configs": configs, "batched": batched, "adjoint": adjoint}
        # the key figures once more at the end of the line (a reader that keeps
        # only its tail still sees them)
        summ = {"value": line["value"], "e2e": r["e2e"]["value"],
                "k_agent_de_ms": r["roof"]["avg_ms"] if r["roof"] else None,
                "issue_frac": (r["roof"] or {}).get("issue", {}).get("frac"),
                "cpu_baseline": round(cb["value"], 1) if cb else None}
        if batched:
            summ.update(batched=batched.get("value"), batched_vs_plain=batched.get("speedup_vs_plain"))
        if adjoint:
            summ["adjoint_cost_ratio"] = adjoint.get("cost_ratio")
        if configs:
            summ["aggregation_2d_us_per_step"] = configs["aggregation_2d"]["us_per_step"]
            summ["colony_3d_f64"] = configs["colony_3d_f64"]["value"]
            summ["colony_3d_f64_e2e"] = configs["colony_3d_f64"]["e2e"]["value"]
        line["summary"] = summ
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
