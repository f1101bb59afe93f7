#!/usr/bin/env python
"""Throughput of Ash3d's transport step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config C2]

One "step" is one reference time step of the transport path through the
C-ABI (src/Ash3d.F90:376-595): step prologue, device met-step interpolation,
Adjust_DT, source insertion, Set_BC(1), AdvectHorz, AdvectVert, Set_BC(2),
DiffuseHorz, DiffuseVert, TimeStepTotals.  The workload is the lon/lat
720x360x60 grid with 10 grain bins, Crank-Nicolson diffusion and hourly FP32
met steps (a 0.25-degree jet plus a meridional wave with seeded 5% noise), on
synthetic data.  The concentration starts from a seeded field that fills the
whole domain, so every cell exercises the limiter.

value  = cell-grain-steps/s with the met steps already on the device.
e2e    = the same through the same public calls, with one met step uploaded
         from pinned host memory inside the timed window (on the copy stream,
         as the loop uploads the step after next at each hour) and dt + totals
         read back every step.
On one GPU the host runs the lag-one loop (driver.Pipeline): the source is
scheduled on the device and dt and the totals are read back behind events,
so the host never waits for the GPU while it queues a step.
N > 1: grains are sharded across GPUs (weak scaling: 10 grains per GPU of a
10*N-grain run); the only exchange is an all-reduce MAX of three CFL maxima
and an all-reduce SUM of the totals per step (NCCL).

Build choices: FAST_DT on (dt from the met steps, interpolated every step:
the reference's default makefile, src/makefile:91) unless --no-fast-dt;
FAST_SUBGRID off (the filled domain's box is the whole grid).

--impl reference times the CPU restatement of the reference (the oracle,
OpenMP in the advection rows as the reference) on the host cores, on the
same full grid, state and build choices: at most 4 timed steps after one
warm-up step (a full-grid CPU step takes ~15 s).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import pathlib
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent


def _load_pkg():
    if "volcano_ash3d_b200" in sys.modules:
        return sys.modules["volcano_ash3d_b200"]
    d = ROOT / "volcano-ash3d_b200"
    spec = importlib.util.spec_from_file_location("volcano_ash3d_b200", d / "__init__.py",
                                                  submodule_search_locations=[str(d)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["volcano_ash3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_pkg()
from volcano_ash3d_b200 import driver, synthetic as syn  # noqa: E402

METRIC = "cell-grain-steps/s FP64"
UNIT = "cell-grain-steps/s"
WORKLOAD = {
    "C2": "lon/lat 720x360x60 (0.25 deg, dz 0.5 km), 10 grains (v_s 1e-3..3 m/s), superbee, "
          "Crank-Nicolson diffusion 500 m^2/s, hourly FP32 met steps (jet + wave + 5% noise)",
    "C1": "projected 100x100x40 (5 km, dz 0.5 km), 4 grains, superbee, explicit diffusion",
    "C4": "projected 200x200x50, 6 grains, superbee, explicit diffusion",
    "C5": "projected 1500x1000x80 (3 km, dz 0.4 km), 20 grains, superbee, Crank-Nicolson",
}


def _load_oracle():
    p = str(ROOT / "oracle")
    if p not in sys.path:
        sys.path.insert(0, p)
    import ash3d_oracle
    ash3d_oracle.build()
    return ash3d_oracle


def filled_state(cfg, seed=17):
    """A seeded concentration filling the whole domain (kg/km^3), (nx,ny,nz,ns)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz, ns = cfg.nx, cfg.ny, cfg.nz, cfg.ns
    x = np.sin(np.linspace(0, 6 * math.pi, nx))[:, None, None]
    y = np.cos(np.linspace(0, 4 * math.pi, ny))[None, :, None]
    z = np.exp(-((np.linspace(0, 1, nz) - 0.4) ** 2) * 4)[None, None, :]
    base = (2.0 + x + y) * z * 100.0
    q = np.empty((nx, ny, nz, ns), order="F")
    for g in range(ns):
        noise = rng.random((nx, ny, nz), dtype=np.float32)
        q[:, :, :, g] = base * (0.2 + 0.1 * g) * (0.9 + 0.2 * noise)
    return q


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic bytes per launch, per kernel class
# ---------------------------------------------------------------------------
def algorithmic_bytes(cfg, kclass: str) -> float:
    cells = cfg.nx * cfg.ny * cfg.nz
    cg = cells * cfg.ns
    table = {
        "advect_x": 16 * cg + 8 * cells, "advect_y": 16 * cg + 8 * cells,
        "advect_z": 16 * cg + 8 * cells, "diff_x": 16 * cg, "diff_y": 16 * cg, "diff_z": 16 * cg,
        "cn_solve_x": 16 * cg, "cn_solve_y": 16 * cg, "cn_solve_z": 16 * cg,
        "cfl": 24 * cells, "totals": 8 * cg, "winds": 48 * cells,
    }
    return float(table.get(kclass, 0.0))


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


def compute_floors(config: str, cell_grains: float):
    """The step's FP64-pipe and instruction-issue floors (ms) on 148 SMs at
    1965 MHz from the committed per-cell-grain instruction counts, or None."""
    p = ROOT / "profiles" / "instruction_mix.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text()).get(config)
    if not d:
        return None
    inst = sum(v["thread_inst_per_cg"] for v in d.values())
    fp64 = sum(v["fp64_inst_per_cg"] for v in d.values())
    sms, hz = 148, 1965e6
    return {"fp64_floor_ms": cell_grains * fp64 / (sms * 64 * hz) * 1e3,
            "issue_floor_ms": cell_grains * inst / 32 / (sms * 4 * hz) * 1e3,
            "thread_inst_per_cell_grain": inst, "fp64_inst_per_cell_grain": fp64,
            "source": "profiles/instruction_mix.json (ncu counters of the C2 slab)"}


def ncu_traffic(config: str, kclass: str):
    """dram read+write bytes per launch from the committed ncu summary."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    v = d.get(config, {}).get(kclass)
    return float(v) if v is not None else None


# ---------------------------------------------------------------------------
# CPU arm: the oracle on a bounded slab of the workload
# ---------------------------------------------------------------------------
def bench_config(args):
    """The workload of both arms: the named configuration with the bench's
    build choices (FAST_DT on unless --no-fast-dt: the reference's default
    build, src/makefile:91) and an optional y-slab for profiling."""
    cfg = syn.make_config(args.config)
    if args.ny:
        cfg.ny = args.ny
        cfg.jvent = max(1, args.ny // 2)
    cfg.limiter = args.limiter
    cfg.fast_dt = not args.no_fast_dt
    return cfg


def cpu_sample(cfg, steps: int, warmup: int):
    """The oracle (the CPU restatement of the reference step, OpenMP on the
    advection rows as the reference has it) on the same grid, state and
    build choices as the GPU arm: `warmup` untimed steps, then `steps` timed
    ones."""
    orc = _load_oracle()
    m = orc.OracleModel(cfg)
    m.set_interior(filled_state(cfg))
    st = driver.new_state(cfg)
    for _ in range(warmup):
        driver.step(m, st)
    t0 = time.perf_counter()
    for _ in range(steps):
        driver.step(m, st)
    el = time.perf_counter() - t0
    value = cfg.cell_grains * steps / el
    threads = orc.load().orc_get_threads()
    sample = (f"oracle port of the reference step on the full grid {cfg.nx}x{cfg.ny}x{cfg.nz}x{cfg.ns}, "
              f"{steps} steps after {warmup} warm-up, {threads} OpenMP threads on the advection rows "
              "(diffusion, Adjust_DT and the sums serial, as in the reference)")
    return value, el, threads, sample


def host_cpu():
    try:
        for ln in pathlib.Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    cfg = bench_config(args)
    # full-grid CPU steps take ~15 s each: the arm times at most 4 of them after
    # one warm-up step so that the run ends within a few minutes
    steps, warmup = min(args.steps, 4), 1
    value, el, threads, sample = cpu_sample(cfg, steps, warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": warmup, "requested_steps": args.steps, "requested_warmup": args.warmup,
        "ms_per_step": 1e3 * el / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.config}: {WORKLOAD[args.config]}", "grid": [cfg.nx, cfg.ny, cfg.nz],
                   "grains": cfg.ns, "fast_dt": cfg.fast_dt, "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "cpu_model": host_cpu(), "same_config": True},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
class NoMetUpload:
    """Model proxy that keeps the resident met pair (the `value` loop)."""

    def __init__(self, model):
        self._m = model

    def set_met_steps(self, last, nxt):
        return None

    def prefetch_met_step(self, step):
        return None

    def advance_met_step(self):
        return None

    def __getattr__(self, name):
        return getattr(self._m, name)


class PinnedMet:
    """Met steps generated before timing, held in pinned host memory."""

    def __init__(self, met: syn.MetSource, hours, torch):
        self.cache = {}
        for h in hours:
            arrs = []
            for a in met.step(h):
                t = torch.empty(a.shape[::-1], dtype=torch.float32, pin_memory=True)
                v = t.numpy().reshape(-1)
                v[:] = np.asarray(a, dtype=np.float32).reshape(-1, order="F")
                arrs.append(v)
            self.cache[h] = tuple(arrs)

    def step(self, h):
        return self.cache[h]


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import torch.distributed as dist
    from volcano_ash3d_b200.model import Ash3dGPU

    torch.cuda.set_device(local_rank)
    comm = None
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
        comm = driver.Comm(device=torch.device("cuda", local_rank))
    cfg_g = bench_config(args)
    cfg = driver.shard_config(cfg_g, rank, world)
    geo = syn.geometry(cfg)
    gpu = Ash3dGPU(cfg, device=local_rank, geo=geo)
    for dv in args.variant:  # kernel variant overrides, "dir=variant"
        d, v = (int(x) for x in dv.split("="))
        gpu.set_variant(d, v)
    gpu.set_interior(filled_state(cfg, seed=17 + rank))
    stream = torch.cuda.ExternalStream(gpu.stream_handle(), device=torch.device("cuda", local_rank))
    n_total = cfg.ns * world

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # the lag-one loop (no host wait while a step is queued); several ranks
    # all-reduce the CFL maxima on the device, in place on the context's
    # stream (with FAST_DT only at met-step loads)
    pipe = driver.Pipeline(gpu, cfg, geo, comm=comm, n_gs_aloft_total=n_total)
    st = pipe.st

    def do_step(m):
        pipe.model = m
        pipe.step()

    for _ in range(args.warmup):
        do_step(gpu)

    # ---- value: met steps resident --------------------------------------
    resident = NoMetUpload(gpu)
    sampler = ClockSampler(local_rank)
    n0 = gpu.kernel_launches()
    barrier()
    torch.cuda.synchronize()
    gpu.sync()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler.start()
    time.sleep(0.3)
    ev0.record(stream)
    for _ in range(args.steps):
        do_step(resident)
    ev1.record(stream)
    gpu.sync()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    launches = gpu.kernel_launches() - n0
    value = cfg.cell_grains * world * args.steps / (ms / 1e3)

    # ---- per-kernel CUDA-event times (same workload, short pass) ---------
    gpu.kernel_timing(True)
    nk = min(args.steps, 5)
    for _ in range(nk):
        do_step(resident)
    ktimes = gpu.kernel_times()
    gpu.kernel_timing(False)

    # ---- e2e: met uploads from pinned memory + per-step H2D/D2H ----------
    # The window holds at least one met-step upload from pinned memory, issued
    # as the loop issues it at an hour boundary: the step after next, on the
    # copy stream, overlapping the steps.  Crossing an hour in the window adds
    # the loop's own advance and prefetch.  The compute stream waits for the
    # copies before the window closes, so they are inside the timed region.
    h0 = max(st.hour, 0)
    pinned = PinnedMet(st.met, range(h0, h0 + 3 + int(args.steps * 0.2)), torch)
    st.met = pinned
    step_bytes_met = 3 * cfg.cells * 4  # one FP32 met step (vx, vy, vz)
    barrier()
    torch.cuda.synchronize()
    gpu.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    uploads = 0
    e0.record(stream)
    gpu.prefetch_met_step(pinned.step(st.met_ahead))
    uploads += 1
    for _ in range(args.steps):
        before = st.hour
        do_step(gpu)
        if st.hour != before:  # an advance and a prefetch, or a pair and a prefetch
            uploads += 1 if before >= 0 else 3
    gpu.met_prefetch_fence()
    e1.record(stream)
    gpu.sync()
    torch.cuda.synchronize()
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = cfg.cell_grains * world * args.steps / (ms_e2e / 1e3)
    met_bytes = step_bytes_met
    # the source is formed on the device; dt and the totals partials come back
    h2d = (uploads * met_bytes) / args.steps
    d2h = 64 + 8 * 7 * cfg.ns

    if rank == 0:
        # dominant kernel and its roofline
        cand = {k: v for k, v in ktimes.items() if k not in ("other",) and v[1] > 0}
        dom = max(cand, key=lambda k: cand[k][0])
        tot_ms, cnt = cand[dom]
        avg_s = tot_ms / cnt / 1e3
        alg = algorithmic_bytes(cfg, dom)
        achieved = alg / avg_s / 1e9
        peak, peak_src = measured_peak()
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": ncu_traffic(args.config, dom),
                "alg_bytes_per_launch": alg, "avg_launch_ms": avg_s * 1e3, "peak_source": peak_src,
                "step_frac": None}
        step_bytes = (48 + 24 / cfg.ns) * cfg.cell_grains if cfg.use_cn else (16 + 24 / cfg.ns) * cfg.cell_grains
        roof["step_frac"] = (step_bytes * args.steps / (ms / 1e3) / 1e9) / peak
        fl = compute_floors(args.config, cfg.cell_grains) if not args.ny else None
        if fl:
            fl["step_ms"] = ms / args.steps
            fl["issue_frac"] = fl["issue_floor_ms"] / fl["step_ms"]
            roof["compute"] = fl
        kt = {k: {"ms": round(v[0] / max(v[1], 1), 4), "launches_per_step": v[1] / nk}
              for k, v in ktimes.items() if v[1] > 0}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            # one full-grid step (~15 s of CPU work) after one warm-up step
            cv, cel, thr, sample = cpu_sample(cfg_g, steps=1, warmup=1)
            cpu = {"value": cv, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample,
                   "cpu_model": host_cpu(), "same_config": True}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded filled concentration, analytic winds with seeded noise)",
            "config": {"workload": f"{args.config}: {WORKLOAD[args.config]}",
                       "grid": [cfg.nx, cfg.ny, cfg.nz], "grains_per_gpu": cfg.ns, "fast_dt": cfg.fast_dt,
                       "grains_total": n_total, "parallelism": f"grain-sharded x{world}",
                       "l2": "inputs larger than L2 (one concentration level is "
                             f"{cfg.cell_grains * 8 / 1e9:.2f} GB)"},
            "roofline": roof,
            "kernel_ms": kt,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e / args.steps,
                    "met_uploads": uploads},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    gpu.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_adjoint(args):
    """Source inversion on C4 (projected 200x200x50, 6 grains, 24 h, explicit
    diffusion) through the library's forward/adjoint pair
    (a3g_forward_checkpointed, a3g_adjoint): control = mass rate per (level,
    hour, grain) = 7200 parameters; observations = hourly column loads of a
    seeded truth (the prior times a lognormal sigma=0.5 perturbation) with 5%
    noise.  Times a plain forward run (one checkpoint slot, so nothing is
    stored), the gradient with every state kept (the budget holds them all)
    and the gradient under a 16-slot budget (binomial recomputation), and
    checks the gradient against central differences on --fd seeded active
    parameters over a sweep of relative steps."""
    import torch
    from volcano_ash3d_b200 import adjoint as adj
    from volcano_ash3d_b200.model import Ash3dGPU
    cfg = syn.make_config("C4")
    hours = int(cfg.sim_hours)
    inv = adj.SourceInversion(cfg, hours=hours)
    gpu = Ash3dGPU(cfg)
    p_true = inv.prior(seed=4, lognormal_sigma=0.5, active_hours=hours)
    level = 8.0 * (-(-cfg.nx // 8) * 8) * cfg.ny * cfg.nz * cfg.ns  # one device level (bytes)
    truth = adj.InversionGPU(gpu, cfg, hours, obs={h: np.zeros((cfg.nx, cfg.ny)) for h in range(hours)},
                             snapshot_bytes=1.5 * level)
    _, loads, _ = truth.forward(p_true)
    obs = {h: loads[h] * (1 + 0.05 * np.random.default_rng(100 + h).standard_normal(loads[h].shape))
           for h in range(hours)}
    p = inv.prior(active_hours=hours)

    def timed(fn):
        torch.cuda.synchronize()
        gpu.sync()
        t0 = time.perf_counter()
        out = fn()
        gpu.sync()
        return out, time.perf_counter() - t0

    plain = adj.InversionGPU(gpu, cfg, hours, obs=obs, snapshot_bytes=1.5 * level)
    plain.forward(p)  # warm-up
    (J, _, _), t_fwd = timed(lambda: plain.forward(p))
    full = adj.InversionGPU(gpu, cfg, hours, obs=obs)
    full.forward(p)
    full.adjoint()  # warm-up (allocates every checkpoint slot)
    (_, t_fwd_ck) = timed(lambda: full.forward(p))
    g, t_adj = timed(lambda: full.adjoint())
    st_full = dict(full.stats)
    tight = adj.InversionGPU(gpu, cfg, hours, obs=obs, snapshot_bytes=16.5 * level)
    tight.forward(p)
    (_, t_fwd16) = timed(lambda: tight.forward(p))
    g16, t_adj16 = timed(lambda: tight.adjoint())
    st16 = dict(tight.stats)
    fd = None
    if args.fd:
        rng = np.random.default_rng(7)
        active = np.argwhere(p > 0)
        picks = [tuple(int(v) for v in active[rng.integers(0, len(active))]) for _ in range(args.fd)]
        sweep = {}
        rels = (1e-3, 1e-4, 1e-5, 1e-6, 1e-7)
        fdv = np.zeros((len(rels), len(picks)))
        for a, rel in enumerate(rels):
            errs = []
            for b, i in enumerate(picks):
                h = rel * p[i]
                pp, pm = p.copy(), p.copy()
                pp[i] += h
                pm[i] -= h
                d = (plain.forward(pp)[0] - plain.forward(pm)[0]) / (2 * h)
                fdv[a, b] = d
                errs.append(abs(g[i] - d) / max(abs(d), 1e-300))
            sweep[f"{rel:g}"] = {"max_rel_err": float(max(errs)), "median_rel_err": float(np.median(errs))}
        best = min(sweep, key=lambda k: sweep[k]["max_rel_err"])
        # a step per parameter chosen without the adjoint: the pair of
        # neighbouring steps (h, h/10) whose central differences agree best
        # (the plateau between the limiter kinks a large step crosses and the
        # rounding a small step amplifies); the smaller step's estimate counts
        per_err, per_step = [], []
        for b, i in enumerate(picks):
            agree = [abs(fdv[a, b] - fdv[a + 1, b]) / max(abs(fdv[a + 1, b]), 1e-300) for a in range(len(rels) - 1)]
            a = int(np.argmin(agree)) + 1
            per_step.append(rels[a])
            per_err.append(abs(g[i] - fdv[a, b]) / max(abs(fdv[a, b]), 1e-300))
        # the exact directional derivative on the run's limiter branches: the
        # tangent-linear run along each parameter, dotted with the residuals
        plain.forward(p)
        res = np.stack([plain.observations()[0][h] - obs[h] for h in range(hours)])
        tl_err = []
        for i in picks:
            e = np.zeros_like(p)
            e[i] = 1.0
            dl, _ = plain.tangent_linear(p, e)
            d_tl = float(np.sum(res * dl))
            tl_err.append(abs(g[i] - d_tl) / max(abs(d_tl), 1e-300))
        fd = {"params": args.fd, "steps_relative": sweep, "chosen_step": best,
              "max_rel_err": sweep[best]["max_rel_err"], "median_rel_err": sweep[best]["median_rel_err"],
              "plateau_step": {"max_rel_err": float(max(per_err)), "median_rel_err": float(np.median(per_err)),
                               "steps": [f"{v:g}" for v in per_step]},
              "tangent_linear_max_rel_err": float(max(tl_err)),
              "note": "central differences against the adjoint gradient; the tangent-linear line is the "
                      "exact derivative on the run's limiter branches, which central differences cross"}
    steps = st_full["steps"]
    line = {
        "metric": "C4 source-inversion gradient wall time", "value": t_fwd_ck + t_adj, "unit": "s",
        "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C4: " + WORKLOAD["C4"] + ", 24 h, 7200 controls, hourly column loads",
                   "grid": [cfg.nx, cfg.ny, cfg.nz], "grains": cfg.ns, "steps": steps,
                   "path": "C-ABI a3g_forward_checkpointed + a3g_adjoint (whole run in the library)"},
        "forward_s": t_fwd, "adjoint_forward_ratio": (t_fwd_ck + t_adj) / t_fwd,
        "checkpointed_forward_s": t_fwd_ck, "reverse_s": t_adj, "checkpoint_slots": st_full["slots"],
        "recomputed_steps": st_full["recomputed"],
        "budget_16_slots": {"gradient_s": t_fwd16 + t_adj16, "ratio": (t_fwd16 + t_adj16) / t_fwd,
                            "recomputed_steps": st16["recomputed"],
                            "same_gradient_bits": bool(np.array_equal(g, g16))},
        "J": J, "forward_cell_grain_steps_per_s": cfg.cell_grains * steps / t_fwd,
        "gradient_norm": float(np.linalg.norm(g)), "fd_check": fd,
        "gpu_launches": int(gpu.kernel_launches()),
    }
    print(json.dumps(line), flush=True)
    gpu.close()


class CachedMet:
    """Every met step of a run generated once, by a thread pool (numpy
    releases the interpreter lock in the generator's fills and array
    arithmetic), and kept in host memory; an all-zero vz is shared."""

    def __init__(self, cfg, nsteps: int, threads: int = 8):
        import concurrent.futures as cf
        src = syn.MetSource(cfg)
        self.zero = None
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            steps = list(ex.map(src.step, range(nsteps)))
        self.steps = []
        for u, v, w in steps:
            if not w.any():
                if self.zero is None:
                    self.zero = w
                w = self.zero
            self.steps.append((u, v, w))

    def step(self, hour: int):
        return self.steps[hour]


def run_adjoint_scale(args):
    """C5: projected 1500x1000x80 (3 km, dz 0.4 km), 20 grains, superbee, CN,
    FAST_DT: the forward run of --hours simulated hours (default 48) through
    the library's checkpointed forward, then the adjoint of the deposit misfit
    over the last --adj-hours (default 12).  Control: the vent column's mass
    rate per (level, hour, grain), the Suzuki column for a 25 km plume over 12
    h with seeded heavy-tailed (Pareto) hourly rates.  Observation: a seeded
    Gaussian deposit pattern downwind of the vent.  Checkpoints: device memory
    only, every byte left after the run's buffers but 2 GiB (the library's
    default budget), binomial placement over the reversal window."""
    import ctypes as C
    import torch
    from volcano_ash3d_b200 import _lib
    from volcano_ash3d_b200 import adjoint as adj
    from volcano_ash3d_b200.model import Ash3dGPU
    cfg = syn.make_config("C5")
    hours = int(args.hours) if args.hours > 1.0 else int(cfg.sim_hours)
    win = min(int(args.adj_hours), hours - 1)
    cfg.sim_hours = float(hours)
    cfg.fast_dt = not args.no_fast_dt
    cfg.fast_subgrid = False  # the inversion runs the full box
    t0 = time.perf_counter()
    met = CachedMet(cfg, hours + 2)
    t_met = time.perf_counter() - t0
    gpu = Ash3dGPU(cfg)
    prior = adj.SourceInversion(cfg, hours, geo=gpu.geo)
    p = prior.prior(active_hours=cfg.duration_h)
    rng = np.random.default_rng(55)
    rate = 1.0 + rng.pareto(1.5, hours)
    rate = rate / rate[:int(cfg.duration_h)].mean()
    p = p * rate[None, :, None]
    ii, jj = np.meshgrid(np.arange(cfg.nx), np.arange(cfg.ny), indexing="ij")
    x0, y0 = cfg.ivent + rng.uniform(100, 300), cfg.jvent + rng.uniform(-50, 50)
    obs_dep = 1.0 * np.exp(-0.5 * (((ii - x0) / 150.0) ** 2 + ((jj - y0) / 40.0) ** 2))

    def timed(fn):
        torch.cuda.synchronize()
        gpu.sync()
        t = time.perf_counter()
        out = fn()
        gpu.sync()
        return out, time.perf_counter() - t

    free0, total = torch.cuda.mem_get_info()
    (inv, t_setup) = timed(lambda: adj.InversionGPU(gpu, cfg, hours, obs_dep=obs_dep, nbins=hours,
                                                    dep_from=hours - win, adj_from=hours - win,
                                                    fast_dt=cfg.fast_dt, met=met, met_cache=False))
    (J, _, dep), t_fwd = timed(lambda: inv.forward(p))
    g, t_adj = timed(lambda: inv.adjoint())
    st = dict(inv.stats)
    free1, _ = torch.cuda.mem_get_info()
    steps, wsteps = st["steps"], st["window_steps"]
    lib = _lib.load()
    ms_fwd = 1000.0 * t_fwd / steps
    rec = C.c_int64()
    lib.a3g_checkpoint_cost(max(wsteps, 1), max(st["slots"] - 1, 0), C.byref(rec), None)
    level = 8.0 * cfg.nx * cfg.ny * cfg.nz * cfg.ns
    line = {
        "metric": "C5 deposit-misfit adjoint wall time", "value": t_adj, "unit": "s", "higher_is_better": False,
        "n_gpus": 1, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"C5: projected 1500x1000x80, 20 grains, superbee, CN, "
                               f"{'FAST_DT' if cfg.fast_dt else 'Adjust_DT every step'}, forward {hours} h, "
                               f"adjoint of the deposit misfit over the last {win} h",
                   "grid": [cfg.nx, cfg.ny, cfg.nz], "grains": cfg.ns, "controls": int(p.size),
                   "path": "C-ABI a3g_forward_checkpointed / a3g_adjoint"},
        "forward_s": t_fwd, "forward_ms_per_step": ms_fwd, "setup_s": t_setup, "met_generation_s": t_met,
        "steps": steps, "slots": st["slots"], "slot_gb": level / 1e9,
        "checkpoint_gb": st["slots"] * level / 1e9, "recomputed_steps": st["recomputed"],
        "recomputed_predicted": int(rec.value), "window_steps": wsteps,
        "adjoint_over_window_forward": t_adj / (ms_fwd * wsteps / 1000.0),
        "device_free_gb_before": free0 / 1e9, "device_free_gb_after": free1 / 1e9, "device_total_gb": total / 1e9,
        "J": J, "grad_abs_max": float(np.abs(g).max()), "grad_finite": bool(np.isfinite(g).all()),
        "grad_nonzero_bins": int(np.count_nonzero(np.abs(g).sum(axis=(0, 2)))),
    }
    print(json.dumps(line), flush=True)
    gpu.close()


def run_ensemble(args):
    """C3: 64 seeded members (nx, ny in [80,400], nz in [30,80], 2-10 grains,
    CN), each run for --hours simulated hours from a clean atmosphere, first
    one after another (the single-member path), then concurrently (one
    context, stream and host thread per member), both after a per-member
    variant autotune."""
    from volcano_ash3d_b200 import ensemble as ens
    cfgs = ens.c3_members(64, seed=3, hours=args.hours)
    t0 = time.perf_counter()
    e = ens.Ensemble(cfgs, tune=True)
    t_tune = time.perf_counter() - t0
    e.run_concurrent(min(args.hours, 0.1))  # warm-up: first launches, allocations
    seq, t_seq = e.run_sequential(args.hours)
    con, t_con = e.run_concurrent(args.hours)
    work = sum(r.cell_grain_steps for r in con)
    assert [r.steps for r in seq] == [r.steps for r in con]
    line = {
        "metric": "C3 ensemble cell-grain-steps/s FP64", "value": work / t_con, "unit": "cell-grain-steps/s",
        "higher_is_better": True, "n_gpus": 1, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"C3: 64 members, {args.hours} h each, CN, superbee, autotuned variants",
                   "members": len(cfgs), "cell_grains_total": int(sum(c.cell_grains for c in cfgs)),
                   "steps_total": int(sum(r.steps for r in con))},
        "speedup_vs_sequential": t_seq / t_con, "sequential_s": t_seq, "concurrent_s": t_con,
        "sequential_value": work / t_seq, "autotune_s": t_tune,
        "variant_counts": {str(k): {str(v): sum(1 for m in e.variants if m.get(k) == v) for v in range(8)
                                    if any(m.get(k) == v for m in e.variants)} for k in range(5)},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="C2", choices=sorted(WORKLOAD))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fast-dt", action="store_true",
                    help="Adjust_DT every step instead of FAST_DT (the reference's default build)")
    ap.add_argument("--limiter", default="superbee",
                    choices=["none", "laxwen", "bw", "fromm", "minmod", "superbee", "mc"],
                    help="the reference's LIM_* build choice (default superbee)")
    ap.add_argument("--ny", type=int, default=0,
                    help="run a y-slab of the workload with this many rows (profiling case)")
    ap.add_argument("--adjoint", action="store_true",
                    help="time the C4 source-inversion gradient instead of the forward step")
    ap.add_argument("--fd", type=int, default=0,
                    help="with --adjoint: central-difference checks on this many parameters")
    ap.add_argument("--ensemble", action="store_true",
                    help="time the 64-member C3 ensemble, sequential and concurrent")
    ap.add_argument("--hours", type=float, default=1.0,
                    help="with --ensemble: simulated hours per member; with --config C5 --adjoint: the "
                         "forward run's hours (default 48)")
    ap.add_argument("--adj-hours", type=float, default=12.0,
                    help="with --config C5 --adjoint: the reversal window (the last hours of the run)")
    ap.add_argument("--variant", action="append", default=[], metavar="DIR=V",
                    help="kernel variant override (a3g_set_variant), repeatable")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.adjoint:
        if args.config == "C5":
            run_adjoint_scale(args)
        else:
            run_adjoint(args)
        return
    if args.ensemble:
        run_ensemble(args)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
