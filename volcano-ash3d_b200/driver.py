"""The time loop of src/Ash3d.F90:372-642, restricted to the transport path.

``run`` drives any model object that exposes the reference routine names
(``Ash3dGPU`` here; the oracle in the test suite offers the same names), in
the reference's order:

  prologue (ts0 <- ts1, :376-378) -> MesoInterpolater (FP32 met steps,
  device interpolation, :396) -> Adjust_DT -> CheckEruptivePulses + source
  insertion (:407-434) -> Set_BC(1) -> AdvectHorz(itime) -> AdvectVert ->
  [Set_BC(2) -> DiffuseHorz(itime) -> DiffuseVert] -> time += dt ->
  TimeStepTotals (every log step, :568-595) -> stop tests (:597-641).

Met steps are hourly; the next pair is uploaded when the simulation clock
crosses an hour, as Read_NextMesoStep does (src/MesoInterpolater.f90:169-197).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import synthetic as syn


@dataclasses.dataclass
class StepRecord:
    itime: int
    time: float
    dt: float
    aloft: float
    dep: float
    outflow: float
    tot: float
    source_cum: float


@dataclasses.dataclass
class RunState:
    cfg: syn.Config
    time: float = 0.0
    itime: int = 0
    hour: int = -1
    source_cum: float = 0.0
    norm_col: np.ndarray = None
    kappa: np.ndarray = None
    met: syn.MetSource = None
    history: list = dataclasses.field(default_factory=list)
    umbrella: syn.UmbrellaSetup = None
    prev_dt: float = None    # time_data::dt when MesoInterpolater runs (the previous step's)
    met_ahead: int = -1      # the hour whose met step was prefetched into the spare slot


def new_state(cfg: syn.Config, geo: dict | None = None) -> RunState:
    geo = geo if geo is not None else syn.geometry(cfg)
    um = syn.umbrella_setup(cfg, geo["kappa"]) if syn.is_umbrella(cfg) else None
    return RunState(cfg=cfg, norm_col=syn.suzuki_column(cfg), kappa=geo["kappa"],
                    met=syn.MetSource(cfg), umbrella=um)


class Comm:
    """The two reductions a grain-sharded run needs (torch.distributed
    all-reduces of a few doubles): MAX of the CFL maxima, SUM of the totals."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group, self.device = torch, dist, group, device

    def _reduce(self, a: np.ndarray, op) -> np.ndarray:
        t = self.torch.tensor(np.asarray(a, dtype=np.float64), device=self.device)
        self.dist.all_reduce(t, op=op, group=self.group)
        return t.cpu().numpy()

    def max(self, a):
        return self._reduce(a, self.dist.ReduceOp.MAX)

    def max_inplace(self, buf):
        """MAX all-reduce of ``buf`` in place, with no host read-back: a numpy
        array (a CPU group), or device memory with __cuda_array_interface__
        and the `stream` its producer was queued on (model.cfl_maxima_device),
        in which case the collective is ordered on that stream and the
        stream's later work waits for it."""
        torch = self.torch
        t = torch.as_tensor(buf) if isinstance(buf, np.ndarray) else torch.as_tensor(buf, device=self.device)
        stream = getattr(buf, "stream", None)
        if t.is_cuda and stream is not None:
            with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=t.device)):
                self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
        else:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)

    def sum(self, a):
        return self._reduce(a, self.dist.ReduceOp.SUM)

    # --- per-rank grain blocks (the last axis of ashcon / depocon) -----------
    def _world(self):
        return self.dist.get_rank(self.group), self.dist.get_world_size(self.group)

    def _peer(self, r: int) -> int:
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def _empty(self, n: int, dtype):
        tdt = self.torch.from_numpy(np.empty(0, dtype=dtype)).dtype
        return self.torch.empty(n, dtype=tdt, device=self.device)

    def gather_grains(self, arr: np.ndarray, ns_total: int, root: int = 0):
        """The full array on ``root`` from every rank's block of grain bins
        (the last axis, blocks in rank order as split_grains deals them),
        Fortran order; None on the other ranks.  Point-to-point sends, one
        per non-root rank."""
        rank, world = self._world()
        shape = arr.shape[:-1]
        if rank != root:
            t = self.torch.from_numpy(np.ascontiguousarray(arr.ravel(order="F"))).to(self.device)
            self.dist.send(t, dst=self._peer(root), group=self.group)
            return None
        out = np.empty(shape + (ns_total,), dtype=arr.dtype, order="F")
        for r in range(world):
            lo, hi = grain_range(ns_total, r, world)
            if r == root:
                out[..., lo:hi] = arr
                continue
            t = self._empty(int(np.prod(shape)) * (hi - lo), arr.dtype)
            self.dist.recv(t, src=self._peer(r), group=self.group)
            out[..., lo:hi] = t.cpu().numpy().reshape(shape + (hi - lo,), order="F")
        return out

    def scatter_grains(self, full, shape: tuple, dtype, ns_total: int, root: int = 0) -> np.ndarray:
        """This rank's block of grain bins of ``full`` (given on ``root``;
        ``shape`` is its shape without the grain axis on every rank)."""
        rank, world = self._world()
        lo, hi = grain_range(ns_total, rank, world)
        if rank == root:
            for r in range(world):
                if r != root:
                    a, b = grain_range(ns_total, r, world)
                    blk = np.asarray(full, dtype=dtype)[..., a:b].ravel(order="F")
                    self.dist.send(self.torch.from_numpy(np.ascontiguousarray(blk)).to(self.device),
                                   dst=self._peer(r), group=self.group)
            return np.asfortranarray(np.asarray(full, dtype=dtype)[..., lo:hi])
        t = self._empty(int(np.prod(shape)) * (hi - lo), dtype)
        self.dist.recv(t, src=self._peer(root), group=self.group)
        return np.asfortranarray(t.cpu().numpy().reshape(tuple(shape) + (hi - lo,), order="F"))


def shard_config(cfg: syn.Config, rank: int, world: int) -> syn.Config:
    """Grain sharding: the global run has ns*world grain bins (fall speeds
    log-spaced over the global range, equal mass fractions); rank r keeps
    bins r, r+world, r+2*world, ...  Dealing the bins round-robin gives every
    rank the same spread of fall speeds, so the fast-settling bins, which
    leave the domain early and stop costing anything, are spread over the
    ranks instead of idling the last ones.  Every operator acts on grains
    independently, so only dt (a MAX over all grains' settling speeds) and
    the totals couple ranks."""
    if world == 1:
        return cfg
    ns = cfg.ns
    lo, hi = min(cfg.fall_mps), max(cfg.fall_mps)
    fall = np.logspace(math.log10(lo), math.log10(hi), ns * world)
    c = dataclasses.replace(cfg)
    c.fall_mps = tuple(float(v) for v in fall[rank::world])
    c.bin_mass = tuple(1.0 / (ns * world) for _ in range(ns))
    return c


def split_grains(cfg: syn.Config, rank: int, world: int) -> syn.Config:
    """Strong split of one run's grain bins over ``world`` ranks: rank r keeps
    a contiguous block of bins (the first ``ns % world`` ranks one more), with
    the global run's fall speeds and mass fractions unchanged, so the union of
    the ranks' fields is the single-process run's field."""
    if world == 1:
        return cfg
    if cfg.ns < world:
        raise ValueError(f"{cfg.ns} grain bins cannot be split over {world} ranks")
    base, extra = divmod(cfg.ns, world)
    lo = rank * base + min(rank, extra)
    n = base + (1 if rank < extra else 0)
    c = dataclasses.replace(cfg)
    c.ns = n
    c.fall_mps = tuple(cfg.fall_mps[lo:lo + n])
    c.bin_mass = tuple(cfg.bin_mass[lo:lo + n])
    return c


def grain_range(ns: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of the global grain bins that split_grains gives ``rank``."""
    base, extra = divmod(ns, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_netcdf(model, comm: Comm, ns_total: int, root: int = 0):
    """(ashcon, depocon) of the whole grain-sharded run on ``root`` (None
    elsewhere): each rank forms its bins' arrays on its device
    (a3g_output_ashcon) and root places them at the rank's bin offset."""
    ash, dep = model.output_ashcon()
    return comm.gather_grains(ash, ns_total, root), comm.gather_grains(dep, ns_total, root)


def scatter_restart(model, comm: Comm, cfg: syn.Config, ns_total: int, ashcon=None, depocon=None,
                    root: int = 0):
    """NC_RestartFile_LoadConcen for a grain-sharded run: ``root`` holds the
    file's arrays; every rank loads its own bins (a3g_restart_load)."""
    a = comm.scatter_grains(ashcon, (cfg.nx, cfg.ny, cfg.nz), np.float32, ns_total, root)
    d = comm.scatter_grains(depocon, (cfg.nx, cfg.ny), np.float32, ns_total, root)
    model.restart_load(a, d)


def next_write_time(write_times, time: float) -> float:
    """NextWriteTime: the first output time still ahead (Output_Results.f90:
    183-189), or 1/EPS_SMALL once none is left."""
    for t in write_times or ():
        if t > time + 1.0e-5:  # within DT_MIN of it: that output is done
            return float(t)
    return 1.0 / 1.0e-6


def met_interval(time: float, hour: int) -> int:
    """MR_iMetStep_Now at `time` after interval `hour` (-1 before the first
    call), hourly met steps: the interval holding the time at the first call
    (H(i) <= t < H(i+1), src/MesoInterpolater.f90:122-129), then one interval
    ahead whenever the time has moved strictly past the interval's end
    (t > H(now+1), :135-145), so a time landing exactly on an hour still
    interpolates the old pair at Interval_Frac = 1."""
    if hour < 0:
        return int(math.floor(time))
    return hour + 1 if time > hour + 1 else hour


def met_hour(st: RunState) -> int:
    """met_interval for a run's state."""
    return met_interval(st.time, st.hour)


def update_met(model, st: RunState, h: int):
    """The met pair for hour h.  Crossing into the next hour advances onto the
    step prefetched an hour earlier (Read_NextMesoStep's toggle,
    src/MesoInterpolater.f90:168-199); any other jump uploads the pair.  The
    step after next is then prefetched on the copy stream.  Returns "advance",
    "pair" or None (no load)."""
    if h == st.hour:
        return None
    if st.hour >= 0 and h == st.hour + 1 and st.met_ahead == h + 1:
        model.advance_met_step()
        loaded = "advance"
    else:
        model.set_met_steps(st.met.step(h), st.met.step(h + 1))
        loaded = "pair"
    st.hour = h
    model.prefetch_met_step(st.met.step(h + 2))
    st.met_ahead = h + 2
    return loaded


def meso_dt(model, st: RunState, loaded: str, next_write_time: float, simtime: float,
            comm: Comm | None = None, n_gs_aloft_total: int | None = None, wait: bool = True):
    """FAST_DT's Adjust_DT(mesostep=.true.) calls at a met-step load
    (src/MesoInterpolater.f90:142-150 on the first load: the last step, then
    dt_meso_last = dt_meso_next and the next step; :187-195 at every later
    load: dt_meso_last = dt_meso_next, then the next step).  A grain-sharded
    run takes the maxima's MAX over the ranks once per load; the per-step dt
    then needs no exchange."""
    loads = ((0, False), (1, True)) if loaded == "pair" else ((1, True),)
    for slot, shift in loads:
        if comm is None:
            model.adjust_dt_meso(slot, shift, st.time, next_write_time, simtime, wait=wait)
        else:
            vmax = comm.max(model.cfl_maxima_meso(slot))
            model.adjust_dt_meso_from_maxima(vmax, n_gs_aloft_total, shift, st.time, next_write_time, simtime)


def step(model, st: RunState, simtime: float | None = None, totals: bool = True,
         comm: Comm | None = None, n_gs_aloft_total: int | None = None,
         write_times=None) -> StepRecord:
    """Advances the model by one reference time step.  dt is clipped to the
    next of write_times (the control file's output times), when given, and to
    simtime."""
    cfg = st.cfg
    simtime = cfg.sim_hours if simtime is None else simtime
    nwt = next_write_time(write_times, st.time) if write_times is not None else simtime
    st.itime += 1
    model.step_prologue()
    h = met_hour(st)
    loaded = update_met(model, st, h)
    if cfg.fast_dt and loaded:
        meso_dt(model, st, loaded, nwt, simtime, comm, n_gs_aloft_total)
    frac = st.time - h  # Interval_Frac (hourly met steps)
    model.interp_winds(frac)

    def adjust_dt():
        if comm is None:
            return model.Adjust_DT(st.time, nwt, simtime)
        vmax = comm.max(model.cfl_maxima())
        return model.adjust_dt_from_maxima(vmax, n_gs_aloft_total, st.time, nwt, simtime)

    def fast_dt():
        return model.fast_dt(frac, st.time, nwt, simtime)

    # FastDt_suppress while the umbrella spreads (src/MesoInterpolater.f90:233-248)
    suppress = st.umbrella is not None and st.time < cfg.duration_h
    if suppress:
        if st.prev_dt is None:
            # before the time loop MesoInterpolater ran on the winds without
            # the umbrella's (e_EndTime is still 0 then, src/Ash3d.F90:301,354),
            # so its dt is the FAST_DT one when FAST_DT is on
            st.prev_dt = fast_dt() if cfg.fast_dt else adjust_dt()
        w = syn.umbrella_winds(cfg, st.time, st.prev_dt)
        if w is not None:
            model.add_umbrella_winds(*w)
    dt = fast_dt() if (cfg.fast_dt and not suppress) else adjust_dt()
    st.prev_dt = dt
    frac = syn.pulse_fraction(cfg, st.time, dt)
    if frac > 0.0:
        flux = syn.source_flux(cfg, st.norm_col, st.kappa, frac)
        if st.umbrella is not None:
            model.add_source_umbrella(syn.umbrella_flux(cfg, flux, st.umbrella), dt)
            st.source_cum = st.source_cum + syn.umbrella_vol_inc(cfg, flux, st.umbrella, st.kappa, dt)
        else:
            model.add_source(flux, dt)
            st.source_cum = st.source_cum + syn.source_vol_inc(cfg, flux, st.kappa, dt)
    model.Set_BC(1)
    model.AdvectHorz(st.itime)
    model.AdvectVert()
    if cfg.use_diffusion:
        model.Set_BC(2)
        model.DiffuseHorz(st.itime)
        model.DiffuseVert()
    st.time = st.time + dt
    rec = StepRecord(st.itime, st.time, dt, 0.0, 0.0, 0.0, 0.0, st.source_cum)
    if totals:
        vols, _ = model.TimeStepTotals()
        if comm is not None:
            vols = comm.sum(vols)
            rec.source_cum = float(comm.sum(np.array([st.source_cum]))[0])
        rec.aloft, rec.dep, rec.outflow, rec.tot = (float(v) for v in vols)
    st.history.append(rec)
    return rec


class Pipeline:
    """Lag-one host loop for the GPU model: the same operator sequence as
    step(), but no call waits for the GPU while a step is being queued.  dt
    stays on the device (Adjust_DT, the scheduled source and the sweeps read
    it there); the host reads it back after queuing the whole step, waiting
    only for the early Adjust_DT copy while the GPU runs the step's sweeps,
    and needs it for the next step's time.  The totals of a step are
    collected after the next step is queued.  The host mirrors the source
    arithmetic for SourceCumulativeVol once it knows dt.  Vent-column
    sources, FAST_SUBGRID off (the subgrid box needs the state on the host
    every step).

    With ``comm`` (a grain-sharded run) the CFL maxima are all-reduced on the
    device, in place and ordered on the context's stream
    (model.cfl_maxima_device, Comm.max_inplace,
    model.adjust_dt_device_maxima_async), so the loop still queues each step
    without waiting; with FAST_DT they are exchanged only at met-step loads.
    The totals and SourceCumulativeVol are summed over the ranks when a step's
    record is collected."""

    def __init__(self, model, cfg: syn.Config, geo: dict | None = None, comm: Comm | None = None,
                 n_gs_aloft_total: int | None = None):
        if cfg.fast_subgrid or syn.is_umbrella(cfg):
            raise ValueError("the pipelined loop needs FAST_SUBGRID off and a vent-column source")
        self.model, self.cfg = model, cfg
        self.comm = comm
        self.n_total = cfg.ns if n_gs_aloft_total is None else n_gs_aloft_total
        self.st = new_state(cfg, geo)
        self.pulses = syn.eruption_pulses(cfg)
        model.set_source_pulses(cfg.ivent, cfg.jvent, self.pulses, self.st.norm_col)
        self.state = [1, 1]      # ieruption, jeruption (host mirror of the device's)
        self.pending = None      # (record, totals ticket) of the previous step

    def step(self, simtime: float | None = None, totals: bool = True, write_times=None) -> StepRecord:
        m, cfg, st = self.model, self.cfg, self.st
        simtime = cfg.sim_hours if simtime is None else simtime
        nwt = next_write_time(write_times, st.time) if write_times is not None else simtime
        st.itime += 1
        m.step_prologue()
        h = met_hour(st)
        loaded = update_met(m, st, h)
        if cfg.fast_dt and loaded:
            meso_dt(m, st, loaded, nwt, simtime, self.comm, self.n_total, wait=False)
        frac = st.time - h
        m.interp_winds(frac)
        if cfg.fast_dt:
            m.fast_dt_async(frac, st.time, nwt, simtime)
        elif self.comm is None:
            m.adjust_dt_async(st.time, nwt, simtime)
        else:
            self.comm.max_inplace(m.cfl_maxima_device())
            m.adjust_dt_device_maxima_async(self.n_total, st.time, nwt, simtime)
        m.add_source_scheduled(st.time)
        m.Set_BC(1)
        m.AdvectHorz(st.itime)
        m.AdvectVert()
        if cfg.use_diffusion:
            m.Set_BC(2)
            m.DiffuseHorz(st.itime)
            m.DiffuseVert()
        ticket = m.totals_async() if totals else None
        self._collect()
        dt = m.wait_dt()
        flux = syn.scheduled_source_flux(cfg, self.pulses, st.norm_col, st.kappa, self.state, st.time, dt)
        if flux is not None:
            st.source_cum = st.source_cum + syn.source_vol_inc(cfg, flux, st.kappa, dt)
        st.time = st.time + dt
        rec = StepRecord(st.itime, st.time, dt, 0.0, 0.0, 0.0, 0.0, st.source_cum)
        st.history.append(rec)
        self.pending = (rec, ticket) if totals else None
        return rec

    def _collect(self):
        if self.pending is not None:
            rec, ticket = self.pending
            vols, _ = self.model.totals_get(ticket)
            if self.comm is not None:  # one SUM of the totals and SourceCumulativeVol
                s = self.comm.sum(np.append(np.asarray(vols, dtype=np.float64), rec.source_cum))
                vols, rec.source_cum = s[:4], float(s[4])
            rec.aloft, rec.dep, rec.outflow, rec.tot = (float(v) for v in vols)
            self.pending = None

    def flush(self) -> RunState:
        """Fills the last step's totals; returns the run state."""
        self._collect()
        return self.st


def run_pipelined(model, cfg: syn.Config, max_steps: int | None = None, sim_hours: float | None = None,
                  geo: dict | None = None, totals: bool = True, comm: Comm | None = None,
                  n_gs_aloft_total: int | None = None) -> RunState:
    """run() through the lag-one loop (Pipeline)."""
    p = Pipeline(model, cfg, geo, comm, n_gs_aloft_total)
    simtime = cfg.sim_hours if sim_hours is None else sim_hours
    while p.st.time < simtime and (max_steps is None or p.st.itime < max_steps):
        p.step(simtime, totals)
    return p.flush()


def run(model, cfg: syn.Config, max_steps: int | None = None, sim_hours: float | None = None,
        geo: dict | None = None, totals: bool = True, comm: Comm | None = None,
        n_gs_aloft_total: int | None = None) -> RunState:
    """Runs until sim_hours (or max_steps) like the reference's stop test 2.
    With ``comm`` (a grain-sharded run), dt comes from the all-reduced CFL
    maxima and the totals are summed over ranks; every rank takes the same
    number of steps because every rank gets the same dt."""
    st = new_state(cfg, geo)
    simtime = cfg.sim_hours if sim_hours is None else sim_hours
    while st.time < simtime and (max_steps is None or st.itime < max_steps):
        step(model, st, simtime, totals, comm, n_gs_aloft_total)
    return st
