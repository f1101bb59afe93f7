"""Source inversion by the discrete adjoint of the transport step.

No counterpart in the reference: Ash3d runs forward only.  The control is
the erupted mass rate per (model level, hour, grain bin), inserted at the
vent column the way src/Ash3d.F90:428-431 inserts SourceNodeFlux:
concen(ivent,jvent,k,g) += dt * p(k,h,g) / kappa(ivent,jvent,k).  The
observations are hourly unmasked column loads (CloudLoad of
src/Output_Vars.f90:1061-1069), and the misfit is
J(p) = 1/2 sum_h |H c(t_h) - y_h|^2.

The gradient is one forward run that stores the state every K steps and one
reverse sweep: per segment of K steps the forward states are recomputed from
the checkpoint (the transport is nonlinear through the limiter, so the
reverse sweep needs each step's state), then the steps are reversed with the
model's adj_step.  dt depends only on the winds, so it is recorded in the
forward run and replayed, not differentiated.

Every model call goes through the same method names on the GPU model
(Ash3dGPU, state and lam on the device) and on the oracle (tests only).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import synthetic as syn


@dataclasses.dataclass
class StepLog:
    itime: int
    time: float
    dt: float
    hour: int
    obs_hour: int  # hour whose observation this step ends on, or -1


class SourceInversion:
    """A source-inversion problem on one configuration."""

    def __init__(self, cfg: syn.Config, hours: int, geo: dict | None = None):
        self.cfg = cfg
        self.hours = hours
        self.geo = geo if geo is not None else syn.geometry(cfg)
        kap = self.geo["kappa"]
        # kappa at the vent column, levels 1..nz (ghosted array index +1)
        self.kappa_col = np.array([kap[cfg.ivent + 1, cfg.jvent + 1, k + 1] for k in range(1, cfg.nz + 1)])
        self.met = syn.MetSource(cfg)
        self._met_hour = {}

    @property
    def shape(self):
        return (self.cfg.nz, self.hours, self.cfg.ns)

    def prior(self, seed: int = 0, lognormal_sigma: float = 0.0,
              active_hours: float | None = None) -> np.ndarray:
        """Mass rate (kg/h) per level, hour, grain: the reference's Suzuki
        column for the configuration's plume, times the grain mass fraction,
        for the hours of the eruption (active_hours, default the
        configuration's duration); optionally perturbed lognormally."""
        cfg = self.cfg
        col = syn.suzuki_column(cfg)[:cfg.nz]
        rate = syn.mass_flux_rate(cfg)
        active = cfg.duration_h if active_hours is None else active_hours
        p = np.zeros(self.shape)
        for h in range(self.hours):
            if h < active:
                for g in range(cfg.ns):
                    p[:, h, g] = rate * cfg.bin_mass[g] * col
        if lognormal_sigma > 0.0:
            rng = np.random.default_rng(seed)
            p = p * np.exp(lognormal_sigma * rng.standard_normal(p.shape))
        return p

    def flux(self, p: np.ndarray, hour: int) -> np.ndarray:
        """SourceNodeFlux (nz+1) x ns for the given hour bin."""
        cfg = self.cfg
        f = np.zeros((cfg.nz + 1, cfg.ns), order="F")
        if 0 <= hour < self.hours:
            f[:cfg.nz, :] = p[:, hour, :] / self.kappa_col[:, None]
        return f

    def _winds(self, model, time: float):
        h = int(math.floor(time))
        if getattr(model, "_inv_met_hour", None) != h:
            model.set_met_steps(self.met.step(h), self.met.step(h + 1))
            model._inv_met_hour = h
        model.interp_winds(time - h)

    # ------------------------------------------------------------------
    def _step_ops(self, model, itime: int):
        model.Set_BC(1)
        model.AdvectHorz(itime)
        model.AdvectVert()
        if self.cfg.use_diffusion:
            model.Set_BC(2)
            model.DiffuseHorz(itime)
            model.DiffuseVert()

    def forward(self, model, p: np.ndarray, obs: dict | None = None, K: int = 0):
        """Runs hours of transport from a clean atmosphere.  Returns
        (J, loads, logs, residuals); with K > 0 the state at the start of
        every K-th step n is kept in snapshot slot K + n // K (slots 0..K-1
        hold a segment's recomputed states during the reverse sweep)."""
        cfg = self.cfg
        model.set_interior(np.zeros((cfg.nx, cfg.ny, cfg.nz, cfg.ns), order="F"))
        model._inv_met_hour = None
        time, itime = 0.0, 0
        logs, loads, resid = [], {}, {}
        J = 0.0
        simtime = float(self.hours)
        while time < simtime - 1e-12:
            itime += 1
            model.step_prologue()
            self._winds(model, time)
            next_obs = math.floor(time + 1e-12) + 1.0
            # dt stays on the device while the step is queued; the host reads
            # it once the step's sweeps are on the stream (lag-one loop)
            model.adjust_dt_async(time, next_obs, simtime)
            hour = int(math.floor(time + 1e-12))
            if K:
                n = itime - 1
                if n % K == 0:
                    model.snapshot_alloc(K + n // K + 1)
                    model.snapshot_save(K + n // K)
            model.add_source_devdt(self.flux(p, hour))
            self._step_ops(model, itime)
            dt = model.wait_dt()
            time = time + dt
            ob = -1
            if abs(time - round(time)) < 1e-9 and round(time) >= 1:
                ob = int(round(time)) - 1
                load = model.cloud_load()
                loads[ob] = load
                if obs is not None and ob in obs:
                    r = load - obs[ob]
                    resid[ob] = r
                    J += 0.5 * float(np.sum(r * r))
            logs.append(StepLog(itime, time - dt, dt, hour, ob))
        return J, loads, logs, resid

    def gradient(self, model, p: np.ndarray, obs: dict, K: int = 32):
        """J(p) and dJ/dp (shape (nz, hours, ns)) by checkpointed reverse
        sweep."""
        cfg = self.cfg
        J, loads, logs, resid = self.forward(model, p, obs, K=K)
        N = len(logs)
        nseg = (N + K - 1) // K
        model.adj_enable()
        model.adj_zero()
        model.adj_grad_reset(self.hours)  # gathered on the device, read back once
        for seg in range(nseg - 1, -1, -1):
            n0, n1 = seg * K, min(N, seg * K + K)
            # recompute the segment, keeping each step's post-source state
            model.snapshot_load(K + seg)
            for n in range(n0, n1):
                lg = logs[n]
                if n > n0:
                    model.step_prologue()
                self._winds(model, lg.time)
                model.set_dt(lg.dt)
                model.add_source(self.flux(p, lg.hour), lg.dt)
                model.snapshot_save(n - n0)
                if n < n1 - 1:
                    self._step_ops(model, lg.itime)
            # reverse
            for n in range(n1 - 1, n0 - 1, -1):
                lg = logs[n]
                if lg.obs_hour in resid:
                    model.adj_add_cloud_load(resid[lg.obs_hour])
                model.snapshot_load(n - n0)
                self._winds(model, lg.time)
                model.set_dt(lg.dt)
                model.adj_step(lg.itime)
                if 0 <= lg.hour < self.hours:
                    # grad[:, hour, :] += dt * lam_vent / kappa, in step order
                    model.adj_vent_accumulate(lg.hour, lg.dt)
        return J, model.adj_grad_get()
