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

``SourceInversion`` is that loop on the host, one model call at a time (the
restatement the oracle runs); ``InversionGPU`` is the same run through the
C-ABI pair a3g_forward_checkpointed / a3g_adjoint, whose loop, binomial
checkpointing and reverse sweep run in the library, and
``TransportObservations`` wraps it as a torch.autograd.Function.
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
    met_hour: int = 0  # met interval of the step (MR_iMetStep_Now)


DEPOSIT_DENSITY = 1000.0  # DepositDensity (kg/m^3), src/Tephra.f90:55


def deposit_thickness(dep: np.ndarray, dz1: float, density: float = DEPOSIT_DENSITY) -> np.ndarray:
    """AshThicknessCalculator without its mask (src/Output_Vars.f90:880-884):
    sum_g DepositGranularity(i,j,g) * dz_vec_pd(1) / KM2_2_M2 / DepositDensity
    * M_2_MM (mm); the grains are summed in order."""
    s = dep[:, :, 0].copy()
    for g in range(1, dep.shape[2]):
        s = s + dep[:, :, g]
    return s * dz1 / 1.0e6 / density * 1.0e3


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

    def _met(self, model, hour: int):
        """The met pair (hour, hour+1) in the model's slots."""
        if getattr(model, "_inv_met_hour", None) != hour:
            model.set_met_steps(self.met.step(hour), self.met.step(hour + 1))
            model._inv_met_hour = hour

    def _winds(self, model, lg: "StepLog"):
        self._met(model, lg.met_hour)
        model.interp_winds(lg.time - lg.met_hour)

    # ------------------------------------------------------------------
    def _step_ops(self, model, itime: int):
        model.Set_BC(1)
        model.AdvectHorz(itime)
        model.AdvectVert()
        if self.cfg.use_diffusion:
            model.Set_BC(2)
            model.DiffuseHorz(itime)
            model.DiffuseVert()

    def forward(self, model, p: np.ndarray, obs: dict | None = None, K: int = 0, fast_dt: bool = False,
                obs_dep: np.ndarray | None = None, dep_from: int = 0, load_from: int = 0):
        """Runs hours of transport from a clean atmosphere.  Returns
        (J, loads, logs, residuals); with K > 0 the state at the start of
        every K-th step n is kept in snapshot slot K + n // K (slots 0..K-1
        hold a segment's recomputed states during the reverse sweep).  The met
        step advances only strictly past the hour (driver.met_hour); with
        fast_dt the dt is FAST_DT's.  With obs_dep the misfit gains
        1/2 |T(D_end - D_from) - obs_dep|^2, T the deposit thickness of the
        deposit laid down after hour dep_from (residuals["dep"]); column loads
        count from hour load_from on."""
        cfg = self.cfg
        from . import driver
        model.set_interior(np.zeros((cfg.nx, cfg.ny, cfg.nz, cfg.ns), order="F"))
        model.zero_outflows()
        model._inv_met_hour = None
        time, itime, mhour = 0.0, 0, -1
        logs, loads, resid = [], {}, {}
        J = 0.0
        simtime = float(self.hours)
        dz1 = float(self.geo["dz_vec"][2])
        d_from = None
        while time < simtime - 1e-12:
            itime += 1
            if obs_dep is not None and dep_from > 0 and abs(time - dep_from) < 1e-9:
                d_from = deposit_thickness(model.outflows()["deposit"], dz1)
            model.step_prologue()
            h = driver.met_interval(time, mhour)
            load_new = h != mhour
            self._met(model, h)
            next_obs = math.floor(time + 1e-12) + 1.0
            if fast_dt and load_new:
                if mhour < 0:
                    model.adjust_dt_meso(0, False, time, next_obs, simtime, wait=False)
                model.adjust_dt_meso(1, True, time, next_obs, simtime, wait=False)
            mhour = h
            model.interp_winds(time - h)
            # dt stays on the device while the step is queued; the host reads
            # it once the step's sweeps are on the stream (lag-one loop)
            if fast_dt:
                model.fast_dt_async(time - h, time, next_obs, simtime)
            else:
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
                if obs is not None and ob in obs and ob >= load_from:
                    r = load - obs[ob]
                    resid[ob] = r
                    J += 0.5 * float(np.sum(r * r))
            logs.append(StepLog(itime, time - dt, dt, hour, ob, h))
        if obs_dep is not None:
            t = deposit_thickness(model.outflows()["deposit"], dz1)
            if d_from is not None:
                t = t - d_from
            loads["dep"] = t
            r = t - obs_dep
            resid["dep"] = r
            J += 0.5 * float(np.sum(r * r))
        return J, loads, logs, resid

    def gradient(self, model, p: np.ndarray, obs: dict, K: int = 32, fast_dt: bool = False,
                 obs_dep: np.ndarray | None = None, dep_from: int = 0, load_from: int = 0):
        """J(p) and dJ/dp (shape (nz, hours, ns)) by checkpointed reverse
        sweep."""
        cfg = self.cfg
        J, loads, logs, resid = self.forward(model, p, obs, K=K, fast_dt=fast_dt, obs_dep=obs_dep,
                                             dep_from=dep_from, load_from=load_from)
        N = len(logs)
        nseg = (N + K - 1) // K
        model.adj_enable()
        model.adj_zero()
        model.adj_grad_reset(self.hours)  # gathered on the device, read back once
        lam_dep = None
        if "dep" in resid:  # T^T r: every grain's deposit gets r * dz_vec(1)/KM2_2_M2/DepositDensity*M_2_MM
            dz1 = float(self.geo["dz_vec"][2])
            w = resid["dep"] * dz1 / 1.0e6 / DEPOSIT_DENSITY * 1.0e3
            lam_dep = np.asfortranarray(np.repeat(w[:, :, None], cfg.ns, axis=2))
        dep_on = False
        for seg in range(nseg - 1, -1, -1):
            n0, n1 = seg * K, min(N, seg * K + K)
            # recompute the segment, keeping each step's post-source state
            model.snapshot_load(K + seg)
            for n in range(n0, n1):
                lg = logs[n]
                if n > n0:
                    model.step_prologue()
                self._winds(model, lg)
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
                if lam_dep is not None:  # the deposit window: steps starting at or after dep_from
                    on = lg.time + 1e-12 >= dep_from
                    if on != dep_on:
                        model.set_lambda_dep(lam_dep if on else None)
                        dep_on = on
                model.snapshot_load(n - n0)
                self._winds(model, lg)
                model.set_dt(lg.dt)
                model.adj_step(lg.itime)
                if 0 <= lg.hour < self.hours:
                    # grad[:, hour, :] += dt * lam_vent / kappa, in step order
                    model.adj_vent_accumulate(lg.hour, lg.dt)
        return J, model.adj_grad_get()


class InversionGPU:
    """The source inversion through the library's forward/adjoint pair
    (a3g_inv_setup, a3g_forward_checkpointed, a3g_adjoint,
    a3g_tangent_linear): the whole run, its binomial checkpoints and the
    reverse sweep execute in the library with no per-step host call.

    Control p: (nz, nbins, ns) mass rates (kg/h).  Observations: the hourly
    column loads (hours, nx, ny) and the deposit thickness (nx, ny).  Met
    steps come from `met` (anything with step(hour) -> (vx, vy, vz); default
    the configuration's synthetic source); met_cache=False keeps them out of
    the device cache, so that large grids leave that memory to checkpoints."""

    def __init__(self, model, cfg: syn.Config, hours: int, obs: dict | None = None,
                 obs_dep: np.ndarray | None = None, nbins: int | None = None, load_from: int = 0,
                 dep_from: int = 0, fast_dt: bool = False, snapshot_bytes: float = 0.0, adj_from: int = 0,
                 met=None, met_cache: bool = True):
        import ctypes as C
        from . import _lib
        self.model, self.cfg, self.hours = model, cfg, hours
        self.nbins = hours if nbins is None else nbins
        self.C, self._lib = C, _lib
        # anything with step(hour) -> (vx, vy, vz); FP32 Fortran-order arrays pass without a copy
        self.met = met if met is not None else syn.MetSource(cfg)
        self._keep = []

        def provider(user, hour, pvx, pvy, pvz):
            try:
                arrs = [np.asfortranarray(a, dtype=np.float32) for a in self.met.step(int(hour))]
                # valid until the next call; the library asks for a pair, so
                # the previous step is kept too
                self._keep = (self._keep + [arrs])[-2:]
                for dst, a in zip((pvx, pvy, pvz), arrs):
                    dst[0] = a.ctypes.data_as(_lib.FP)
                return 0
            except Exception:  # noqa: BLE001 -- reported as a failed provider
                return 1

        self._provider = _lib.MET_PROVIDER(provider)
        d = _lib.InvDesc()
        d.ivent, d.jvent, d.nbins = cfg.ivent, cfg.jvent, self.nbins
        d.misfit = (_lib.MISFIT_LOAD if obs is not None else 0) | (_lib.MISFIT_DEPOSIT if obs_dep is not None else 0)
        if d.misfit == 0:
            d.misfit = _lib.MISFIT_LOAD
        d.fast_dt, d.load_from, d.dep_from, d.adj_from = int(fast_dt), load_from, dep_from, adj_from
        d.sim_hours, d.snapshot_bytes = float(hours), float(snapshot_bytes)
        d.met_cache = 0 if met_cache else 1
        nxy = (cfg.nx, cfg.ny)
        ol = np.zeros((hours, cfg.ny, cfg.nx))
        for h, y in (obs or {}).items():
            if isinstance(h, int) and 0 <= h < hours:
                ol[h] = np.asarray(y).T
        od = np.ascontiguousarray(np.asarray(obs_dep).T) if obs_dep is not None else np.zeros(nxy[::-1])
        self.desc = d
        _lib.check(model.lib.a3g_inv_setup(model.ctx, C.byref(d), self._provider, None, _lib.dptr(ol),
                                           _lib.dptr(od)))
        self.nsteps = None

    def _ctl(self, p):
        c = self.cfg
        a = np.asfortranarray(p, dtype=np.float64)
        assert a.shape == (c.nz, self.nbins, c.ns), a.shape
        return a

    def forward(self, p: np.ndarray):
        """J, hourly loads (hours, nx, ny) and deposit thickness (nx, ny)."""
        C, L = self.C, self._lib
        J, n = C.c_double(), C.c_int32()
        L.check(self.model.lib.a3g_forward_checkpointed(self.model.ctx, L.dptr(self._ctl(p)), C.byref(J), C.byref(n)))
        self.nsteps = n.value
        loads, dep = self.observations()
        return J.value, loads, dep

    def observations(self):
        c, L = self.cfg, self._lib
        loads = np.zeros((self.hours, c.ny, c.nx))
        dep = np.zeros((c.ny, c.nx))
        st = (self.C.c_int64 * 4)()
        L.check(self.model.lib.a3g_inv_observations(self.model.ctx, L.dptr(loads), L.dptr(dep), st))
        self.stats = {"steps": st[0], "slots": st[1], "recomputed": st[2], "window_steps": st[3]}
        return loads.transpose(0, 2, 1).copy(), dep.T.copy()

    def adjoint(self, w_load: np.ndarray | None = None, w_dep: np.ndarray | None = None) -> np.ndarray:
        """dJ/dp after forward(), or the vector-Jacobian product with the
        given weights on the observations ((hours, nx, ny) and (nx, ny))."""
        c, L = self.cfg, self._lib
        wl = None if w_load is None else np.ascontiguousarray(np.asarray(w_load, dtype=np.float64).transpose(0, 2, 1))
        wd = None if w_dep is None else np.ascontiguousarray(np.asarray(w_dep, dtype=np.float64).T)
        if (wl is None) != (wd is None):  # one weight given: the other observation has weight 0
            wl = np.zeros((self.hours, c.ny, c.nx)) if wl is None else wl
            wd = np.zeros((c.ny, c.nx)) if wd is None else wd
        g = np.zeros((c.nz, self.nbins, c.ns), order="F")
        L.check(self.model.lib.a3g_adjoint(self.model.ctx, L.dptr(wl), L.dptr(wd), L.dptr(g)))
        self.observations()
        return g

    def tangent_linear(self, p: np.ndarray, dp: np.ndarray):
        """The observations' perturbation for dp at p: (hours, nx, ny), (nx, ny)."""
        c, L = self.cfg, self._lib
        dl = np.zeros((self.hours, c.ny, c.nx))
        dd = np.zeros((c.ny, c.nx))
        L.check(self.model.lib.a3g_tangent_linear(self.model.ctx, L.dptr(self._ctl(p)), L.dptr(self._ctl(dp)),
                                                  L.dptr(dl), L.dptr(dd)))
        return dl.transpose(0, 2, 1).copy(), dd.T.copy()


def TransportObservations():
    """torch.autograd.Function over InversionGPU: apply(p, inv) returns the
    hourly column loads and the deposit thickness as float64 tensors; their
    backward is the adjoint run with the incoming gradients as weights, so
    any loss built on them in torch differentiates through the transport."""
    import torch

    class _Fn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, p, inv):
            _, loads, dep = inv.forward(p.detach().cpu().numpy())
            ctx.inv = inv
            return torch.from_numpy(loads), torch.from_numpy(dep)

        @staticmethod
        def backward(ctx, g_loads, g_dep):
            g = ctx.inv.adjoint(g_loads.detach().cpu().numpy(), g_dep.detach().cpu().numpy())
            return torch.from_numpy(np.ascontiguousarray(g)), None

    return _Fn
