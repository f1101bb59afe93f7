"""ctypes wrapper of the C oracle (ash3d_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker and the timed CPU baseline.  The
product path (volcano-ash3d_b200) never imports this module.

``OracleModel`` owns every reference module array in its Fortran layout
(numpy, order='F', ghost extents included) and exposes the same routine names
as the GPU model, so a parity test drives both through one host loop.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SRC = HERE / "ash3d_oracle.c"

CFLAGS = ["-O3", "-fno-fast-math", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-Wall"]


def build(force: bool = False) -> pathlib.Path:
    """Compiles the oracle (gcc; IEEE double, no contraction)."""
    if force or not LIB.exists() or LIB.stat().st_mtime < max(SRC.stat().st_mtime,
                                                              (HERE / "ash3d_oracle.h").stat().st_mtime):
        subprocess.check_call(["gcc", *CFLAGS, "-o", str(LIB), str(SRC), "-lm"])
    return LIB


class OrcState(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("ns", C.c_int32),
        ("periodic", C.c_int32), ("latlon", C.c_int32),
        ("limiter", C.c_int32), ("use_cn", C.c_int32), ("use_diffusion", C.c_int32),
        ("fast_subgrid", C.c_int32), ("nocycle", C.c_int32),
        ("imin", C.c_int32), ("imax", C.c_int32), ("jmin", C.c_int32), ("jmax", C.c_int32),
        ("kmin", C.c_int32), ("kmax", C.c_int32),
        ("have_dt_diffus", C.c_int32), ("n_gs_aloft", C.c_int32),
        ("nthreads", C.c_int32), ("pad0", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double),
        ("cfl", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
        ("imp_fac", C.c_double), ("imp_dt_fac", C.c_double), ("eps_thresh", C.c_double),
        ("eps_small", C.c_double), ("cloudcon_grid_thresh", C.c_double),
        ("magma_density", C.c_double), ("dt", C.c_double), ("time_diffuse", C.c_double),
    ] + [(n, C.POINTER(C.c_double)) for n in (
        "concen", "vx", "vy", "vz", "vh", "vf", "kappa", "sig_nx", "sig_ny", "sig_nz", "dz_vec",
        "kx", "ky", "kz", "outflow_yz1", "outflow_yz2", "outflow_xz1", "outflow_xz2",
        "outflow_xy1", "outflow_xy2", "deposit")] + [
        ("is_aloft", C.POINTER(C.c_int32)), ("mass_aloft", C.POINTER(C.c_double)),
        ("zscaling_id", C.c_int32), ("use_topo", C.c_int32), ("ztop", C.c_double)] + [
        (n, C.POINTER(C.c_double)) for n in ("dhdx", "dhdy", "deldx", "deldy", "s_cc")]


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        S = C.POINTER(OrcState)
        D = C.POINTER(C.c_double)
        F = C.POINTER(C.c_float)
        for name, res, args in [
            ("orc_set_bc", C.c_int, [S, C.c_int]),
            ("orc_advect_x", None, [S]), ("orc_advect_y", None, [S]), ("orc_advect_z", None, [S]),
            ("orc_advect_horz", C.c_int, [S, C.c_int, C.c_int, C.c_int, C.c_int]),
            ("orc_advect_vert", None, [S]), ("orc_calc_vmod_topo", None, [S]),
            ("orc_diff_x", None, [S]), ("orc_diff_y", None, [S]), ("orc_diff_z", None, [S]),
            ("orc_diffcn_x", None, [S]), ("orc_diffcn_y", None, [S]), ("orc_diffcn_z", None, [S]),
            ("orc_diffuse_horz", None, [S, C.c_int]), ("orc_diffuse_vert", None, [S]),
            ("orc_adjust_dt", None, [S, C.c_double, C.c_double, C.c_double, D]),
            ("orc_cfl_maxima", None, [S, D]),
            ("orc_dt_from_maxima", None, [S, D, C.c_int, C.c_double, C.c_double, C.c_double, D]),
            ("orc_cfl_maxima_meso", None, [S, F, F, F, F, C.c_int, D]),
            ("orc_fast_dt", C.c_double, [S, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_double]),
            ("orc_timestep_totals", None, [S, D]),
            ("orc_get_minmax_index", C.c_int, [S, C.c_int, C.c_int, C.c_int]),
            ("orc_step_prologue", None, [S]),
            ("orc_add_source", None, [S, C.c_int, C.c_int, D, C.c_double]),
            ("orc_interp_winds", None, [S, F, F, F, F, F, F, C.c_double]),
            ("orc_prune_gs", None, [S, C.c_double]),
            ("orc_vprofiles", None, [S, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_double, D,
                                     C.POINTER(C.c_int32)]),
            ("orc_add_umbrella_winds", None, [S, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, D, D]),
            ("orc_add_source_umbrella", None, [S, C.c_int, C.c_int, C.c_int, C.c_int, D, D, C.c_double]),
            ("orc_dgtsv", C.c_int, [C.c_int, D, D, D, D]),
            ("orc_set_threads", None, [C.c_int]), ("orc_get_threads", C.c_int, []),
            ("orc_adj_advect_x", None, [S, D]), ("orc_adj_advect_y", None, [S, D]),
            ("orc_adj_advect_z", None, [S, D, D]),
            ("orc_adj_diffuse_horz", None, [S, D, C.c_int]), ("orc_adj_diffuse_vert", None, [S, D]),
            ("orc_output_vars", None, [S, D, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                       D, D, D, D, C.POINTER(C.c_int32), D, C.POINTER(C.c_int32), D, D, D]),
        ]:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def dgtsv(dl, d, du, b):
    """The oracle's dgtsv restatement on copies of the inputs; returns (x, info)."""
    lib = load()
    dl = np.array(dl, dtype=np.float64)
    d = np.array(d, dtype=np.float64)
    du = np.array(du, dtype=np.float64)
    b = np.array(b, dtype=np.float64)
    info = lib.orc_dgtsv(len(d), _d(dl), _d(d), _d(du), _d(b))
    return b, info


class OracleModel:
    """Reference module state + the restated per-step routines."""

    def __init__(self, cfg, geo=None, limiter: str = None, threads: int = 0):
        import importlib
        syn = importlib.import_module("volcano_ash3d_b200.synthetic")
        self.syn = syn
        self.cfg = cfg
        lib = load()
        self.lib = lib
        if threads:
            lib.orc_set_threads(threads)
        nx, ny, nz, ns = cfg.nx, cfg.ny, cfg.nz, cfg.ns
        NX, NY, NZ = nx + 4, ny + 4, nz + 4
        geo = geo if geo is not None else syn.geometry(cfg)
        self.geo = geo
        z = lambda *s: np.zeros(s, order="F")
        self.concen = z(NX, NY, NZ, ns, 2)
        self.vx, self.vy, self.vz, self.vh = z(NX, NY, NZ), z(NX, NY, NZ), z(NX, NY, NZ), z(NX, NY, NZ)
        self.vf = np.asfortranarray(syn.fall_velocity(cfg))
        self.kappa = np.asfortranarray(geo["kappa"])
        self.sig_nx = np.asfortranarray(geo["sig_nx"])
        self.sig_ny = np.asfortranarray(geo["sig_ny"])
        self.sig_nz = np.asfortranarray(geo["sig_nz"])
        self.dz_vec = np.ascontiguousarray(geo["dz_vec"])
        self.kx, self.ky, self.kz = [np.asfortranarray(a) for a in syn.diffusivity(cfg)]
        self.out_yz1, self.out_yz2 = z(NY, NZ, ns), z(NY, NZ, ns)
        self.out_xz1, self.out_xz2 = z(NX, NZ, ns), z(NX, NZ, ns)
        self.out_xy1, self.out_xy2 = z(NX, NY, ns), z(NX, NY, ns)
        self.deposit = z(nx, ny, ns)
        self.is_aloft = np.ones(ns, dtype=np.int32)
        self.mass_aloft = np.zeros(ns)
        dx, dy = syn.projected_dxdy(cfg)
        lim = limiter or cfg.limiter
        from volcano_ash3d_b200._lib import LIMITERS
        s = OrcState()
        s.nx, s.ny, s.nz, s.ns = nx, ny, nz, ns
        s.periodic, s.latlon = int(cfg.periodic), int(cfg.latlon)
        s.limiter = LIMITERS[lim]
        s.use_cn, s.use_diffusion = int(cfg.use_cn), int(cfg.use_diffusion)
        s.fast_subgrid, s.nocycle = int(cfg.fast_subgrid), 0
        s.imin, s.imax, s.jmin, s.jmax, s.kmin, s.kmax = 1, nx, 1, ny, 1, nz
        s.have_dt_diffus, s.n_gs_aloft = 0, ns
        s.dx, s.dy = dx, dy
        s.cfl, s.dt_min, s.dt_max = cfg.cfl, 1.0e-5, 1.0
        s.imp_fac, s.imp_dt_fac, s.eps_thresh = 0.5, 4.0, 1.0e-10
        s.eps_small, s.cloudcon_grid_thresh, s.magma_density = 1.0e-6, 1.0e-7, cfg.magma_density
        for name, arr in [("concen", self.concen), ("vx", self.vx), ("vy", self.vy), ("vz", self.vz),
                          ("vh", self.vh), ("vf", self.vf), ("kappa", self.kappa),
                          ("sig_nx", self.sig_nx), ("sig_ny", self.sig_ny), ("sig_nz", self.sig_nz),
                          ("dz_vec", self.dz_vec), ("kx", self.kx), ("ky", self.ky), ("kz", self.kz),
                          ("outflow_yz1", self.out_yz1), ("outflow_yz2", self.out_yz2),
                          ("outflow_xz1", self.out_xz1), ("outflow_xz2", self.out_xz2),
                          ("outflow_xy1", self.out_xy1), ("outflow_xy2", self.out_xy2),
                          ("deposit", self.deposit), ("mass_aloft", self.mass_aloft)]:
            setattr(s, name, _d(arr))
        s.is_aloft = self.is_aloft.ctypes.data_as(C.POINTER(C.c_int32))
        s.zscaling_id, s.use_topo, s.ztop = int(cfg.zscaling_id), 0, 0.0
        self.s = s
        self.ps = C.byref(s)
        self._topo = None
        if syn.use_topo(cfg):
            self.set_topo(**syn.topo_fields(cfg))
        self.umbrella = syn.umbrella_setup(cfg, self.kappa) if syn.is_umbrella(cfg) else None
        self.dt_meso_last = self.dt_meso_next = 0.0
        self.set_fall_velocity_meso(syn.fall_velocity_meso(cfg), per_grain=True)

    # --- routines with the reference names ---------------------------------
    def Set_BC(self, code):
        if self.lib.orc_set_bc(self.ps, code):
            raise ValueError("ERROR BC code not recognized")

    def AdvectHorz(self, itoggle):
        cfg = self.cfg
        if self.lib.orc_advect_horz(self.ps, itoggle, cfg.ivent, cfg.jvent, 1):
            raise RuntimeError("ERROR: kmax<kmin in get_minmax_index")

    def advect_x(self):
        self.lib.orc_advect_x(self.ps)

    def advect_y(self):
        self.lib.orc_advect_y(self.ps)

    def AdvectVert(self):
        self.lib.orc_advect_vert(self.ps)

    def DiffuseHorz(self, itime):
        self.lib.orc_diffuse_horz(self.ps, itime)

    def DiffuseVert(self):
        self.lib.orc_diffuse_vert(self.ps)

    def Adjust_DT(self, time, next_write_time, simtime):
        out = C.c_double()
        self.lib.orc_adjust_dt(self.ps, time, next_write_time, simtime, C.byref(out))
        return out.value

    def cfl_maxima(self):
        v = np.zeros(3)
        self.lib.orc_cfl_maxima(self.ps, _d(v))
        return v

    def adjust_dt_from_maxima(self, vmax3, n_gs_aloft_total, time, next_write_time, simtime):
        v = np.ascontiguousarray(vmax3, dtype=np.float64)
        out = C.c_double()
        self.lib.orc_dt_from_maxima(self.ps, _d(v), n_gs_aloft_total, time, next_write_time, simtime,
                                    C.byref(out))
        return out.value

    def set_dt(self, dt):
        self.s.dt = dt

    # --- FAST_DT (src/Adjust_dt.f90:96-135, src/MesoInterpolater.f90:142-150,
    #     187-195, 250-258) ---------------------------------------------------
    def set_fall_velocity_meso(self, vf_sp, per_grain=True):
        self._vf_meso = (np.asfortranarray(vf_sp, dtype=np.float32), int(bool(per_grain)))

    def _met_slot(self, slot):
        return self._met[0:3] if slot == 0 else self._met[3:6]

    def cfl_maxima_meso(self, slot):
        vx, vy, vz = self._met_slot(slot)
        vf, pg = self._vf_meso
        v = np.zeros(3)
        self.lib.orc_cfl_maxima_meso(self.ps, _f(vx), _f(vy), _f(vz), _f(vf), pg, _d(v))
        return v

    def adjust_dt_meso_from_maxima(self, vmax3, n_gs_aloft_total, shift, time, next_write_time, simtime):
        if shift:
            self.dt_meso_last = self.dt_meso_next
        dt = self.adjust_dt_from_maxima(vmax3, n_gs_aloft_total, time, next_write_time, simtime)
        self.dt_meso_next = dt
        return dt

    def adjust_dt_meso(self, slot, shift, time, next_write_time, simtime, wait=True):
        return self.adjust_dt_meso_from_maxima(self.cfl_maxima_meso(slot), self.s.n_gs_aloft, shift, time,
                                               next_write_time, simtime)

    def fast_dt_async(self, frac, time, next_write_time, simtime):
        self._dt_pending = self.lib.orc_fast_dt(self.ps, self.dt_meso_last, self.dt_meso_next, frac, time,
                                                next_write_time, simtime)

    def fast_dt(self, frac, time, next_write_time, simtime):
        self.fast_dt_async(frac, time, next_write_time, simtime)
        return self._dt_pending

    def TimeStepTotals(self):
        out = np.zeros(4)
        self.lib.orc_timestep_totals(self.ps, _d(out))
        return out, self.mass_aloft.copy()

    def get_minmax_index(self):
        cfg = self.cfg
        if self.lib.orc_get_minmax_index(self.ps, cfg.ivent, cfg.jvent, 1):
            raise RuntimeError("ERROR: kmax<kmin in get_minmax_index")
        s = self.s
        return (s.imin, s.imax, s.jmin, s.jmax, s.kmin, s.kmax)

    def set_subgrid(self, box):
        s = self.s
        s.imin, s.imax, s.jmin, s.jmax, s.kmin, s.kmax = box

    def step_prologue(self):
        self.lib.orc_step_prologue(self.ps)

    def add_source(self, flux, dt):
        f = np.asfortranarray(flux, dtype=np.float64)
        self.lib.orc_add_source(self.ps, self.cfg.ivent, self.cfg.jvent, _d(f), dt)

    def set_met_steps(self, last, nxt):
        self._met = [np.asfortranarray(a, dtype=np.float32) for a in (*last, *nxt)]

    # --- the device loop's entry points, restated on the host --------------
    def adjust_dt_async(self, time, next_write_time, simtime):
        self._dt_pending = self.Adjust_DT(time, next_write_time, simtime)

    def wait_dt(self):
        return self._dt_pending

    def add_source_devdt(self, flux):
        self.add_source(flux, self.s.dt)

    def adj_grad_reset(self, nbins):
        c = self.cfg
        self._grad = np.zeros((c.nz, nbins, c.ns))
        kap = self.kappa
        self._kap_col = np.array([kap[c.ivent + 1, c.jvent + 1, k + 1] for k in range(1, c.nz + 1)])

    def adj_vent_accumulate(self, bin_, dt):
        col = self.adj_vent_column()
        self._grad[:, bin_, :] += dt * col[:self.cfg.nz, :] / self._kap_col[:, None]

    def adj_grad_get(self):
        return self._grad.copy()

    def prefetch_met_step(self, step):
        self._met_ahead = [np.asfortranarray(a, dtype=np.float32) for a in step]

    def advance_met_step(self):
        self._met = [*self._met[3:], *self._met_ahead]
        self._met_ahead = None

    def interp_winds(self, frac):
        m = self._met
        self.lib.orc_interp_winds(self.ps, _f(m[0]), _f(m[3]), _f(m[1]), _f(m[4]), _f(m[2]), _f(m[5]), frac)
        if self.s.use_topo:  # Ash3d.F90:398, right after MesoInterpolater
            self.lib.orc_calc_vmod_topo(self.ps)

    def set_winds(self, vx, vy, vz):
        self.vx[...] = vx
        self.vy[...] = vy
        self.vz[...] = vz
        if self.s.use_topo:
            self.lib.orc_calc_vmod_topo(self.ps)

    def vprofiles(self, points, pr_ash=None, thresh=1.0e-3):
        """Calc_vprofile: (pr_ash (nz, npts) in mg/m3, written flags)."""
        ip = np.ascontiguousarray([p[0] for p in points], dtype=np.int32)
        jp = np.ascontiguousarray([p[1] for p in points], dtype=np.int32)
        out = np.zeros((self.cfg.nz, len(points)), order="F") if pr_ash is None else pr_ash
        w = np.zeros(len(points), dtype=np.int32)
        I = C.POINTER(C.c_int32)
        self.lib.orc_vprofiles(self.ps, len(points), ip.ctypes.data_as(I), jp.ctypes.data_as(I), thresh,
                               _d(out), w.ctypes.data_as(I))
        return out, w

    def add_umbrella_winds(self, i0, i1, j0, j1, uvx, uvy):
        u = self.umbrella
        a, b = np.asfortranarray(uvx, dtype=np.float64), np.asfortranarray(uvy, dtype=np.float64)
        self.lib.orc_add_umbrella_winds(self.ps, u.ibase, u.itop, i0, i1, j0, j1, _d(a), _d(b))
        if self.s.use_topo:  # Calc_Vmod_Topo follows MesoInterpolater
            self.lib.orc_calc_vmod_topo(self.ps)

    def add_source_umbrella(self, flux_umbrella, dt):
        u, c = self.umbrella, self.cfg
        st = np.asfortranarray(u.stencil, dtype=np.float64)
        f = np.asfortranarray(flux_umbrella, dtype=np.float64)
        self.lib.orc_add_source_umbrella(self.ps, c.ivent, c.jvent, u.ibase, u.itop, _d(st), _d(f), dt)

    def set_topo(self, dhdx, dhdy, deldx, deldy, s_cc, ztop):
        """useTopo: dhdx_comp, dhdy_comp, DelDxonD_cc, DelDyonD_cc
        (-1:nx+2,-1:ny+2), s_cc_pd (-1:nz+2), Ztop (km).  vh is recomputed
        after every wind update (Calc_Vmod_Topo)."""
        c = self.cfg
        a2 = [np.asfortranarray(a, dtype=np.float64) for a in (dhdx, dhdy, deldx, deldy)]
        for a in a2:
            assert a.shape == (c.nx + 4, c.ny + 4)
        sc = np.ascontiguousarray(s_cc, dtype=np.float64)
        assert sc.shape == (c.nz + 4,)
        self._topo = (*a2, sc)
        s = self.s
        s.dhdx, s.dhdy, s.deldx, s.deldy, s.s_cc = [_d(a) for a in self._topo]
        s.ztop, s.use_topo = float(ztop), 1
        self.lib.orc_calc_vmod_topo(self.ps)

    def set_aloft(self, flags):
        self.is_aloft[:] = np.asarray(flags, dtype=np.int32)
        self.s.n_gs_aloft = int(self.is_aloft.sum())

    def prune_gs(self, thresh=1.0e-3):
        self.lib.orc_prune_gs(self.ps, thresh)

    # --- discrete adjoint (no counterpart in the reference) ------------------
    # lam arrays are interior-shaped (nx, ny, nz, ns); each call applies the
    # transpose of one sweep, linearised at the state now in ts0.
    def _lam_in(self, lam):
        c = self.cfg
        w = np.zeros(self.concen.shape[:4], order="F")
        w[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :] = lam
        return w

    def _lam_out(self, w):
        c = self.cfg
        return w[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :].copy(order="F")

    def adj_advect_x(self, lam):
        w = self._lam_in(lam)
        self.lib.orc_adj_advect_x(self.ps, _d(w))
        return self._lam_out(w)

    def adj_advect_y(self, lam):
        w = self._lam_in(lam)
        self.lib.orc_adj_advect_y(self.ps, _d(w))
        return self._lam_out(w)

    def adj_advect_z(self, lam, lam_dep=None):
        w = self._lam_in(lam)
        ld = None if lam_dep is None else np.asfortranarray(lam_dep, dtype=np.float64)
        self.lib.orc_adj_advect_z(self.ps, _d(w), None if ld is None else _d(ld))
        return self._lam_out(w)

    def adj_diffuse_horz(self, lam, itime):
        w = self._lam_in(lam)
        self.lib.orc_adj_diffuse_horz(self.ps, _d(w), itime)
        return self._lam_out(w)

    def adj_diffuse_vert(self, lam):
        w = self._lam_in(lam)
        self.lib.orc_adj_diffuse_vert(self.ps, _d(w))
        return self._lam_out(w)

    # stateful form (the GPU model's interface): lam kept here
    def adj_enable(self):
        if getattr(self, "lam", None) is None:
            self.adj_zero()

    def adj_zero(self):
        c = self.cfg
        self.lam = np.zeros((c.nx, c.ny, c.nz, c.ns), order="F")
        self.lam_dep = np.zeros((c.nx, c.ny, c.ns), order="F")

    def set_lambda(self, lam):
        self.adj_enable()
        self.lam = np.asfortranarray(lam, dtype=np.float64).copy(order="F")

    def get_lambda(self):
        return self.lam.copy(order="F")

    def set_lambda_dep(self, lam_dep):
        self.adj_enable()
        c = self.cfg
        self.lam_dep = np.zeros((c.nx, c.ny, c.ns), order="F") if lam_dep is None else \
            np.asfortranarray(lam_dep, dtype=np.float64).copy(order="F")

    def get_lambda_dep(self):
        return self.lam_dep.copy(order="F")

    def adj_step(self, itime):
        """Reverse of one transport step; ts0 holds the state after the
        step's source insertion and is left unchanged."""
        a = self.interior()
        keep = [x.copy() for x in (self.out_yz1, self.out_yz2, self.out_xz1, self.out_xz2,
                                   self.out_xy1, self.out_xy2, self.deposit)]
        even = itime % 2 == 0
        self.set_interior(a)
        (self.advect_y if even else self.advect_x)()
        b = self.interior()
        (self.advect_x if even else self.advect_y)()
        cst = self.interior()
        for dst, src in zip((self.out_yz1, self.out_yz2, self.out_xz1, self.out_xz2, self.out_xy1,
                             self.out_xy2, self.deposit), keep):
            dst[...] = src
        lam = self.lam
        if self.cfg.use_diffusion:
            lam = self.adj_diffuse_vert(lam)
            lam = self.adj_diffuse_horz(lam, itime)
        self.set_interior(cst)
        lam = self.adj_advect_z(lam, self.lam_dep)
        self.set_interior(b)
        lam = (self.adj_advect_x if even else self.adj_advect_y)(lam)
        self.set_interior(a)
        lam = (self.adj_advect_y if even else self.adj_advect_x)(lam)
        self.lam = lam

    def adj_vent_column(self):
        c = self.cfg
        out = np.zeros((c.nz + 1, c.ns), order="F")
        out[:c.nz, :] = self.lam[c.ivent - 1, c.jvent - 1, :, :]
        return out

    def cloud_load(self):
        """Unmasked CloudLoad (src/Output_Vars.f90:1061-1069), same order."""
        c = self.cfg
        q = self.interior()
        load = np.zeros((c.nx, c.ny))
        for k in range(c.nz):
            s = np.zeros((c.nx, c.ny))
            for g in range(c.ns):
                s = s + q[:, :, k, g]
            load = load + s * self.dz_vec[k + 2] / 1.0e3
        return load

    def adj_add_cloud_load(self, w):
        c = self.cfg
        for k in range(c.nz):
            add = w * self.dz_vec[k + 2] / 1.0e3
            for g in range(c.ns):
                self.lam[:, :, k, g] = self.lam[:, :, k, g] + add

    def snapshot_alloc(self, n):
        if not hasattr(self, "_snaps"):
            self._snaps = {}

    def snapshot_save(self, slot):
        self._snaps[slot] = self.interior()

    def snapshot_load(self, slot):
        self.set_interior(self._snaps[slot])

    # --- output products (Gen_Output_Vars) ----------------------------------
    OUTPUT_DEFAULTS = dict(cloudcon_thresh=1.0e-3, cloudload_thresh=0.2, depo_thresh=1.0e-2,
                           deposit_density=1000.0)

    def output_reset(self):
        c = self.cfg
        self._arr_cloud = np.full((c.nx, c.ny), -1.0, order="F")
        self._arr_dep = np.full((c.nx, c.ny), -1.0, order="F")

    def output_vars(self, time, **thresholds):
        """Gen_Output_Vars products of the current state (dict of arrays)."""
        c = self.cfg
        t = dict(self.OUTPUT_DEFAULTS, **thresholds)
        if getattr(self, "_arr_cloud", None) is None:
            self.output_reset()
        _, zcc, _ = self.syn.zgrid(c)
        z_cc = np.ascontiguousarray(zcc[2:c.nz + 2])
        f = lambda: np.zeros((c.nx, c.ny), order="F")
        out = dict(cloud_load=f(), max_height=f(), min_height=f(), max_conc=f(), dep_thick=f())
        mc = np.zeros((c.nx, c.ny), dtype=np.int32, order="F")
        md = np.zeros((c.nx, c.ny), dtype=np.int32, order="F")
        areas = np.zeros(7)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        self.lib.orc_output_vars(self.ps, _d(z_cc), t["cloudcon_thresh"], t["cloudload_thresh"],
                                 t["depo_thresh"], t["deposit_density"], time,
                                 _d(out["cloud_load"]), _d(out["max_height"]), _d(out["min_height"]),
                                 _d(out["max_conc"]), ip(mc), _d(out["dep_thick"]), ip(md),
                                 _d(self._arr_cloud), _d(self._arr_dep), _d(areas))
        out.update(mask_cloud=mc.astype(bool), mask_dep=md.astype(bool),
                   cloud_arrival=self._arr_cloud.copy(), dep_arrival=self._arr_dep.copy(),
                   cloud_area=areas[0], dep_area=areas[1], cloud_load_area=areas[2:].copy())
        return out

    def zero_outflows(self):
        for a in (self.out_yz1, self.out_yz2, self.out_xz1, self.out_xz2, self.out_xy1, self.out_xy2,
                  self.deposit):
            a[...] = 0.0

    # --- state access --------------------------------------------------------
    def interior(self):
        """Interior of ts0 as (nx, ny, nz, ns), Fortran order."""
        c = self.cfg
        return self.concen[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :, 0].copy(order="F")

    def set_interior(self, q):
        c = self.cfg
        self.concen[...] = 0.0
        self.concen[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :, 0] = q
        self.concen[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :, 1] = q

    def outflows(self):
        c = self.cfg
        return dict(
            yz1=self.out_yz1[2:c.ny + 2, 2:c.nz + 2, :].copy(), yz2=self.out_yz2[2:c.ny + 2, 2:c.nz + 2, :].copy(),
            xz1=self.out_xz1[2:c.nx + 2, 2:c.nz + 2, :].copy(), xz2=self.out_xz2[2:c.nx + 2, 2:c.nz + 2, :].copy(),
            xy1=self.out_xy1[2:c.nx + 2, 2:c.ny + 2, :].copy(), xy2=self.out_xy2[2:c.nx + 2, 2:c.ny + 2, :].copy(),
            deposit=self.deposit.copy())

    # --- NetCDF output arrays and restart (src/write_NETCDF.f90) -------------
    def output_ashcon(self):
        """ashcon = real(concen_pd(1:nx,1:ny,1:nz,1:ns,ts1), op) (:3296-3298);
        depocon = real(DepositGranularity*dz_vec_pd(0)/KM2_2_M2, op), then
        0.0 where depocon <= EPS_SMALL (:3320-3330).  op = 4 (FP32,
        src/Ash3d_VariableModules.f90:31); Fortran compares the FP32 value
        with the FP64 EPS_SMALL after promoting it."""
        c = self.cfg
        ash = np.asfortranarray(self.concen[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :, 1].astype(np.float32))
        dz0 = self.dz_vec[1]  # dz_vec_pd(0) (index = Fortran k + 1)
        dep = np.asfortranarray((self.deposit * dz0 / 1.0e6).astype(np.float32))
        dep[dep.astype(np.float64) <= 1.0e-6] = np.float32(0.0)
        return ash, dep

    def restart_load(self, ashcon, depocon):
        """NC_RestartFile_LoadConcen (src/write_NETCDF.f90:3701-3709):
        concen_pd(1:nx,1:ny,1:nz,i,ts1) = real(ashcon(:,:,:,i), ip),
        outflow_xy1_pd = DepositGranularity = real(depocon, ip), then
        concen(:,:,:,:,ts0) = concen(:,:,:,:,ts1)."""
        c = self.cfg
        self.concen[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :, 1] = np.asarray(ashcon, np.float32).astype(np.float64)
        self.out_xy1[2:c.nx + 2, 2:c.ny + 2, :] = np.asarray(depocon, np.float32).astype(np.float64)
        self.deposit[...] = self.out_xy1[2:c.nx + 2, 2:c.ny + 2, :]
        self.concen[..., 0] = self.concen[..., 1]

    @property
    def dt(self):
        return self.s.dt
