"""Host-side mirror of the reference's per-step routines over the C-ABI.

``Ash3dGPU`` keeps the names, argument meaning and error behaviour of the
Fortran subroutines that Ash3d.F90's main loop calls (src/Ash3d.F90:372-642):
``Set_BC(bc_code)``, ``AdvectHorz(itoggle)``, ``AdvectVert()``,
``DiffuseHorz(i)``, ``DiffuseVert()``, ``Adjust_DT(...)`` and
``TimeStepTotals()``.  All work runs on the GPU through
``libash3d_b200.so``; a failing call raises ``A3GError`` (the reference's
``stop 1``).  Arrays crossing the boundary use the reference's Fortran
layouts (numpy order='F' with ghost cells).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from . import synthetic as syn
from ._lib import check, dptr, fptr, iptr


class DeviceDoubles:
    """A few doubles in a context's device memory, exposed through
    __cuda_array_interface__ so that torch.as_tensor wraps them without a
    copy; `stream` is the context's stream, on which their producer was
    queued."""

    def __init__(self, ptr: int, n: int, stream: int):
        self.ptr, self.n, self.stream = ptr, n, stream

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self.n,), "typestr": "<f8", "data": (self.ptr, False), "version": 3}


class Ash3dGPU:
    def __init__(self, cfg: syn.Config, device: int = 0, geo: dict | None = None,
                 limiter: str | None = None, use_winds_fp64: bool = False):
        self.lib = lib = _lib.load()
        self.cfg = cfg
        g = _lib.GridDesc()
        g.nx, g.ny, g.nz, g.ns = cfg.nx, cfg.ny, cfg.nz, cfg.ns
        g.periodic, g.latlon = int(cfg.periodic), int(cfg.latlon)
        g.dx, g.dy = syn.projected_dxdy(cfg)
        p = _lib.Params()
        lib.a3g_default_params(C.byref(p))
        p.limiter = _lib.LIMITERS[limiter or cfg.limiter]
        p.use_cn = int(cfg.use_cn)
        p.use_diffusion = int(cfg.use_diffusion)
        p.fast_subgrid = int(cfg.fast_subgrid)
        p.cfl = cfg.cfl
        p.magma_density = cfg.magma_density
        p.zscaling_id = int(cfg.zscaling_id)
        self.ctx = C.c_void_p()
        check(lib.a3g_create(C.byref(g), C.byref(p), device, C.byref(self.ctx)))
        geo = geo if geo is not None else syn.geometry(cfg)
        self.geo = geo
        check(lib.a3g_set_geometry(self.ctx, dptr(geo["kappa"]), dptr(geo["sig_nx"]),
                                   dptr(geo["sig_ny"]), dptr(geo["sig_nz"]), dptr(geo["dz_vec"])))
        kx, ky, kz = syn.diffusivity(cfg)
        check(lib.a3g_set_diffusivity(self.ctx, dptr(kx), dptr(ky), dptr(kz)))
        self._vf = syn.fall_velocity(cfg)
        check(lib.a3g_set_fall_velocity(self.ctx, dptr(self._vf)))
        self.set_fall_velocity_meso(syn.fall_velocity_meso(cfg), per_grain=True)
        self._dt = 0.0
        if syn.use_topo(cfg):
            self.set_topo(**syn.topo_fields(cfg))
        self.umbrella = None
        if syn.is_umbrella(cfg):
            u = syn.umbrella_setup(cfg, geo["kappa"])
            st = np.asfortranarray(u.stencil, dtype=np.float64)
            check(lib.a3g_set_umbrella(self.ctx, cfg.ivent, cfg.jvent, u.ibase, u.itop, dptr(st)))
            self.umbrella = u

    # --- lifetime ----------------------------------------------------------
    def close(self):
        if self.ctx:
            self.lib.a3g_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        check(self.lib.a3g_sync(self.ctx))

    def stream_handle(self) -> int:
        """cudaStream_t of this context (for torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        check(self.lib.a3g_get_stream(self.ctx, C.byref(s)))
        return s.value or 0

    def kernel_timing(self, enable: bool):
        check(self.lib.a3g_kernel_timing(self.ctx, 1 if enable else 0))

    def kernel_times(self) -> dict:
        """{class: (total_ms, launches)} since kernel_timing(True)."""
        n = len(_lib.KERNEL_CLASSES)
        ms = np.zeros(n)
        cnt = (C.c_uint64 * n)()
        check(self.lib.a3g_kernel_times(self.ctx, dptr(ms), cnt))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_lib.KERNEL_CLASSES)}

    def set_variant(self, direction: int, variant: int):
        check(self.lib.a3g_set_variant(self.ctx, direction, variant))

    def kernel_launches(self) -> int:
        n = C.c_uint64()
        check(self.lib.a3g_kernel_launches(self.ctx, C.byref(n)))
        return n.value

    # --- routines with the reference names -----------------------------------
    def Set_BC(self, bc_code: int):
        check(self.lib.a3g_set_bc(self.ctx, bc_code))

    def AdvectHorz(self, itoggle: int):
        c = self.cfg
        check(self.lib.a3g_advect_horz(self.ctx, itoggle, c.ivent, c.jvent, 1))

    def advect_x(self):
        check(self.lib.a3g_advect_x(self.ctx))

    def advect_y(self):
        check(self.lib.a3g_advect_y(self.ctx))

    def AdvectVert(self):
        check(self.lib.a3g_advect_vert(self.ctx))

    def DiffuseHorz(self, i: int):
        check(self.lib.a3g_diffuse_horz(self.ctx, i))

    def DiffuseVert(self):
        check(self.lib.a3g_diffuse_vert(self.ctx))

    def Adjust_DT(self, time: float, next_write_time: float, simtime: float) -> float:
        out = C.c_double()
        check(self.lib.a3g_adjust_dt(self.ctx, time, next_write_time, simtime, C.byref(out)))
        self._dt = out.value
        return out.value

    def cfl_maxima(self) -> np.ndarray:
        v = np.zeros(3)
        check(self.lib.a3g_cfl_maxima(self.ctx, dptr(v)))
        return v

    def cfl_maxima_device(self) -> "DeviceDoubles":
        """The three CFL maxima reduced on the context's stream into device
        memory (a3g_cfl_maxima_device), as an object a torch all-reduce can
        work on in place (__cuda_array_interface__)."""
        ptr = C.POINTER(C.c_double)()
        check(self.lib.a3g_cfl_maxima_device(self.ctx, C.byref(ptr)))
        return DeviceDoubles(C.cast(ptr, C.c_void_p).value, 3, self.stream_handle())

    def adjust_dt_device_maxima_async(self, n_gs_aloft_total: int, time: float, next_write_time: float,
                                      simtime: float):
        check(self.lib.a3g_adjust_dt_device_maxima_async(self.ctx, n_gs_aloft_total, time, next_write_time,
                                                         simtime))

    def adjust_dt_from_maxima(self, vmax3, n_gs_aloft_total: int, time: float,
                              next_write_time: float, simtime: float) -> float:
        v = np.ascontiguousarray(vmax3, dtype=np.float64)
        out = C.c_double()
        check(self.lib.a3g_adjust_dt_from_maxima(self.ctx, dptr(v), n_gs_aloft_total, time,
                                                 next_write_time, simtime, C.byref(out)))
        self._dt = out.value
        return out.value

    def set_dt(self, dt: float):
        self._dt = dt
        check(self.lib.a3g_set_dt(self.ctx, dt))

    # --- FAST_DT: Adjust_DT(mesostep=.true.) at met-step loads, the
    #     interpolated dt every step (src/MesoInterpolater.f90:142-150,187-195,
    #     250-258) ----------------------------------------------------------
    def set_fall_velocity_meso(self, vf_sp, per_grain: bool = True):
        a = np.asfortranarray(vf_sp, dtype=np.float32)
        check(self.lib.a3g_set_fall_velocity_meso(self.ctx, fptr(a), 1 if per_grain else 0))

    def cfl_maxima_meso(self, slot: int) -> np.ndarray:
        v = np.zeros(3)
        check(self.lib.a3g_cfl_maxima_meso(self.ctx, slot, dptr(v)))
        return v

    def adjust_dt_meso(self, slot: int, shift: bool, time: float, next_write_time: float, simtime: float,
                       wait: bool = True):
        """Adjust_DT(mesostep=.true.) on met slot 0 (last) or 1 (next); the
        result is dt_meso_next on the device.  With wait=False nothing is
        read back (returns None)."""
        if not wait:
            check(self.lib.a3g_adjust_dt_meso(self.ctx, slot, 1 if shift else 0, time, next_write_time,
                                              simtime, None))
            return None
        out = C.c_double()
        check(self.lib.a3g_adjust_dt_meso(self.ctx, slot, 1 if shift else 0, time, next_write_time, simtime,
                                          C.byref(out)))
        return out.value

    def adjust_dt_meso_from_maxima(self, vmax3, n_gs_aloft_total: int, shift: bool, time: float,
                                   next_write_time: float, simtime: float) -> float:
        v = np.ascontiguousarray(vmax3, dtype=np.float64)
        out = C.c_double()
        check(self.lib.a3g_adjust_dt_meso_from_maxima(self.ctx, dptr(v), n_gs_aloft_total, 1 if shift else 0,
                                                      time, next_write_time, simtime, C.byref(out)))
        return out.value

    def fast_dt_async(self, frac: float, time: float, next_write_time: float, simtime: float):
        check(self.lib.a3g_fast_dt_async(self.ctx, frac, time, next_write_time, simtime))

    def fast_dt(self, frac: float, time: float, next_write_time: float, simtime: float) -> float:
        self.fast_dt_async(frac, time, next_write_time, simtime)
        return self.wait_dt()

    def TimeStepTotals(self):
        out = np.zeros(4)
        mass = np.zeros(self.cfg.ns)
        check(self.lib.a3g_timestep_totals(self.ctx, dptr(out), dptr(mass)))
        return out, mass

    def get_minmax_index(self):
        c = self.cfg
        box = np.zeros(6, dtype=np.int32)
        check(self.lib.a3g_get_minmax_index(self.ctx, c.ivent, c.jvent, 1, iptr(box)))
        return tuple(int(v) for v in box)

    def set_subgrid(self, box):
        b = np.asarray(box, dtype=np.int32)
        check(self.lib.a3g_set_subgrid(self.ctx, iptr(b)))

    def step_prologue(self):
        check(self.lib.a3g_step_prologue(self.ctx))

    def add_source(self, flux: np.ndarray, dt: float):
        f = np.asfortranarray(flux, dtype=np.float64)
        check(self.lib.a3g_add_source_column(self.ctx, self.cfg.ivent, self.cfg.jvent, dptr(f), dt))

    def set_met_steps(self, last, nxt):
        arrs = [np.asfortranarray(a, dtype=np.float32) for a in (*last, *nxt)]
        check(self.lib.a3g_set_met_steps(self.ctx, *[fptr(a) for a in arrs]))
        self._met_keep = arrs  # the copies are asynchronous

    def prefetch_met_step(self, step):
        """Copies one met step (vx, vy, vz) into the spare slot on the copy stream."""
        arrs = [np.asfortranarray(a, dtype=np.float32) for a in step]
        check(self.lib.a3g_prefetch_met_step(self.ctx, *[fptr(a) for a in arrs]))
        self._prefetch_keep = arrs  # the copy may still be reading them

    def advance_met_step(self):
        check(self.lib.a3g_advance_met_step(self.ctx))

    def met_prefetch_fence(self):
        check(self.lib.a3g_met_prefetch_fence(self.ctx))

    def interp_winds(self, frac: float):
        check(self.lib.a3g_interp_winds(self.ctx, frac))

    def set_winds(self, vx, vy, vz):
        a = [np.asfortranarray(v, dtype=np.float64) for v in (vx, vy, vz)]
        check(self.lib.a3g_set_winds(self.ctx, *[dptr(v) for v in a]))

    # --- lag-one host loop (driver.Pipeline) -----------------------------------
    def adjust_dt_async(self, time, next_write_time, simtime):
        check(self.lib.a3g_adjust_dt_async(self.ctx, time, next_write_time, simtime))

    def wait_dt(self) -> float:
        d = C.c_double()
        check(self.lib.a3g_wait_dt(self.ctx, C.byref(d)))
        self._dt = d.value
        return d.value

    def totals_async(self) -> int:
        t = C.c_int64()
        check(self.lib.a3g_timestep_totals_async(self.ctx, C.byref(t)))
        return t.value

    def totals_get(self, ticket: int):
        out = np.zeros(4)
        ma = np.zeros(self.cfg.ns)
        check(self.lib.a3g_totals_get(self.ctx, ticket, dptr(out), dptr(ma)))
        return out, ma

    def set_source_pulses(self, ivent, jvent, pulses, norm_col):
        t0 = np.ascontiguousarray([p[0] for p in pulses], dtype=np.float64)
        t1 = np.ascontiguousarray([p[1] for p in pulses], dtype=np.float64)
        mfr = np.ascontiguousarray([p[2] for p in pulses], dtype=np.float64)
        # NormSourceColumn(npulses, nz+1); one column given for one pulse
        c = np.asarray(norm_col, dtype=np.float64)
        col = np.asfortranarray(c.reshape(len(pulses), self.cfg.nz + 1))
        bm = np.ascontiguousarray(self.cfg.bin_mass, dtype=np.float64)
        check(self.lib.a3g_set_source_pulses(self.ctx, ivent, jvent, len(pulses), dptr(t0), dptr(t1), dptr(mfr),
                                             dptr(col), dptr(bm)))

    def add_source_scheduled(self, time):
        check(self.lib.a3g_add_source_scheduled(self.ctx, time))

    def vprofiles(self, points, pr_ash=None):
        """Calc_vprofile: (pr_ash (nz, npts) in mg/m3, written flags).  Points
        whose column is below CLOUDCON_THRESH keep pr_ash's previous column."""
        ip = np.ascontiguousarray([p[0] for p in points], dtype=np.int32)
        jp = np.ascontiguousarray([p[1] for p in points], dtype=np.int32)
        out = np.zeros((self.cfg.nz, len(points)), order="F") if pr_ash is None else pr_ash
        w = np.zeros(len(points), dtype=np.int32)
        check(self.lib.a3g_vprofiles(self.ctx, len(points), iptr(ip), iptr(jp), dptr(out), iptr(w)))
        return out, w

    def add_umbrella_winds(self, i0, i1, j0, j1, uvx, uvy):
        a, b = np.asfortranarray(uvx, dtype=np.float64), np.asfortranarray(uvy, dtype=np.float64)
        check(self.lib.a3g_add_umbrella_winds(self.ctx, i0, i1, j0, j1, dptr(a), dptr(b)))

    def add_source_umbrella(self, flux_umbrella, dt):
        f = np.asfortranarray(flux_umbrella, dtype=np.float64)
        check(self.lib.a3g_add_source_umbrella(self.ctx, dptr(f), dt))

    def set_topo(self, dhdx, dhdy, deldx, deldy, s_cc, ztop):
        """useTopo: dhdx_comp, dhdy_comp, DelDxonD_cc, DelDyonD_cc
        (-1:nx+2,-1:ny+2), s_cc_pd (-1:nz+2), Ztop (km); vh is formed on
        the device after every wind update (a3g_set_topo)."""
        a = [np.asfortranarray(v, dtype=np.float64) for v in (dhdx, dhdy, deldx, deldy)]
        sc = np.ascontiguousarray(s_cc, dtype=np.float64)
        check(self.lib.a3g_set_topo(self.ctx, *[dptr(v) for v in a], dptr(sc), float(ztop)))

    def set_aloft(self, flags):
        f = np.asarray(flags, dtype=np.int32)
        check(self.lib.a3g_set_aloft(self.ctx, iptr(f)))

    # --- discrete adjoint (no counterpart in the reference) ------------------
    # Stateful calls keep lam on the device (adj_step, adj_add_cloud_load,
    # adj_vent_column); the adj_<sweep>(lam) helpers upload lam, apply one
    # sweep's transpose at the current state and return the result.
    def adj_enable(self):
        if not getattr(self, "_adj_on", False):
            check(self.lib.a3g_adj_enable(self.ctx))
            self._adj_on = True

    def adj_zero(self):
        self.adj_enable()
        check(self.lib.a3g_adj_zero(self.ctx))

    def set_lambda(self, lam: np.ndarray):
        self.adj_enable()
        c = self.cfg
        lv = np.zeros((c.nx + 4, c.ny + 4, c.nz + 4, c.ns), order="F")
        lv[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :] = lam
        check(self.lib.a3g_adj_set_lambda(self.ctx, dptr(lv)))

    def get_lambda(self) -> np.ndarray:
        c = self.cfg
        lv = np.zeros((c.nx + 4, c.ny + 4, c.nz + 4, c.ns), order="F")
        check(self.lib.a3g_adj_get_lambda(self.ctx, dptr(lv)))
        return lv[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :].copy(order="F")

    def set_lambda_dep(self, lam_dep):
        self.adj_enable()
        c = self.cfg
        ld = np.zeros((c.nx, c.ny, c.ns), order="F") if lam_dep is None else \
            np.asfortranarray(lam_dep, dtype=np.float64)
        check(self.lib.a3g_adj_set_lambda_dep(self.ctx, dptr(ld)))

    def get_lambda_dep(self) -> np.ndarray:
        c = self.cfg
        ld = np.zeros((c.nx, c.ny, c.ns), order="F")
        check(self.lib.a3g_adj_get_lambda_dep(self.ctx, dptr(ld)))
        return ld

    def _adj1(self, fn, lam, *args):
        self.set_lambda(lam)
        check(fn(self.ctx, *args))
        return self.get_lambda()

    def adj_advect_x(self, lam):
        return self._adj1(self.lib.a3g_adj_advect_x, lam)

    def adj_advect_y(self, lam):
        return self._adj1(self.lib.a3g_adj_advect_y, lam)

    def adj_advect_z(self, lam, lam_dep=None):
        self.set_lambda_dep(lam_dep)
        return self._adj1(self.lib.a3g_adj_advect_vert, lam)

    def adj_diffuse_horz(self, lam, itime):
        return self._adj1(self.lib.a3g_adj_diffuse_horz, lam, itime)

    def adj_diffuse_vert(self, lam):
        return self._adj1(self.lib.a3g_adj_diffuse_vert, lam)

    def adj_step(self, itime: int):
        check(self.lib.a3g_adj_step(self.ctx, itime))

    def adj_grad_reset(self, nbins: int):
        check(self.lib.a3g_adj_grad_reset(self.ctx, nbins))
        self._grad_bins = nbins

    def adj_vent_accumulate(self, bin_: int, dt: float):
        check(self.lib.a3g_adj_vent_accumulate(self.ctx, self.cfg.ivent, self.cfg.jvent, bin_, dt))

    def adj_grad_get(self) -> np.ndarray:
        """The accumulated gradient, (nz, nbins, ns)."""
        c = self.cfg
        out = np.zeros(self._grad_bins * c.ns * c.nz)
        check(self.lib.a3g_adj_grad_get(self.ctx, dptr(out)))
        return np.ascontiguousarray(out.reshape(self._grad_bins, c.ns, c.nz).transpose(2, 0, 1))

    def add_source_devdt(self, flux: np.ndarray):
        f = np.asfortranarray(flux, dtype=np.float64)
        check(self.lib.a3g_add_source_column_devdt(self.ctx, self.cfg.ivent, self.cfg.jvent, dptr(f)))

    def adj_vent_column(self) -> np.ndarray:
        c = self.cfg
        out = np.zeros((c.nz + 1, c.ns), order="F")
        check(self.lib.a3g_adj_vent_column(self.ctx, c.ivent, c.jvent, dptr(out)))
        return out

    def cloud_load(self) -> np.ndarray:
        self.adj_enable()
        c = self.cfg
        out = np.zeros((c.nx, c.ny), order="F")
        check(self.lib.a3g_cloud_load(self.ctx, dptr(out)))
        return out

    def adj_add_cloud_load(self, w: np.ndarray):
        wf = np.asfortranarray(w, dtype=np.float64)
        check(self.lib.a3g_adj_add_cloud_load(self.ctx, dptr(wf)))

    def snapshot_alloc(self, n: int):
        check(self.lib.a3g_snapshot_alloc(self.ctx, n))

    def snapshot_save(self, slot: int):
        check(self.lib.a3g_snapshot_save(self.ctx, slot))

    def snapshot_load(self, slot: int):
        check(self.lib.a3g_snapshot_load(self.ctx, slot))

    # --- output products (Gen_Output_Vars) ----------------------------------
    OUTPUT_DEFAULTS = dict(cloudcon_thresh=1.0e-3, cloudload_thresh=0.2, depo_thresh=1.0e-2,
                           deposit_density=1000.0)

    def set_output_params(self, **thresholds):
        c = self.cfg
        t = dict(self.OUTPUT_DEFAULTS, **thresholds)
        _, zcc, _ = syn.zgrid(c)
        z = np.ascontiguousarray(zcc[2:c.nz + 2])
        check(self.lib.a3g_set_output_params(self.ctx, dptr(z), t["cloudcon_thresh"], t["cloudload_thresh"],
                                             t["depo_thresh"], t["deposit_density"]))
        self._ov_params = True

    def output_reset(self):
        if not getattr(self, "_ov_params", False):
            self.set_output_params()
        check(self.lib.a3g_output_reset(self.ctx))

    def output_vars(self, time: float) -> dict:
        """Gen_Output_Vars products of the current state (dict of arrays)."""
        if not getattr(self, "_ov_params", False):
            self.set_output_params()
        c = self.cfg
        f = lambda: np.zeros((c.nx, c.ny), order="F")
        out = dict(cloud_load=f(), max_height=f(), min_height=f(), max_conc=f(), dep_thick=f(),
                   cloud_arrival=f(), dep_arrival=f())
        mc = np.zeros((c.nx, c.ny), dtype=np.int32, order="F")
        md = np.zeros((c.nx, c.ny), dtype=np.int32, order="F")
        areas = np.zeros(7)
        check(self.lib.a3g_output_vars(self.ctx, time, dptr(out["cloud_load"]), dptr(out["max_height"]),
                                       dptr(out["min_height"]), dptr(out["max_conc"]), iptr(mc),
                                       dptr(out["dep_thick"]), iptr(md), dptr(out["cloud_arrival"]),
                                       dptr(out["dep_arrival"]), dptr(areas)))
        out.update(mask_cloud=mc.astype(bool), mask_dep=md.astype(bool), cloud_area=areas[0],
                   dep_area=areas[1], cloud_load_area=areas[2:].copy())
        return out

    # --- state access --------------------------------------------------------
    def upload_level(self, level: np.ndarray):
        lv = np.asfortranarray(level, dtype=np.float64)
        check(self.lib.a3g_upload_concen(self.ctx, dptr(lv)))

    def download_level(self) -> np.ndarray:
        c = self.cfg
        lv = np.zeros((c.nx + 4, c.ny + 4, c.nz + 4, c.ns), order="F")
        check(self.lib.a3g_download_concen(self.ctx, dptr(lv)))
        return lv

    def interior(self) -> np.ndarray:
        c = self.cfg
        return self.download_level()[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :].copy(order="F")

    def set_interior(self, q: np.ndarray):
        c = self.cfg
        lv = np.zeros((c.nx + 4, c.ny + 4, c.nz + 4, c.ns), order="F")
        lv[2:c.nx + 2, 2:c.ny + 2, 2:c.nz + 2, :] = q
        self.upload_level(lv)

    def zero_outflows(self):
        """The outflow accumulators and the deposit back to zero."""
        c = self.cfg
        NX, NY, NZ, ns = c.nx + 4, c.ny + 4, c.nz + 4, c.ns
        z = lambda *s: np.zeros(s, order="F")
        check(self.lib.a3g_upload_outflow(self.ctx, dptr(z(NY, NZ, ns)), dptr(z(NY, NZ, ns)), dptr(z(NX, NZ, ns)),
                                          dptr(z(NX, NZ, ns)), dptr(z(NX, NY, ns)), dptr(z(NX, NY, ns))))

    def outflows(self) -> dict:
        c = self.cfg
        NX, NY, NZ, ns = c.nx + 4, c.ny + 4, c.nz + 4, c.ns
        z = lambda *s: np.zeros(s, order="F")
        yz1, yz2, xz1, xz2, xy1, xy2 = z(NY, NZ, ns), z(NY, NZ, ns), z(NX, NZ, ns), z(NX, NZ, ns), z(NX, NY, ns), z(NX, NY, ns)
        dep = z(c.nx, c.ny, ns)
        check(self.lib.a3g_download_outflow(self.ctx, dptr(yz1), dptr(yz2), dptr(xz1), dptr(xz2),
                                            dptr(xy1), dptr(xy2), dptr(dep)))
        return dict(yz1=yz1[2:c.ny + 2, 2:c.nz + 2, :], yz2=yz2[2:c.ny + 2, 2:c.nz + 2, :],
                    xz1=xz1[2:c.nx + 2, 2:c.nz + 2, :], xz2=xz2[2:c.nx + 2, 2:c.nz + 2, :],
                    xy1=xy1[2:c.nx + 2, 2:c.ny + 2, :], xy2=xy2[2:c.nx + 2, 2:c.ny + 2, :], deposit=dep)

    # --- NetCDF output arrays and restart (src/write_NETCDF.f90) --------------
    def output_ashcon(self) -> tuple[np.ndarray, np.ndarray]:
        """(ashcon, depocon) as the NetCDF writer forms them: FP32,
        (nx, ny, nz, ns) and (nx, ny, ns), Fortran order
        (src/write_NETCDF.f90:3296-3298, 3320-3330)."""
        c = self.cfg
        ash = np.empty((c.nx, c.ny, c.nz, c.ns), np.float32, order="F")
        dep = np.empty((c.nx, c.ny, c.ns), np.float32, order="F")
        check(self.lib.a3g_output_ashcon(self.ctx, ash.ctypes.data, dep.ctypes.data))
        return ash, dep

    def restart_load(self, ashcon: np.ndarray, depocon: np.ndarray):
        """NC_RestartFile_LoadConcen (src/write_NETCDF.f90:3646-3716): the
        state from ashcon, outflow_xy1 and DepositGranularity from depocon."""
        c = self.cfg
        ash = np.asfortranarray(ashcon, dtype=np.float32)
        dep = np.asfortranarray(depocon, dtype=np.float32)
        if ash.shape != (c.nx, c.ny, c.nz, c.ns) or dep.shape != (c.nx, c.ny, c.ns):
            raise ValueError(f"ashcon {ash.shape} / depocon {dep.shape} do not match the grid")
        check(self.lib.a3g_restart_load(self.ctx, ash.ctypes.data, dep.ctypes.data))

    @property
    def dt(self):
        return self._dt
