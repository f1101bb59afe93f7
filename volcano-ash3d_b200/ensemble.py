"""Ensembles of independent transport runs on one GPU.

No counterpart in the reference (one Ash3d process runs one eruption).  An
ensemble (different grids, grain sets, plumes and durations) runs its members
concurrently: every member owns a context, and so its own CUDA stream, and a
host thread drives the member's time loop (driver.run_pipelined, which
queues each step without waiting for the GPU; driver.run where a member needs
the host every step).  The C-ABI releases the interpreter lock on every call, so one
member's host work and small launches overlap the other members' kernels.
Each member's results are the bits its run gives alone, because members
share no device data.

autotune() picks, per member, the fastest advection kernel variant for each
direction (x: marching rows, 4- or 8-cell blocks, warp tiles, warp rows; y
and z: marching lines, 4- or 8-cell blocks, the column march) and the CN
solve variants by timing short runs on a scratch context; the choice changes
speed only, never results.
"""
from __future__ import annotations

import concurrent.futures as cf
import dataclasses
import time

import numpy as np

from . import driver
from . import synthetic as syn


def c3_members(n: int = 64, seed: int = 3, hours: float = 12.0) -> list[syn.Config]:
    """Seeded members: nx, ny in [80, 400], nz in [30, 80] (top at 35 km),
    2-10 grain bins, plume height U(5, 30) km, duration U(1, 12) h, 5 km
    projected cells, jet + wave winds over each member's extent, CN diffusion."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        nx, ny = (int(v) for v in rng.integers(80, 401, 2))
        nz = int(rng.integers(30, 81))
        ns = int(rng.integers(2, 11))
        plume = float(rng.uniform(5.0, 30.0))
        dur = float(rng.uniform(1.0, 12.0))
        fall = tuple(float(v) for v in np.logspace(-3, np.log10(3.0), ns))
        out.append(syn.Config(f"C3m{m:02d}", nx, ny, nz, ns, dx=5.0, dy=5.0, dz=35.0 / nz,
                              ivent=nx // 2, jvent=ny // 2, fall_mps=fall, bin_mass=(1.0 / ns,) * ns,
                              plume_km=plume, volume_km3=1.0e-2, duration_h=dur,
                              diffusivity_m2s=500.0, use_cn=True, sim_hours=hours, winds="c2",
                              seed=1000 + m))
    return out


def autotune(cfg: syn.Config, device: int = 0, steps: int = 2) -> dict:
    """{direction: variant} for directions 0..2 (advection), 3 (CN x solve)
    and 4 (CN y and z solves), timed with the per-kernel CUDA events on a
    scratch context."""
    from .model import Ash3dGPU
    m = Ash3dGPU(cfg, device=device)
    rng = np.random.default_rng(0)
    m.set_interior(np.asfortranarray(rng.uniform(0.0, 1.0e3, (cfg.nx, cfg.ny, cfg.nz, cfg.ns))))
    st = driver.new_state(cfg)
    far = 1.0e9  # never clip dt to the end of the run while timing
    driver.step(m, st, simtime=far, totals=False)
    choice = {}
    keys = {0: ("advect_x",), 1: ("advect_y",), 2: ("advect_z",), 3: ("cn_solve_x",),
            4: ("cn_solve_y", "cn_solve_z")}
    for d, options in ((0, (0, 1, 2, 3, 4, 5)), (1, (0, 1, 2, 5, 6)), (2, (0, 1, 2, 5, 6)), (3, (0, 1, 2)), (4, (0, 1, 2, 3))):
        if d >= 3 and not cfg.use_cn:
            continue
        best, best_ms = None, None
        for v in options:
            m.set_variant(d, v)
            m.kernel_timing(True)
            for _ in range(steps):
                driver.step(m, st, simtime=far, totals=False)
            kt = m.kernel_times()
            ms = sum(kt[k][0] for k in keys[d])
            m.kernel_timing(False)
            if best_ms is None or ms < best_ms:
                best, best_ms = v, ms
        m.set_variant(d, best)
        choice[d] = best
    m.close()
    return choice


@dataclasses.dataclass
class MemberResult:
    name: str
    steps: int
    cell_grain_steps: float
    seconds: float
    final_tot: float
    state: np.ndarray | None = None


class Ensemble:
    def __init__(self, cfgs: list[syn.Config], device: int = 0, tune: bool = False,
                 keep_state: bool = False):
        self.cfgs = cfgs
        self.device = device
        self.keep_state = keep_state
        self.variants = [autotune(c, device) if tune else {} for c in cfgs]

    def _run_member(self, i: int, hours: float) -> MemberResult:
        from .model import Ash3dGPU
        cfg = self.cfgs[i]
        m = Ash3dGPU(cfg, device=self.device)
        for d, v in self.variants[i].items():
            m.set_variant(d, v)
        m.set_interior(np.zeros((cfg.nx, cfg.ny, cfg.nz, cfg.ns), order="F"))
        t0 = time.perf_counter()
        # the lag-one loop when the member allows it (same bits as driver.run)
        if cfg.fast_subgrid or syn.is_umbrella(cfg):
            st = driver.run(m, cfg, sim_hours=hours)
        else:
            st = driver.run_pipelined(m, cfg, sim_hours=hours)
        m.sync()
        el = time.perf_counter() - t0
        res = MemberResult(cfg.name, st.itime, float(cfg.cell_grains) * st.itime, el,
                           st.history[-1].tot if st.history else 0.0,
                           m.interior() if self.keep_state else None)
        m.close()
        return res

    def run_sequential(self, hours: float) -> tuple[list[MemberResult], float]:
        t0 = time.perf_counter()
        res = [self._run_member(i, hours) for i in range(len(self.cfgs))]
        return res, time.perf_counter() - t0

    def run_concurrent(self, hours: float, threads: int | None = None) -> tuple[list[MemberResult], float]:
        from . import _lib
        _lib.load()  # once, before the worker threads start
        n = len(self.cfgs)
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=threads or n) as ex:
            res = list(ex.map(lambda i: self._run_member(i, hours), range(n)))
        return res, time.perf_counter() - t0
