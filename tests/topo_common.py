"""Terrain (useTopo) cases shared by the CPU and GPU terrain tests."""
import dataclasses

import numpy as np

from volcano_ash3d_b200 import synthetic as syn


def topo_config(name: str, zscaling_id: int, topo_km: float = 1.5) -> syn.Config:
    """A small configuration with a Gaussian hill under the vent."""
    return dataclasses.replace(syn.make_config(name), zscaling_id=zscaling_id, topo_km=topo_km)


def level_winds(cfg, seed):
    """Ghosted FP64 (vx, vy, vz) in km/h with sign changes, shaped the way the
    reference holds them when Calc_Vmod_Topo runs: vx and vy are zero on the
    ghost levels k = -1, 0, nz+1, nz+2 (MesoInterpolater writes 1:nz only
    and Set_BC never touches them, src/MesoInterpolater.f90:207-223,
    src/Set_BC.f90:41-66)."""
    rng = np.random.default_rng(seed)
    shp = (cfg.nx + 4, cfg.ny + 4, cfg.nz + 4)
    vx = 60.0 * rng.standard_normal(shp) + 20.0
    vy = 50.0 * rng.standard_normal(shp) - 10.0
    vz = 5.0 * rng.standard_normal(shp)
    for v in (vx, vy):
        v[:, :, :2] = 0.0
        v[:, :, -2:] = 0.0
    return tuple(np.asfortranarray(v) for v in (vx, vy, vz))


def vh_restated(cfg, vx, vy, fields):
    """Calc_Vmod_Topo (src/Topography.f90:2151-2163) in numpy, every i, j, k."""
    g = vx * fields["dhdx"][:, :, None] + vy * fields["dhdy"][:, :, None]
    if cfg.zscaling_id == 1:
        return -1.0 * g
    fac = fields["s_cc"] / fields["ztop"] - 1.0
    return fac[None, None, :] * g
