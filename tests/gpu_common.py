"""Helpers shared by the GPU parity tests: seeded states and winds, and a
pair of models (GPU through the C-ABI, oracle on the CPU) on one geometry."""
import numpy as np

import ash3d_oracle as orc
from volcano_ash3d_b200 import synthetic as syn
from volcano_ash3d_b200.model import Ash3dGPU


def pair(name_or_cfg, **over):
    cfg = syn.make_config(name_or_cfg) if isinstance(name_or_cfg, str) else name_or_cfg
    for k, v in over.items():
        setattr(cfg, k, v)
    geo = syn.geometry(cfg)
    return cfg, Ash3dGPU(cfg, geo=geo), orc.OracleModel(cfg, geo=geo)


def random_state(cfg, seed):
    """Plume-like non-negative field with exact zeros, values straddling
    EPS_THRESH (1e-10) and a few large cells, (nx,ny,nz,ns) Fortran order."""
    rng = np.random.default_rng(seed)
    nx, ny, nz, ns = cfg.nx, cfg.ny, cfg.nz, cfg.ns
    x = np.linspace(-1, 1, nx)[:, None, None, None]
    y = np.linspace(-1, 1, ny)[None, :, None, None]
    z = np.linspace(0, 1, nz)[None, None, :, None]
    g = np.arange(ns)[None, None, None, :]
    q = 1.0e4 * np.exp(-((x - 0.1 * g) ** 2 + y ** 2) * 6.0 - (z - 0.4) ** 2 * 8.0)
    q = q * rng.uniform(0.5, 1.5, q.shape)
    q[rng.uniform(size=q.shape) < 0.1] = 0.0
    tiny = rng.uniform(size=q.shape) < 0.05
    q[tiny] = rng.uniform(0.0, 3.0e-10, tiny.sum())
    return np.asfortranarray(q)


def random_winds(cfg, seed):
    """Ghosted FP64 (vx, vy, vz) in km/h with sign changes (both upwind branches)."""
    rng = np.random.default_rng(seed)
    shp = (cfg.nx + 4, cfg.ny + 4, cfg.nz + 4)
    vx = 60.0 * rng.standard_normal(shp) + 20.0
    vy = 50.0 * rng.standard_normal(shp) - 10.0
    vz = 5.0 * rng.standard_normal(shp)
    return tuple(np.asfortranarray(v) for v in (vx, vy, vz))


def prime(cfg, gpu, ref, seed, box=None):
    """Identical state, winds and dt on both models; returns dt."""
    q = random_state(cfg, seed)
    vx, vy, vz = random_winds(cfg, seed + 1)
    for m in (gpu, ref):
        m.set_interior(q)
        m.set_winds(vx, vy, vz)
    dg = gpu.Adjust_DT(0.0, 1.0e9, 1.0e9)
    dr = ref.Adjust_DT(0.0, 1.0e9, 1.0e9)
    assert dg == dr, (dg, dr)
    if box is not None:
        gpu.set_subgrid(box)
        ref.set_subgrid(box)
    return dg
