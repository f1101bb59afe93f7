"""Host-side set-up for the transport path: grids, geometry, winds and source.

These are the pieces the reference computes on the host before and around
the per-step path (they are inputs of the path, not part of it):

* ``geometry``: cell volumes and face areas of ``calc_mesh_params``
  (src/Calc_Mesh.f90:23-220) for projected and spherical lon/lat grids, in the
  Fortran layouts with two ghost cells.
* ``suzuki_column`` / ``source_flux``: the normalised Suzuki column
  (src/Source.f90:287-490), the pulse fraction of CheckEruptivePulses
  (:613-685) and SourceNodeFlux of TephraSourceNodes (:708-783).
* synthetic FP32 met steps for the named workloads (no met data is read:
  MetReader is not part of this path).  Every random draw is seeded.

Workloads (interior cells x grains):
  C1  projected 100x100x40, 4 grains, explicit diffusion, steady winds
  C2  lon/lat 720x360x60 at 0.25 deg, 10 grains, Crank-Nicolson, hourly winds
  C4  projected 200x200x50, 6 grains, explicit diffusion
  C5  projected 1500x1000x80, 20 grains, Crank-Nicolson
  plus small cases (``tiny_*``) used by the parity tests.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

DEG2RAD = 1.7453292519943295e-2
PI = 3.141592653589793
RAD_EARTH = 6371.229
MPS_2_KMPHR = 3.6
M2PS_2_KM2PHR = 3.6e-3
KM3_2_M3 = 1.0e9
DEG2KMLAT = 111.0
DEG2KMLON = 111.321
KM_2_M = 1.0e3
HR_2_S = 3.6e3
# umbrella-cloud parameters (src/Source_Umbrella.f90:47-52 defaults)
UMB_VELMOD = 1
UMB_K_ENTRAIN = 0.1
UMB_LAMBDA = 0.2
UMB_N_BV = 0.02
UMB_SUZUKI_K = 12.0


@dataclasses.dataclass
class Config:
    name: str
    nx: int
    ny: int
    nz: int
    ns: int
    latlon: bool = False
    periodic: bool = False
    dx: float = 5.0          # km (projected)
    dy: float = 5.0
    de: float = 0.25         # deg (lon/lat)
    dn: float = 0.25
    lonLL: float = 0.0
    latLL: float = 0.0
    xLL: float = 0.0
    yLL: float = 0.0
    dz: float = 0.5          # km
    dz_profile: tuple = ()   # per-level thicknesses (km), overriding dz when given
    ivent: int = 1
    jvent: int = 1
    z_volcano: float = 0.0   # vent elevation (km)
    fall_mps: tuple = (0.1,)
    bin_mass: tuple = (1.0,)
    plume_km: float = 15.0
    volume_km3: float = 1.0e-2
    duration_h: float = 3.0
    suzuki_a: float = 4.0
    diffusivity_m2s: float = 500.0
    use_cn: bool = False
    use_diffusion: bool = True
    limiter: str = "superbee"
    cfl: float = 0.8
    sim_hours: float = 6.0
    winds: str = "c1"        # 'c1' steady shear, 'c2' jet + wave + noise, 'random', 'const', 'sounding'
    wind_uv: tuple = (0.0, 0.0)   # 'const': uniform (u, v) in m/s
    sounding: tuple = ()     # 'sounding': ((z_m, u_mps, v_mps), ...) of a 1-D wind profile
    seed: int = 1
    fast_subgrid: bool = False
    fast_dt: bool = False    # FAST_DT: dt from the met steps, interpolated every step
    magma_density: float = 2500.0
    source_type: str = "suzuki"   # 'suzuki', 'umbrella', 'umbrella_air' (lon/lat grids; suzuki_a 12)
    zscaling_id: int = 0     # ZScaling_ID: 0 s = z, 1 shifted by topography, 2 scaled (sigma-altitude)
    topo_km: float = 0.0     # height of a Gaussian hill centred on the vent (0: no topography)
    topo_width_km: float = 0.0   # its standard deviation (km); 0: three cell widths

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def cell_grains(self) -> int:
        return self.nx * self.ny * self.nz * self.ns


def _logspace(a, b, n):
    return tuple(float(x) for x in np.logspace(math.log10(a), math.log10(b), n))


def make_config(name: str) -> Config:
    """The workloads named in the benchmark definition, plus small test cases."""
    if name == "C1":
        return Config("C1", 100, 100, 40, 4, dx=5.0, dy=5.0, dz=0.5, ivent=50, jvent=50,
                      fall_mps=(0.01, 0.1, 0.5, 2.0), bin_mass=(0.25,) * 4, plume_km=15.0,
                      volume_km3=1.0e-2, duration_h=3.0, diffusivity_m2s=500.0, use_cn=False,
                      sim_hours=6.0, winds="c1", seed=1)
    if name == "C2":
        # 5 S - 85 N: a top boundary on the pole itself gives the pole interface
        # zero area and the ghost cells beyond it negative volume, so the CN
        # coefficient of the last row is 0/0 in the reference's formulas.
        return Config("C2", 720, 360, 60, 10, latlon=True, de=0.25, dn=0.25, lonLL=0.0, latLL=-5.0,
                      dz=0.5, ivent=360, jvent=180, fall_mps=_logspace(1e-3, 3.0, 10),
                      bin_mass=(0.1,) * 10, plume_km=15.0, volume_km3=1.0e-2, duration_h=3.0,
                      diffusivity_m2s=500.0, use_cn=True, sim_hours=24.0, winds="c2", seed=2)
    if name == "C4":
        return Config("C4", 200, 200, 50, 6, dx=5.0, dy=5.0, dz=0.5, ivent=100, jvent=100,
                      fall_mps=_logspace(1e-2, 2.0, 6), bin_mass=(1.0 / 6,) * 6, plume_km=15.0,
                      volume_km3=1.0e-2, duration_h=3.0, diffusivity_m2s=500.0, use_cn=False,
                      sim_hours=24.0, winds="c1", seed=4)
    if name == "C5":
        return Config("C5", 1500, 1000, 80, 20, dx=3.0, dy=3.0, dz=0.4, ivent=750, jvent=500,
                      fall_mps=_logspace(1e-3, 3.0, 20), bin_mass=(0.05,) * 20, plume_km=25.0,
                      volume_km3=1.0e-1, duration_h=12.0, diffusivity_m2s=500.0, use_cn=True,
                      sim_hours=48.0, winds="c2p", seed=5)
    if name == "tiny_proj":
        return Config("tiny_proj", 24, 20, 12, 3, dx=5.0, dy=5.0, dz=0.5, ivent=12, jvent=10,
                      fall_mps=(0.05, 0.5, 2.0), bin_mass=(0.3, 0.3, 0.4), plume_km=5.0,
                      volume_km3=1.0e-3, duration_h=1.0, use_cn=False, sim_hours=2.0,
                      winds="random", seed=11)
    if name == "tiny_cn":
        return Config("tiny_cn", 22, 18, 14, 2, dx=4.0, dy=6.0, dz=0.5, ivent=10, jvent=9,
                      fall_mps=(0.2, 1.0), bin_mass=(0.5, 0.5), plume_km=6.0, volume_km3=1.0e-3,
                      duration_h=1.0, use_cn=True, sim_hours=2.0, winds="random", seed=12)
    if name == "tiny_latlon":
        return Config("tiny_latlon", 30, 16, 10, 2, latlon=True, de=1.0, dn=1.0, lonLL=10.0,
                      latLL=30.0, dz=0.5, ivent=15, jvent=8, fall_mps=(0.3, 1.5),
                      bin_mass=(0.5, 0.5), plume_km=4.0, volume_km3=1.0e-3, duration_h=1.0,
                      use_cn=True, sim_hours=2.0, winds="random", seed=13)
    if name == "tiny_periodic":
        return Config("tiny_periodic", 36, 12, 8, 2, latlon=True, periodic=True, de=10.0, dn=5.0,
                      lonLL=0.0, latLL=20.0, dz=0.5, ivent=3, jvent=6, fall_mps=(0.3, 1.5),
                      bin_mass=(0.5, 0.5), plume_km=3.0, volume_km3=1.0e-3, duration_h=1.0,
                      use_cn=False, sim_hours=2.0, winds="random", seed=14)
    if name == "tiny_subgrid":
        return Config("tiny_subgrid", 40, 36, 16, 2, dx=5.0, dy=5.0, dz=0.5, ivent=20, jvent=18,
                      fall_mps=(0.1, 1.0), bin_mass=(0.5, 0.5), plume_km=5.0, volume_km3=1.0e-3,
                      duration_h=1.0, use_cn=True, sim_hours=2.0, winds="random", seed=15,
                      fast_subgrid=True)
    if name == "tiny_wide":  # rows longer than one x segment (1024 cells)
        return Config("tiny_wide", 1100, 6, 5, 2, dx=2.0, dy=5.0, dz=0.5, ivent=550, jvent=3,
                      fall_mps=(0.1, 1.0), bin_mass=(0.5, 0.5), plume_km=2.0, volume_km3=1.0e-3,
                      duration_h=1.0, use_cn=True, sim_hours=1.0, winds="random", seed=16)
    if name == "tiny_tall":  # y and z lines longer than one march segment (96 cells)
        return Config("tiny_tall", 20, 200, 110, 3, dx=5.0, dy=2.0, dz=0.1, ivent=10, jvent=100,
                      fall_mps=(0.05, 0.4, 1.5), bin_mass=(0.3, 0.3, 0.4), plume_km=8.0,
                      volume_km3=1.0e-3, duration_h=1.0, use_cn=True, sim_hours=1.0,
                      winds="random", seed=17)
    if name == "tiny_deep":  # z lines of 80 cells, as in the 1500x1000x80 scale workload
        return Config("tiny_deep", 26, 14, 80, 2, dx=3.0, dy=3.0, dz=0.4, ivent=13, jvent=7,
                      fall_mps=(0.1, 1.0), bin_mass=(0.5, 0.5), plume_km=20.0, volume_km3=1.0e-3,
                      duration_h=1.0, use_cn=True, sim_hours=1.0, winds="random", seed=19)
    if name == "tiny_stretch":  # lon/lat CN, x lines of 3 tiles, dz changing part-way up
        return Config("tiny_stretch", 75, 10, 24, 2, latlon=True, de=0.5, dn=0.5, lonLL=20.0,
                      latLL=40.0, dz=0.3, dz_profile=(0.3,) * 10 + (0.45,) * 8 + (0.7,) * 6,
                      ivent=37, jvent=5, fall_mps=(0.2, 1.2), bin_mass=(0.5, 0.5), plume_km=5.0,
                      volume_km3=1.0e-3, duration_h=1.0, use_cn=True, sim_hours=1.0,
                      winds="random", seed=18)
    if name == "tiny_umbrella":  # umbrella source: 0.1 deg cells so that the cloud outgrows the 3x3 patch
        return Config("tiny_umbrella", 40, 36, 18, 2, latlon=True, de=0.1, dn=0.1, lonLL=120.0,
                      latLL=38.0, dz=1.0, ivent=20, jvent=18, fall_mps=(0.05, 1.0), bin_mass=(0.5, 0.5),
                      plume_km=15.0, volume_km3=0.5, duration_h=2.0, suzuki_a=UMB_SUZUKI_K,
                      use_cn=True, sim_hours=3.0, winds="random", seed=19, source_type="umbrella")
    raise KeyError(name)


# ---------------------------------------------------------------------------
# vertical grid and geometry, src/Calc_Mesh.f90:66-168
# ---------------------------------------------------------------------------
def zgrid(cfg: Config):
    nz = cfg.nz
    if cfg.dz_profile:  # a stretched column: level tops from the listed thicknesses
        assert len(cfg.dz_profile) == nz
        z_vec_init = np.concatenate([[0.0], np.cumsum(np.asarray(cfg.dz_profile, dtype=np.float64))])
    else:
        z_vec_init = np.array([cfg.dz * k for k in range(nz + 1)], dtype=np.float64)  # Input_Data.f90:1579
    dz = np.zeros(nz + 4)          # index k+1 for k=-1..nz+2
    zcc = np.zeros(nz + 4)
    zlb = np.zeros(nz + 4)
    for k in range(1, nz + 1):
        dz[k + 1] = z_vec_init[k] - z_vec_init[k - 1]
        zcc[k + 1] = z_vec_init[k] - 0.5 * dz[k + 1]
        zlb[k + 1] = zcc[k + 1] - 0.5 * dz[k + 1]
    zcc[1] = zcc[2] - dz[2]
    zlb[1] = zcc[1] - dz[2]
    zcc[0] = zcc[1] - dz[2]
    zlb[0] = zcc[0] - dz[2]
    zcc[nz + 2] = zcc[nz + 1] + dz[nz + 1]
    zcc[nz + 3] = zcc[nz + 1] + dz[nz + 1] * 2.0
    zlb[nz + 2] = zlb[nz + 1] + dz[nz + 1]
    zlb[nz + 3] = zlb[nz + 1] + dz[nz + 1] * 2.0
    dz[0] = dz[2]
    dz[1] = dz[2]
    dz[nz + 2] = dz[nz + 1]
    dz[nz + 3] = dz[nz + 1]
    return dz, zcc, zlb


def geometry(cfg: Config) -> dict:
    """kappa_pd, sigma_n{x,y,z}_pd (-1:nx+2,-1:ny+2,-1:nz+2) and dz_vec_pd
    (-1:nz+2) of calc_mesh_params, then calc_s_mesh's Jacobian scaling for
    ZScaling_ID 2 (src/Calc_Mesh.f90:316-328)."""
    g = _geometry_z(cfg)
    if use_topo(cfg) and cfg.zscaling_id == 2:
        jcc = jacobian(cfg)
        for name in ("sig_nx", "sig_ny", "kappa"):
            a = g[name]
            for kk in range(a.shape[2]):
                a[:, :, kk] = a[:, :, kk] * jcc
    return g


def _geometry_z(cfg: Config) -> dict:
    """calc_mesh_params (src/Calc_Mesh.f90:23-220)."""
    NX, NY, NZ = cfg.nx + 4, cfg.ny + 4, cfg.nz + 4
    dz, zcc, zlb = zgrid(cfg)
    shp = (NX, NY, NZ)
    kap = np.zeros(shp, order="F")
    snx = np.zeros(shp, order="F")
    sny = np.zeros(shp, order="F")
    snz = np.zeros(shp, order="F")
    if not cfg.latlon:
        dx, dy = cfg.dx, cfg.dy
        snz[:, :, :] = dy * dx
        for kk in range(NZ):
            snx[:, :, kk] = dz[kk] * dy
            sny[:, :, kk] = dz[kk] * dx
            kap[:, :, kk] = dx * dy * dz[kk]
    else:
        de, dn = cfg.de, cfg.dn
        lat_cc = np.array([cfg.latLL + dn * float(j) - dn * 0.5 for j in range(-1, cfg.ny + 3)])
        for kk in range(NZ):
            r_1 = RAD_EARTH + zcc[kk] - 0.5 * dz[kk]
            r_2 = RAD_EARTH + zcc[kk] + 0.5 * dz[kk]
            rr_1 = r_1 * r_1
            drr = r_2 * r_2 - r_1 * r_1
            drrr = r_2 * r_2 * r_2 - r_1 * r_1 * r_1
            for jj in range(NY):
                phi_1 = DEG2RAD * (lat_cc[jj] - 0.5 * dn)
                phi_2 = DEG2RAD * (lat_cc[jj] + 0.5 * dn)
                theta_1 = 0.5 * PI - phi_1
                theta_2 = 0.5 * PI - phi_2
                del_theta = dn * DEG2RAD
                del_costheta = math.cos(theta_2) - math.cos(theta_1)
                del_lam = de * DEG2RAD
                snx[:, jj, kk] = 0.5 * del_theta * drr
                sny[:, jj, kk] = 0.5 * math.sin(theta_1) * del_lam * drr
                snz[:, jj, kk] = rr_1 * del_lam * del_costheta
                kap[:, jj, kk] = del_lam * drrr * del_costheta / 3.0
    return dict(kappa=kap, sig_nx=snx, sig_ny=sny, sig_nz=snz, dz_vec=dz, z_cc=zcc, z_lb=zlb)


# ---------------------------------------------------------------------------
# terrain (src/Topography.f90, src/Calc_Mesh.f90:237-329)
# ---------------------------------------------------------------------------
def use_topo(cfg: Config) -> bool:
    return cfg.topo_km > 0.0 and cfg.zscaling_id in (1, 2)


def ztop(cfg: Config) -> float:
    """Ztop (km): the top of the computational grid, z_lb(nz+1)."""
    return float(zgrid(cfg)[2][cfg.nz + 2])


def topography(cfg: Config) -> np.ndarray:
    """topo_comp(-1:nx+2,-1:ny+2) in km: a Gaussian hill of height topo_km
    centred on the vent cell.  It stands in for the DEM that Get_Topo reads,
    interpolates and smooths (src/Topography.f90:515-620), host
    preprocessing outside the transport step."""
    ic = np.arange(-1, cfg.nx + 3, dtype=np.float64)
    jc = np.arange(-1, cfg.ny + 3, dtype=np.float64)
    dx, dy = projected_dxdy(cfg)
    X = (ic - cfg.ivent)[:, None] * dx
    Y = (jc - cfg.jvent)[None, :] * dy
    w = cfg.topo_width_km if cfg.topo_width_km > 0.0 else 3.0 * max(dx, dy)
    return np.asfortranarray(cfg.topo_km * np.exp(-(X * X + Y * Y) / (2.0 * w * w)))


def jacobian(cfg: Config) -> np.ndarray:
    """j_cc_pd(-1:nx+2,-1:ny+2) of Get_Topo (src/Topography.f90:608-620)."""
    if cfg.zscaling_id != 2 or not use_topo(cfg):
        return np.ones((cfg.nx + 4, cfg.ny + 4), order="F")
    zt = ztop(cfg)
    return np.asfortranarray((zt - topography(cfg)) / zt)


def topo_fields(cfg: Config) -> dict:
    """Calc_FDGrad_Topo (src/Topography.f90:2471-2536) on the mesh of
    calc_mesh_params (Get_Topo runs before calc_s_mesh scales it,
    src/Ash3d.F90:232-240): dhdx_comp, dhdy_comp, DelDxonD_cc, DelDyonD_cc
    (-1:nx+2,-1:ny+2), plus s_cc_pd (-1:nz+2; s = z for every ZScaling_ID,
    src/Calc_Mesh.f90:271-289) and Ztop.  As in the reference, the interior
    (two-sided) gradient divides the difference over two cells by
    ds = 2*kappa/(sigma_i + sigma_i+1), one cell width, so it is twice the
    slope; the one-sided edge values are the slope itself."""
    g = _geometry_z(cfg)
    kap, snx, sny = g["kappa"], g["sig_nx"], g["sig_ny"]
    topo = topography(cfg)
    zt = ztop(cfg)
    NX, NY = cfg.nx + 4, cfg.ny + 4
    dhdx, dhdy = np.zeros((NX, NY), order="F"), np.zeros((NX, NY), order="F")
    ddx, ddy = np.zeros((NX, NY), order="F"), np.zeros((NX, NY), order="F")
    k1 = 2  # k = 1
    for a in range(NX):          # a = i + 1
        for b in range(NY):      # b = j + 1
            if a == 0:
                ds = kap[a, b, k1] / snx[a, b, k1]
                dhdx[a, b] = (topo[a + 1, b] - topo[a, b]) / ds
                D1, D2, D3 = zt - topo[a, b], zt - topo[a + 1, b], zt - topo[a, b]
                ddx[a, b] = (D2 - D1) / D3
            elif a == NX - 1:
                ds = kap[a, b, k1] / snx[a, b, k1]
                dhdx[a, b] = (topo[a, b] - topo[a - 1, b]) / ds
                D1, D2, D3 = zt - topo[a - 1, b], zt - topo[a, b], zt - topo[a, b]
                ddx[a, b] = (D2 - D1) / D3
            else:
                ds = 2.0 * kap[a, b, k1] / (snx[a, b, k1] + snx[a + 1, b, k1])
                dhdx[a, b] = (topo[a + 1, b] - topo[a - 1, b]) / ds
                D1, D2, D3 = zt - topo[a - 1, b], zt - topo[a + 1, b], zt - topo[a, b]
                ddx[a, b] = 0.5 * (D2 - D1) / D3
            if b == 0:
                ds = kap[a, b, k1] / sny[a, b, k1]
                dhdy[a, b] = (topo[a, b + 1] - topo[a, b]) / ds
                D1, D2, D3 = zt - topo[a, b], zt - topo[a, b + 1], zt - topo[a, b]
                ddy[a, b] = (D2 - D1) / D3
            elif b == NY - 1:
                ds = kap[a, b, k1] / sny[a, b, k1]
                dhdy[a, b] = (topo[a, b] - topo[a, b - 1]) / ds
                D1, D2, D3 = zt - topo[a, b - 1], zt - topo[a, b], zt - topo[a, b]
                ddy[a, b] = (D2 - D1) / D3
            else:
                ds = 2.0 * kap[a, b, k1] / (sny[a, b, k1] + sny[a, b + 1, k1])
                dhdy[a, b] = (topo[a, b + 1] - topo[a, b - 1]) / ds
                D1, D2, D3 = zt - topo[a, b - 1], zt - topo[a, b + 1], zt - topo[a, b]
                ddy[a, b] = 0.5 * (D2 - D1) / D3
    return dict(dhdx=dhdx, dhdy=dhdy, deldx=ddx, deldy=ddy, s_cc=zgrid(cfg)[1].copy(), ztop=zt)


def projected_dxdy(cfg: Config):
    """dx, dy used by Adjust_DT on projected grids (lon/lat: Calc_Mesh.f90:143-149)."""
    if not cfg.latlon:
        return cfg.dx, cfg.dy
    lat_top = cfg.latLL + cfg.dn * (cfg.ny + 1) - cfg.dn * 0.5
    phi_bot = DEG2RAD * (cfg.latLL + cfg.dn * 1 - cfg.dn * 0.5 - cfg.dn * 0.5)
    phi_top = DEG2RAD * (lat_top + cfg.dn * 0.5)
    phi = max(abs(phi_bot), abs(phi_top))
    return RAD_EARTH * cfg.de * DEG2RAD * math.cos(phi), RAD_EARTH * cfg.dn * DEG2RAD


def diffusivity(cfg: Config):
    """kx, ky, kz (0:nx+1,0:ny+1,0:nz+1) in km^2/h (Input_Data.f90:1799-1818)."""
    k = cfg.diffusivity_m2s * M2PS_2_KM2PHR
    shp = (cfg.nx + 2, cfg.ny + 2, cfg.nz + 2)
    return (np.full(shp, k, order="F"), np.full(shp, k, order="F"), np.full(shp, k, order="F"))


def fall_velocity(cfg: Config) -> np.ndarray:
    """vf_pd(-1:nx+2,-1:ny+2,-1:nz+2,1:ns) = -v_s*3.6 (MesoInterpolater.f90:571-572)."""
    vf = np.zeros((cfg.nx + 4, cfg.ny + 4, cfg.nz + 4, cfg.ns), order="F")
    for g in range(cfg.ns):
        vf[:, :, :, g] = (-1.0 * cfg.fall_mps[g]) * MPS_2_KMPHR
    return vf


def fall_velocity_meso(cfg: Config) -> np.ndarray:
    """vf_meso_next_step_sp per grain: real(Tephra_v_s(isize), sp) with
    Tephra_v_s = -v_s (m/s), which Read_NextMesoStep puts in every cell when
    the fall velocities come from the input file (MesoInterpolater.f90:
    567-574)."""
    return np.array([-1.0 * v for v in cfg.fall_mps], dtype=np.float32)


# ---------------------------------------------------------------------------
# synthetic met steps (FP32, m/s, interior nx*ny*nz, i fastest)
# ---------------------------------------------------------------------------
class MetSource:
    """Deterministic generator of hourly FP32 met steps for a workload."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        dz, zcc, _ = zgrid(cfg)
        self.z = zcc[2:cfg.nz + 2]  # km at cell centres
        if cfg.latlon:
            self.lon = np.array([cfg.lonLL + cfg.de * (i + 1) - cfg.de * 0.5 for i in range(cfg.nx)])
            self.lat = np.array([cfg.latLL + cfg.dn * (j + 1) - cfg.dn * 0.5 for j in range(cfg.ny)])
        else:
            self.lon = np.linspace(0.0, 180.0, cfg.nx)
            self.lat = np.linspace(0.0, 90.0, cfg.ny)
        self.steady = cfg.winds == "c1"

    def step(self, hour: int):
        """(vx, vy, vz) FP32 arrays of shape (nx, ny, nz), Fortran order."""
        cfg = self.cfg
        nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
        z = self.z[None, None, :]
        if cfg.winds == "c1":
            u = np.broadcast_to(10.0 + 0.5 * z, (nx, ny, nz))
            v = np.full((nx, ny, nz), 2.0)
            w = np.zeros((nx, ny, nz))
        elif cfg.winds in ("c2", "c2p"):
            lat = self.lat[None, :, None]
            lon = self.lon[:, None, None]
            ztop = 30.0
            u = 40.0 * np.exp(-((lat - 45.0) / 10.0) ** 2) * np.sin(math.pi * z / ztop)
            v = 5.0 * np.sin(2.0 * lon * DEG2RAD) * math.cos(2.0 * math.pi * hour / 24.0)
            u = np.broadcast_to(u, (nx, ny, nz))
            v = np.broadcast_to(v, (nx, ny, nz))
            rng = np.random.default_rng(cfg.seed * 100003 + hour)
            # 5% multiplicative noise, drawn in FP32 to keep generation cheap
            u = u * (1.0 + 0.05 * rng.standard_normal((nx, ny, nz), dtype=np.float32))
            v = v * (1.0 + 0.05 * rng.standard_normal((nx, ny, nz), dtype=np.float32))
            w = np.zeros((nx, ny, nz))
        elif cfg.winds == "const":
            u = np.full((nx, ny, nz), np.float32(cfg.wind_uv[0]))
            v = np.full((nx, ny, nz), np.float32(cfg.wind_uv[1]))
            w = np.zeros((nx, ny, nz))
        elif cfg.winds == "sounding":
            # a 1-D profile (heights in m) at the cell centres: linear in height
            # between its levels, the top level's value above it (the
            # iHeightHandler = 2 rule of the control file), FP32 as met data are
            zs = np.array([p[0] for p in cfg.sounding], dtype=np.float64) / 1000.0
            us = np.array([p[1] for p in cfg.sounding], dtype=np.float64)
            vs = np.array([p[2] for p in cfg.sounding], dtype=np.float64)
            u = np.broadcast_to(np.interp(self.z, zs, us).astype(np.float32), (nx, ny, nz))
            v = np.broadcast_to(np.interp(self.z, zs, vs).astype(np.float32), (nx, ny, nz))
            w = np.zeros((nx, ny, nz))
        else:  # 'random': smooth random field for small parity cases
            rng = np.random.default_rng(cfg.seed * 7919 + hour)
            x = np.linspace(0, 2 * math.pi, nx)[:, None, None]
            y = np.linspace(0, 2 * math.pi, ny)[None, :, None]
            zz = np.linspace(0, 1, nz)[None, None, :]
            a = rng.uniform(-1, 1, 6)
            u = 12.0 * (0.6 + a[0] * np.sin(x + a[1]) * np.cos(y) + 0.5 * zz)
            v = 8.0 * (a[2] + a[3] * np.cos(x) * np.sin(y + a[4]) - 0.3 * zz)
            w = 0.02 * a[5] * np.sin(x) * np.sin(y) * np.ones_like(zz)
            u = u + 0.5 * rng.standard_normal((nx, ny, nz))
            v = v + 0.5 * rng.standard_normal((nx, ny, nz))
        f = lambda a: np.asfortranarray(np.asarray(a, dtype=np.float32).reshape(nx, ny, nz))
        return f(u), f(v), f(w)


# ---------------------------------------------------------------------------
# source, src/Source.f90
# ---------------------------------------------------------------------------
def vent_s_coordinates(cfg: Config):
    """(s_volcano, s_PlumeHeight) of Calc_Normalized_SourceCol
    (src/Source.f90:324-340): the vent elevation and plume top in the
    s-coordinate of ZScaling_ID, Zsurf(ivent,jvent) being the topography at
    the vent."""
    if not use_topo(cfg):
        return cfg.z_volcano, cfg.plume_km
    zs = float(topography(cfg)[cfg.ivent + 1, cfg.jvent + 1])
    zv = max(cfg.z_volcano, zs)
    if cfg.zscaling_id == 1:
        return zv - zs, cfg.plume_km - zs
    zt = ztop(cfg)
    return zt * (zv - zs) / (zt - zs), zt * (cfg.plume_km - zs) / (zt - zs)


def suzuki_column(cfg: Config) -> np.ndarray:
    """NormSourceColumn(1, 1:nz+1) for one eruption (Calc_Normalized_SourceCol,
    src/Source.f90:287-490; the s-grid is the z-grid for every ZScaling_ID)."""
    nz = cfg.nz
    dz, zcc, zlb = zgrid(cfg)
    s_lb = lambda k: zlb[k + 1]
    s_cc = lambda k: zcc[k + 1]
    ds = lambda k: dz[k + 1]
    s_volcano, H = vent_s_coordinates(cfg)
    kground, ktop = 1, 0
    for k in range(1, nz + 1):
        if s_volcano >= s_lb(k) and s_volcano < s_lb(k + 1):
            kground = k
        if H > s_lb(k) and H <= s_lb(k + 1):
            ktop = k
    sground = s_lb(kground)
    Habove = H - sground
    A = cfg.suzuki_a
    sk = A / (1.0 - (A + 1.0) * math.exp(-A))
    col = np.zeros(nz + 1)
    for k in range(kground, ktop + 1):
        top = min(s_cc(k) + 0.5 * ds(k), H)
        bot = s_cc(k) - 0.5 * ds(k)
        sc1 = (top - sground) / Habove
        sc2 = (bot - sground) / Habove
        c1 = 1.0 - sc1
        c2 = 1.0 - sc2
        f1 = 1.0 / A + c1
        f2 = 1.0 / A + c2
        col[k - 1] = sk * (f1 * math.exp(-1.0 * A * c1) - f2 * math.exp(-1.0 * A * c2))
    return col / col.sum()


def mass_flux_rate(cfg: Config) -> float:
    """EruptivePulse_MassFluxRate (src/Source.f90:508-592), kg/h."""
    return cfg.magma_density * cfg.volume_km3 * KM3_2_M3 / cfg.duration_h


def pulse_fraction(cfg: Config, time: float, dt: float) -> float:
    """dt_pulse_frac of CheckEruptivePulses (src/Source.f90:613-685), one pulse from t=0."""
    t0, t1 = 0.0, cfg.duration_h
    tstart, tend = time, time + dt
    contributes = ((tstart >= t0 and tstart < t1) or (tend > t0 and tend <= t1)
                   or (tstart < t0 and tend > t1))
    if not contributes:
        return 0.0
    return (min(tend, t1) - max(tstart, t0)) / dt


def eruption_pulses(cfg: Config):
    """(start_h, end_h, MassFluxRate kg/h) per eruptive pulse: one pulse from t = 0."""
    return [(0.0, 0.0 + cfg.duration_h, mass_flux_rate(cfg))]


def scheduled_source_flux(cfg: Config, pulses, norm_col: np.ndarray, kappa: np.ndarray, state: list,
                          time: float, dt: float):
    """CheckEruptivePulses + TephraSourceNodes (src/Source.f90:613-783) for
    the pulses, with state = [ieruption, jeruption] (1-based, updated): the
    SourceNodeFlux (nz+1) x ns of this step, or None when no pulse is active.
    The same operations as the device's a3g_add_source_scheduled."""
    tstart, tend = time, time + dt
    ie, je = state
    frac = [0.0] * (len(pulses) + 1)
    active = False
    for i in range(ie, len(pulses) + 1):
        t0, t1, _ = pulses[i - 1]
        pc = False
        if tstart >= t0 and tstart < t1:
            pc, je = True, i
        elif tend > t0 and tend <= t1:
            je = i   # the reference exits here before forming this pulse's fraction
            break
        elif tstart < t0 and tend > t1:
            pc, je = True, i
        if pc:
            active = True
            frac[i] = (min(tend, t1) - max(tstart, t0)) / dt
    state[1] = je
    if not active:
        return None
    nz, ns = cfg.nz, cfg.ns
    cols = np.asarray(norm_col, dtype=np.float64).reshape(len(pulses), nz + 1)
    tfr = np.zeros(nz)
    for i in range(ie, je + 1):
        tfr = tfr + pulses[i - 1][2] * frac[i] * cols[ie - 1, :nz]
    flux = np.zeros((nz + 1, ns), order="F")
    iv, jv = cfg.ivent, cfg.jvent
    for k in range(1, nz + 1):
        kap = kappa[iv + 1, jv + 1, k + 1]
        for g in range(ns):
            flux[k - 1, g] = cfg.bin_mass[g] * tfr[k - 1] / kap
    state[0] = je
    return flux


def source_flux(cfg: Config, norm_col: np.ndarray, kappa: np.ndarray, frac: float) -> np.ndarray:
    """SourceNodeFlux(1:nz+1, 1:ns) (k fastest) of TephraSourceNodes, kg/km^3/h."""
    nz, ns = cfg.nz, cfg.ns
    mfr = mass_flux_rate(cfg)
    flux = np.zeros((nz + 1, ns), order="F")
    tfr = np.zeros(nz)
    tfr[:] = 0.0 + mfr * frac * norm_col[:nz]
    iv, jv = cfg.ivent, cfg.jvent
    for k in range(1, nz + 1):
        kap = kappa[iv + 1, jv + 1, k + 1]
        for g in range(ns):
            flux[k - 1, g] = cfg.bin_mass[g] * tfr[k - 1] / kap
    return flux


# ---------------------------------------------------------------------------
# umbrella cloud source (src/Source_Umbrella.f90, src/Ash3d.F90:435-463,
# src/MesoInterpolater.f90:233-248).  Host-side, in the reference's
# operations (the transcendental functions are the C library's, as
# gfortran's are); the device adds the winds and inserts the patch.
# ---------------------------------------------------------------------------
def is_umbrella(cfg: Config) -> bool:
    return cfg.source_type in ("umbrella", "umbrella_air")


def lon_cc(cfg: Config, i: int) -> float:
    return cfg.lonLL + cfg.de * float(i) - cfg.de * 0.5   # src/Calc_Mesh.f90:106


def lat_cc(cfg: Config, j: int) -> float:
    return cfg.latLL + cfg.dn * float(j) - cfg.dn * 0.5   # src/Calc_Mesh.f90:109


def vent_lonlat(cfg: Config):
    """(lon_volcano, lat_volcano): the centre of the vent cell."""
    return lon_cc(cfg, cfg.ivent), lat_cc(cfg, cfg.jvent)


@dataclasses.dataclass
class UmbrellaSetup:
    ibase: int
    itop: int
    stencil: np.ndarray    # AvgStenc_Umbrella(3,3,nz), Fortran order
    scalefac: np.ndarray   # ScaleFac_Umbrella(1:nz)


def umbrella_setup(cfg: Config, kappa: np.ndarray) -> UmbrellaSetup:
    """Allocate_Source_Umbrella (src/Source_Umbrella.f90:85-153): the
    volume-weighted 3x3 averaging stencil and the vent-to-patch scale factor
    per level, and the levels ibase..itop of the umbrella."""
    if not cfg.latlon:
        raise ValueError("umbrella_winds is not set up for projected coordinates (Source_Umbrella.f90:252-259)")
    nz = cfg.nz
    kap = lambda i, j, k: kappa[i + 1, j + 1, k + 1]
    sten = np.zeros((3, 3, nz), order="F")
    fac = np.zeros(nz)
    for k in range(1, nz + 1):
        tot = 0.0
        for i in range(1, 4):
            ii = cfg.ivent - 2 + i
            for j in range(1, 4):
                jj = cfg.jvent - 2 + j
                sten[i - 1, j - 1, k - 1] = kap(ii, jj, k)
                tot = tot + kap(ii, jj, k)
        fac[k - 1] = kap(cfg.ivent, cfg.jvent, k) / tot
        sten[:, :, k - 1] = sten[:, :, k - 1] / tot
    dz = zgrid(cfg)[0]
    zvi = np.zeros(nz + 1)   # z_vec_init(0:nz), the level tops
    for k in range(1, nz + 1):
        zvi[k] = zvi[k - 1] + dz[k + 1] if cfg.dz_profile else cfg.dz * k
    itop = ibase = 0
    H = cfg.plume_km
    for k in range(1, nz + 1):
        if zvi[k] >= H and zvi[k - 1] < H:
            itop = k
        if zvi[k] >= 0.75 * H and zvi[k - 1] < 0.75 * H:
            ibase = k
    return UmbrellaSetup(ibase, itop, sten, fac)


def umbrella_winds(cfg: Config, time: float, dt: float, first_time: bool = False):
    """umbrella_winds (src/Source_Umbrella.f90:206-394): the radial winds
    (km/h) of the spreading umbrella cloud, constant over ibase..itop.
    Returns (i0, i1, j0, j1, uvx, uvy) with uvx, uvy over the bounding box
    of the cloud (i fastest), or None while the cloud is within the source
    nodes."""
    lon_v, lat_v = vent_lonlat(cfg)
    mfr = mass_flux_rate(cfg) / HR_2_S                 # kg/s
    if cfg.source_type == "umbrella_air" and cfg.ns == 1:
        mfr = 20.0 * mfr
    c_costa = 0.43e3 if abs(lat_v) < 23.0 else 0.87e3
    qnow = c_costa * math.sqrt(UMB_K_ENTRAIN) * mfr ** (3.0 / 4.0) / UMB_N_BV ** (5.0 / 4.0)
    if not first_time:
        etime_s = max(time, dt) * HR_2_S
    else:
        etime_s = min(cfg.sim_hours, cfg.duration_h) * HR_2_S
    cloud_radius = (3.0 * UMB_LAMBDA * UMB_N_BV * qnow / (2.0 * PI)) ** (1.0 / 3.0) * \
        etime_s ** (2.0 / 3.0) / KM_2_M
    edge_speed = (2.0 / 3.0) * (3.0 * UMB_LAMBDA * UMB_N_BV * qnow / (2.0 * PI)) ** (1.0 / 3.0) * \
        etime_s ** (-1.0 / 3.0)
    de_km = cfg.de * math.cos(lat_v * DEG2RAD) * DEG2KMLON   # src/Calc_Mesh.f90:103-104
    dn_km = cfg.dn * DEG2KMLAT
    if cloud_radius <= max((3.0 / 2.0) * de_km, (3.0 / 2.0) * dn_km):
        return None
    ew_nodes = int(cloud_radius / de_km) + 1
    ns_nodes = int(cloud_radius / dn_km) + 1
    i0, i1 = max(1, cfg.ivent - ew_nodes), min(cfg.nx, cfg.ivent + ew_nodes)
    j0, j1 = max(1, cfg.jvent - ns_nodes), min(cfg.ny, cfg.jvent + ns_nodes)
    uvx = np.zeros((i1 - i0 + 1, j1 - j0 + 1), order="F")
    uvy = np.zeros_like(uvx)
    for ii in range(i0, i1 + 1):
        for jj in range(j0, j1 + 1):
            if ii == cfg.ivent and jj == cfg.jvent:
                continue
            avg_lat = (lat_cc(cfg, jj) + lat_v) / 2.0
            ns_km = (lat_cc(cfg, jj) - lat_v) * DEG2KMLAT
            ew_km = (lon_cc(cfg, ii) - lon_v) * math.cos(avg_lat * DEG2RAD) * DEG2KMLON
            # x**2.0_ip is folded to x*x by gfortran
            radnow = math.sqrt(ns_km * ns_km + ew_km * ew_km)
            if radnow < cloud_radius:
                if UMB_VELMOD == 1:
                    rexp = 3.0
                    w = edge_speed * MPS_2_KMPHR * (3.0 / 4.0) * (cloud_radius / radnow) * \
                        (1.0 + (1.0 / 3.0) * (radnow / cloud_radius) ** rexp)
                else:
                    w = edge_speed * MPS_2_KMPHR * (cloud_radius / radnow) ** 0.5
                theta = math.atan2(ns_km, ew_km)
                uvx[ii - i0, jj - j0] = w * math.cos(theta)
                uvy[ii - i0, jj - j0] = w * math.sin(theta)
    return i0, i1, j0, j1, uvx, uvy


def umbrella_flux(cfg: Config, flux: np.ndarray, um: UmbrellaSetup) -> np.ndarray:
    """TephraSourceNodes_Umbrella (src/Source_Umbrella.f90:409-448):
    SourceNodeFlux_Umbrella(3,3,nz+1,ns) from the vent column's flux."""
    nz = cfg.nz
    f = np.zeros((3, 3, nz + 1, cfg.ns), order="F")
    for k in range(1, nz + 2):
        if k < um.ibase:
            f[1, 1, k - 1, :] = flux[k - 1, :]
        elif k <= um.itop:
            f[:, :, k - 1, :] = flux[k - 1, :][None, None, :] * um.scalefac[k - 1]
    return f


def umbrella_vol_inc(cfg: Config, flux: np.ndarray, um: UmbrellaSetup, kappa: np.ndarray, dt: float) -> float:
    """SourceVolInc_Umbrella (src/Source_Umbrella.f90:464-522), km^3 DRE."""
    tmp = 0.0
    iv, jv = cfg.ivent, cfg.jvent
    for g in range(cfg.ns):
        for k in range(1, um.ibase):
            tmp = tmp + dt * flux[k - 1, g] * kappa[iv + 1, jv + 1, k + 1] / cfg.magma_density / KM3_2_M3
    for i in range(3):
        for j in range(3):
            for k in range(um.ibase, um.itop + 1):
                for g in range(cfg.ns):
                    tmp = tmp + dt * flux[k - 1, g] * um.stencil[i, j, k - 1] * \
                        kappa[iv + 1, jv + 1, k + 1] / cfg.magma_density / KM3_2_M3
    return tmp


def source_vol_inc(cfg: Config, flux: np.ndarray, kappa: np.ndarray, dt: float) -> float:
    """SourceVolInc (src/Source.f90:798-836), km^3 DRE."""
    tmp = 0.0
    iv, jv = cfg.ivent, cfg.jvent
    for k in range(1, cfg.nz + 2):
        for g in range(cfg.ns):
            tmp = tmp + dt * flux[k - 1, g] * kappa[iv + 1, jv + 1, k + 1] / cfg.magma_density / KM3_2_M3
    return tmp
