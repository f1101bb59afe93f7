"""The umbrella-cloud source (SourceType 'umbrella', src/Source_Umbrella.f90)
in its host-side restatement and in the oracle, on the CPU: the averaging
stencil and levels of Allocate_Source_Umbrella, the radial winds of
umbrella_winds, and a run that keeps the erupted mass (the 3x3 smoothing
and insertion conserve it, and SourceVolInc_Umbrella counts it)."""
import math

import numpy as np

import ash3d_oracle as orc
from volcano_ash3d_b200 import driver
from volcano_ash3d_b200 import synthetic as syn


def test_umbrella_setup():
    cfg = syn.make_config("tiny_umbrella")
    geo = syn.geometry(cfg)
    u = syn.umbrella_setup(cfg, geo["kappa"])
    assert (u.ibase, u.itop) == (12, 15)  # 0.75*15 km and 15 km with 1 km levels
    np.testing.assert_allclose(u.stencil.sum(axis=(0, 1)), 1.0, rtol=1e-14)
    kap = geo["kappa"][cfg.ivent + 1, cfg.jvent + 1, 2:cfg.nz + 2]
    tot = geo["kappa"][cfg.ivent:cfg.ivent + 3, cfg.jvent:cfg.jvent + 3, 2:cfg.nz + 2].sum(axis=(0, 1))
    np.testing.assert_allclose(u.scalefac, kap / tot, rtol=1e-14)
    f = syn.umbrella_flux(cfg, np.ones((cfg.nz + 1, cfg.ns)), u)
    assert f[1, 1, u.ibase - 2, 0] == 1.0 and f[0, 0, u.ibase - 2, 0] == 0.0   # below: vent column only
    assert f[0, 0, u.ibase - 1, 0] == u.scalefac[u.ibase - 1]                    # inside: the patch
    assert not f[:, :, u.itop:, :].any()                                          # above: nothing


def test_umbrella_winds_are_radial():
    cfg = syn.make_config("tiny_umbrella")
    assert syn.umbrella_winds(cfg, 0.0, 1e-4) is None  # the cloud is still inside the 3x3 nodes
    i0, i1, j0, j1, uvx, uvy = syn.umbrella_winds(cfg, 0.5, 0.01)
    lon_v, lat_v = syn.vent_lonlat(cfg)
    n_in = 0
    for a in range(i1 - i0 + 1):
        for b in range(j1 - j0 + 1):
            i, j = i0 + a, j0 + b
            ew = syn.lon_cc(cfg, i) - lon_v
            ns = syn.lat_cc(cfg, j) - lat_v
            w = math.hypot(uvx[a, b], uvy[a, b])
            if (i, j) == (cfg.ivent, cfg.jvent):
                assert w == 0.0
            elif w > 0.0:
                n_in += 1
                assert uvx[a, b] * ew + uvy[a, b] * ns > 0.0  # outward
    assert n_in > 20
    # the speed falls off away from the vent
    assert math.hypot(uvx[cfg.ivent - i0 + 1, cfg.jvent - j0], uvy[cfg.ivent - i0 + 1, cfg.jvent - j0]) > \
        math.hypot(uvx[cfg.ivent - i0 + 4, cfg.jvent - j0], uvy[cfg.ivent - i0 + 4, cfg.jvent - j0])


def test_umbrella_run_conserves_mass():
    cfg = syn.make_config("tiny_umbrella")
    m = orc.OracleModel(cfg, threads=1)
    st = driver.run(m, cfg, max_steps=25)
    h = st.history[-1]
    assert h.source_cum > 0.0
    np.testing.assert_allclose(h.tot, h.source_cum, rtol=1e-11)
    # mass left the vent column sideways at the umbrella levels
    q = m.interior()
    assert q[cfg.ivent - 1 + 3, cfg.jvent - 1, 12:15, 0].max() > 0.0
