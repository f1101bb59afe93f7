"""Terrain-following transport (useTopo, ZScaling_ID 1 and 2) in the oracle
and in the host-side terrain inputs, on the CPU.

* Calc_FDGrad_Topo's gradients and DelD*onD_cc (synthetic.topo_fields)
  against centred / one-sided differences;
* vh (Calc_Vmod_Topo) against a numpy restatement, bit for bit;
* zero topography through the terrain path reproduces the plain run bit for
  bit (the plumbing adds nothing when the terrain is flat);
* the DelD*onD_cc terms cancel between a cell's two interfaces in exact
  arithmetic (fs_r(I) gains T(I), fs_l(I+1) loses it), so a run with them
  matches a run without them to rounding; a term placed on the wrong
  interface would not cancel;
* the run conserves mass: airborne + deposited + outflow volume equals the
  erupted volume.
"""
import dataclasses

import numpy as np
import pytest

import ash3d_oracle as orc
from topo_common import level_winds, topo_config, vh_restated
from volcano_ash3d_b200 import driver
from volcano_ash3d_b200 import synthetic as syn


def test_fd_gradients_and_deld():
    cfg = topo_config("tiny_proj", 2)
    f = syn.topo_fields(cfg)
    t = syn.topography(cfg)
    zt = syn.ztop(cfg)
    # interior: the reference divides the difference over two cells by
    # ds = 2 kappa / (sig + sig'), which is ONE cell width (Topography.f90
    # :2502-2503), so its dhdx is twice the slope there; restated as is
    np.testing.assert_allclose(f["dhdx"][1:-1, :], (t[2:, :] - t[:-2, :]) / cfg.dx, rtol=1e-12)
    np.testing.assert_allclose(f["dhdy"][:, 1:-1], (t[:, 2:] - t[:, :-2]) / cfg.dy, rtol=1e-12)
    # edges: one-sided
    np.testing.assert_allclose(f["dhdx"][0, :], (t[1, :] - t[0, :]) / cfg.dx, rtol=1e-12)
    np.testing.assert_allclose(f["dhdx"][-1, :], (t[-1, :] - t[-2, :]) / cfg.dx, rtol=1e-12)
    D = zt - t
    np.testing.assert_allclose(f["deldx"][1:-1, :], 0.5 * (D[2:, :] - D[:-2, :]) / D[1:-1, :], rtol=1e-12)
    np.testing.assert_allclose(f["deldy"][:, -1], (D[:, -1] - D[:, -2]) / D[:, -1], rtol=1e-12)
    # a hill: the gradient points away from the vent
    iv, jv = cfg.ivent + 1, cfg.jvent + 1
    assert f["dhdx"][iv - 2, jv] > 0 > f["dhdx"][iv + 2, jv]
    # scaled geometry: kappa and the side faces shrink by (Ztop - Zsurf)/Ztop
    g, g0 = syn.geometry(cfg), syn.geometry(dataclasses.replace(cfg, topo_km=0.0))
    jcc = (zt - t) / zt
    np.testing.assert_array_equal(g["kappa"], g0["kappa"] * jcc[:, :, None])
    np.testing.assert_array_equal(g["sig_nz"], g0["sig_nz"])


@pytest.mark.parametrize("z", [1, 2])
def test_vmod_topo_bitwise(z):
    cfg = topo_config("tiny_proj", z)
    m = orc.OracleModel(cfg, threads=1)
    vx, vy, vz = level_winds(cfg, 3)
    m.set_winds(vx, vy, vz)
    ref = vh_restated(cfg, vx, vy, syn.topo_fields(cfg))
    assert np.array_equal(m.vh, ref)
    assert np.abs(m.vh).max() > 0.0
    assert not np.any(m.vh[:, :, :2]) and not np.any(m.vh[:, :, -2:])  # ghost levels


@pytest.mark.parametrize("z", [1, 2])
def test_zero_topography_is_plain_run(z):
    cfg0 = syn.make_config("tiny_cn")
    cfg = dataclasses.replace(cfg0, zscaling_id=z)
    plain = orc.OracleModel(cfg0, threads=1)
    flat = orc.OracleModel(cfg, threads=1)
    zeros = np.zeros((cfg.nx + 4, cfg.ny + 4), order="F")
    dz, zcc, zlb = syn.zgrid(cfg)
    flat.set_topo(zeros, zeros, zeros, zeros, zcc, syn.ztop(cfg))
    driver.run(plain, cfg0, max_steps=10)
    driver.run(flat, cfg, max_steps=10)
    assert np.array_equal(plain.interior(), flat.interior())


def test_deld_terms_cancel_to_rounding():
    cfg = topo_config("tiny_cn", 2)
    fields = syn.topo_fields(cfg)
    with_terms = orc.OracleModel(cfg, threads=1)
    without = orc.OracleModel(cfg, threads=1)
    zeros = np.zeros_like(fields["deldx"])
    without.set_topo(fields["dhdx"], fields["dhdy"], zeros, zeros, fields["s_cc"], fields["ztop"])
    assert np.abs(fields["deldx"]).max() > 0.01
    driver.run(with_terms, cfg, max_steps=12)
    driver.run(without, cfg, max_steps=12)
    a, b = with_terms.interior(), without.interior()
    assert not np.array_equal(a, b)  # the terms are there ...
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max())  # ... and cancel


@pytest.mark.parametrize("z", [1, 2])
def test_terrain_run_conserves_mass(z):
    cfg = topo_config("tiny_proj", z)
    m = orc.OracleModel(cfg, threads=1)
    st = driver.run(m, cfg, max_steps=20)
    h = st.history[-1]
    assert h.source_cum > 0.0
    np.testing.assert_allclose(h.tot, h.source_cum, rtol=1e-11)
    assert np.abs(m.vh).max() > 0.0


def test_source_column_in_s_coordinates():
    cfg = topo_config("tiny_proj", 2)
    s_vent, s_top = syn.vent_s_coordinates(cfg)
    zs = syn.topography(cfg)[cfg.ivent + 1, cfg.jvent + 1]
    zt = syn.ztop(cfg)
    assert s_vent == 0.0
    assert s_top == zt * (cfg.plume_km - zs) / (zt - zs)
    assert syn.vent_s_coordinates(dataclasses.replace(cfg, zscaling_id=1)) == (0.0, cfg.plume_km - zs)
    col = syn.suzuki_column(cfg)
    assert abs(col.sum() - 1.0) < 1e-12
