"""FAST_DT in the oracle (the reference's default build, src/makefile:91).

* the met-step maxima of Adjust_DT(mesostep=.true.) (src/Adjust_dt.f90:96-135)
  against a numpy restatement of the same FP32/FP64 operations, for
  projected and lon/lat grids and for per-grain and per-cell fall speeds;
* every step's dt is the met steps' dt interpolated at Interval_Frac and
  clipped (src/MesoInterpolater.f90:250-258), and dt_meso_last/next move at
  the met-step loads as :142-150 and :187-195 move them;
* a time that lands exactly on an hour keeps the old met pair at
  Interval_Frac = 1 (the strict test of :135);
* a FAST_DT run with FAST_SUBGRID conserves mass to 1e-12.
"""
import dataclasses
import math

import numpy as np
import pytest

import ash3d_oracle as orc
from volcano_ash3d_b200 import driver
from volcano_ash3d_b200 import synthetic as syn


def _maxima_numpy(cfg, geo, vx, vy, vz, vfm):
    """src/Adjust_dt.f90:96-135 with numpy: FP32 |v|, widened, *3.6."""
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    kap = geo["kappa"][2:nx + 2, 2:ny + 2, 2:nz + 2]
    if cfg.latlon:
        snx, sny = geo["sig_nx"], geo["sig_ny"]
        mx = np.minimum(snx[2:nx + 2, 2:ny + 2, 2:nz + 2], snx[3:nx + 3, 2:ny + 2, 2:nz + 2])
        my = np.minimum(sny[2:nx + 2, 2:ny + 2, 2:nz + 2], sny[2:nx + 2, 3:ny + 3, 2:nz + 2])
        v0 = (np.abs(vx).astype(np.float64) * 3.6 * mx / kap).max()
        v1 = (np.abs(vy).astype(np.float64) * 3.6 * my / kap).max()
    else:
        v0 = float(np.abs(vx).max()) * 3.6
        v1 = float(np.abs(vy).max()) * 3.6
    s = (np.abs(vz) + vfm).astype(np.float32)  # the FP32 sum
    dz = geo["dz_vec"][2:nz + 2]
    v2 = (s.astype(np.float64) * 3.6 / dz[None, None, :]).max()
    return np.array([v0, v1, v2])


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_latlon", "tiny_periodic", "tiny_stretch"])
@pytest.mark.parametrize("per_grain", [True, False])
def test_meso_maxima_match_numpy_restatement(name, per_grain):
    cfg = syn.make_config(name)
    geo = syn.geometry(cfg)
    m = orc.OracleModel(cfg, geo=geo)
    met = syn.MetSource(cfg)
    last, nxt = met.step(0), met.step(1)
    m.set_met_steps(last, nxt)
    rng = np.random.default_rng(3)
    if per_grain:
        vf = syn.fall_velocity_meso(cfg)
        vfm = np.float32(np.abs(vf).max())
    else:  # a fall speed per cell and grain, as Set_Vf_Meso gives
        vf = np.asfortranarray(-rng.uniform(0.0, 2.0, (cfg.nx, cfg.ny, cfg.nz, cfg.ns)).astype(np.float32))
        vfm = np.abs(vf).max(axis=3)
    m.set_fall_velocity_meso(vf, per_grain=per_grain)
    for slot, (vx, vy, vz) in ((0, last), (1, nxt)):
        got = m.cfl_maxima_meso(slot)
        want = _maxima_numpy(cfg, geo, vx, vy, vz, vfm)
        assert np.array_equal(got, want), (slot, got, want)


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn", "tiny_latlon"])
def test_fast_dt_sequence_interpolates_met_step_dts(name):
    cfg = dataclasses.replace(syn.make_config(name), fast_dt=True)
    m = orc.OracleModel(cfg)
    st = driver.new_state(cfg)
    metdt = {}  # hour -> (dt_meso_last, dt_meso_next) after that hour's load
    prev_hour = -1
    while st.time < cfg.sim_hours:
        t0 = st.time
        rec = driver.step(m, st)
        if st.hour != prev_hour:
            metdt[st.hour] = (m.dt_meso_last, m.dt_meso_next)
            prev_hour = st.hour
        last, nxt = metdt[st.hour]
        frac = t0 - st.hour
        want = last + (nxt - last) * frac
        if t0 + want > cfg.sim_hours:
            want = cfg.sim_hours - t0
        assert rec.dt == want, (rec.itime, rec.dt, want)
    # the toggle: every later load's dt_meso_last is the previous load's dt_meso_next
    hours = sorted(metdt)
    assert len(hours) >= 2
    for a, b in zip(hours, hours[1:]):
        assert metdt[b][0] == metdt[a][1]
    # and the met steps' dt differ (the winds change by the hour), so the
    # interpolation is exercised
    assert any(v[0] != v[1] for v in metdt.values())


def test_met_pair_kept_when_time_lands_on_the_hour():
    """Output times clip dt so that the time lands on 1.0 h exactly; the next
    step still interpolates hour 0's pair at Interval_Frac = 1."""
    cfg = dataclasses.replace(syn.make_config("tiny_proj"), fast_dt=True)
    m = orc.OracleModel(cfg)
    st = driver.new_state(cfg)
    seen = []
    while st.time < 1.5:
        t0 = st.time
        driver.step(m, st, write_times=[1.0, 2.0])
        seen.append((t0, st.hour))
    on_hour = [(t, h) for t, h in seen if t == 1.0]
    assert on_hour == [(1.0, 0)]
    assert any(t > 1.0 and h == 1 for t, h in seen)


@pytest.mark.parametrize("name", ["tiny_subgrid", "C1"])
def test_fast_dt_and_subgrid_run_conserves_mass(name):
    cfg = dataclasses.replace(syn.make_config(name), fast_dt=True, fast_subgrid=True)
    if name == "C1":
        cfg.sim_hours = 1.5
    m = orc.OracleModel(cfg)
    st = driver.run(m, cfg)
    last = st.history[-1]
    assert last.source_cum > 0.0
    assert abs(last.tot - last.source_cum) <= 1e-12 * last.source_cum
    assert math.isclose(last.time, cfg.sim_hours, rel_tol=0, abs_tol=1e-12)
