"""The NetCDF output arrays (ashcon, depocon) and the restart load in the
oracle, on the CPU (src/write_NETCDF.f90:3287-3330 and
NC_RestartFile_LoadConcen :3646-3716).

* ashcon is the state rounded to FP32 (x fastest); ts0 and ts1 agree at
  output time, so it does not matter which level the writer reads;
* depocon is DepositGranularity*dz_vec_pd(0)/KM2_2_M2 rounded to FP32, with
  values <= EPS_SMALL (negative deposits included) written as 0;
* output -> restart -> output returns ashcon unchanged (FP32 -> FP64 -> FP32
  is exact) and depocon scaled once more by dz_vec_pd(0)/KM2_2_M2: the
  reference loads the file's kg/m^2 into outflow_xy1 without undoing the
  writer's scaling, and that is restated as is;
* a model restarted from the arrays continues exactly like the model that
  wrote them, once that model is reloaded from the same arrays.
"""
import copy

import numpy as np

import ash3d_oracle as orc
from volcano_ash3d_b200 import driver
from volcano_ash3d_b200 import synthetic as syn


def _ran(name="tiny_proj", steps=10):
    cfg = syn.make_config(name)
    m = orc.OracleModel(cfg, threads=1)
    st = driver.run(m, cfg, max_steps=steps)
    return cfg, m, st


def test_ashcon_is_the_state_in_fp32():
    cfg, m, _ = _ran()
    ash, _ = m.output_ashcon()
    assert ash.dtype == np.float32 and ash.shape == (cfg.nx, cfg.ny, cfg.nz, cfg.ns)
    assert ash.flags.f_contiguous
    q = m.interior()
    assert np.array_equal(m.concen[2:cfg.nx + 2, 2:cfg.ny + 2, 2:cfg.nz + 2, :, 1], q)  # ts1 == ts0
    assert np.array_equal(ash, q.astype(np.float32))
    assert ash.max() > 0.0


def test_depocon_scaling_and_threshold():
    cfg, m, _ = _ran(steps=14)
    dz0 = syn.zgrid(cfg)[0][1]  # dz_vec_pd(0) = dz_vec_pd(1)
    m.deposit[0, 0, 0] = -5.0                     # an upward wind at the ground can give this
    m.deposit[1, 0, 0] = 1.0e-6 * 1.0e6 / dz0     # exactly at EPS_SMALL after scaling (or within rounding)
    m.deposit[2, 0, 0] = 0.0
    _, dep = m.output_ashcon()
    assert dep.dtype == np.float32 and dep.shape == (cfg.nx, cfg.ny, cfg.ns)
    exact = m.deposit * dz0 / 1.0e6
    keep = dep != 0.0
    assert np.all(dep[keep].astype(np.float64) > 1.0e-6)
    assert np.all(exact[~keep].astype(np.float32).astype(np.float64) <= 1.0e-6)
    np.testing.assert_allclose(dep[keep], exact[keep], rtol=2.0 ** -24, atol=0)
    assert dep[0, 0, 0] == 0.0 and dep[2, 0, 0] == 0.0
    assert keep.any()


def test_output_restart_output():
    cfg, m, _ = _ran(steps=14)
    dz0 = syn.zgrid(cfg)[0][1]
    ash, dep = m.output_ashcon()
    fresh = orc.OracleModel(cfg, threads=1)
    fresh.restart_load(ash, dep)
    ash2, dep2 = fresh.output_ashcon()
    assert np.array_equal(ash2, ash)
    twice = (dep.astype(np.float64) * dz0 / 1.0e6).astype(np.float32)
    twice[twice.astype(np.float64) <= 1.0e-6] = 0.0
    assert np.array_equal(dep2, twice)
    assert np.array_equal(fresh.outflows()["xy1"], dep.astype(np.float64))
    assert np.array_equal(fresh.deposit, dep.astype(np.float64))


def test_restarted_run_continues_like_the_writer():
    cfg, a, st_a = _ran(steps=8)
    ash, dep = a.output_ashcon()
    b = orc.OracleModel(cfg, threads=1)
    for m in (a, b):
        m.restart_load(ash, dep)
    st_b = copy.deepcopy(st_a)
    st_b.hour = -1  # b has no met steps yet: the first step uploads the pair
    for _ in range(6):
        ra = driver.step(a, st_a)
        rb = driver.step(b, st_b)
        assert ra.dt == rb.dt
    assert np.array_equal(a.interior(), b.interior())
    assert np.array_equal(a.outflows()["xy1"], b.outflows()["xy1"])
