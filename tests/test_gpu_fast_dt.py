"""FAST_DT on the GPU against the oracle: the reference's default build
(FASTFPPFLAG = -DFAST_DT -DFAST_SUBGRID, src/makefile:91).

* the met-step maxima (a3g_cfl_maxima_meso) bit for bit, both met slots,
  per-grain and per-cell fall speeds;
* whole runs with FAST_DT, alone and with FAST_SUBGRID, across met-step
  loads: the dt sequence and the state bit for bit, totals to 1e-13;
* the full C1 workload with both flags on;
* the lag-one loop (dt interpolated on the device, met-step dt computed on
  the device without a read-back) against the oracle's plain loop;
* a C2 slab (full 720-cell rows) with both flags on, started just before an
  hour so that a met step loads inside the run.
"""
import dataclasses

import numpy as np
import pytest

import ash3d_oracle as orc
from volcano_ash3d_b200 import driver
from volcano_ash3d_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _pair(cfg):
    from volcano_ash3d_b200.model import Ash3dGPU
    geo = syn.geometry(cfg)
    return Ash3dGPU(cfg, geo=geo), orc.OracleModel(cfg, geo=geo)


def _assert_same_run(sg, sr, gpu, ref):
    assert [h.dt for h in sg.history] == [h.dt for h in sr.history]
    assert np.array_equal(gpu.interior(), ref.interior())
    og, orf = gpu.outflows(), ref.outflows()
    for key in og:
        assert np.array_equal(og[key], orf[key]), key
    for a, b in zip(sg.history, sr.history):
        np.testing.assert_allclose([a.aloft, a.dep, a.outflow, a.tot], [b.aloft, b.dep, b.outflow, b.tot],
                                   rtol=1e-13, atol=1e-30)


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_latlon", "tiny_periodic", "tiny_stretch"])
@pytest.mark.parametrize("per_grain", [True, False])
def test_meso_maxima_bitwise(name, per_grain):
    cfg = syn.make_config(name)
    gpu, ref = _pair(cfg)
    met = syn.MetSource(cfg)
    for m in (gpu, ref):
        m.set_met_steps(met.step(3), met.step(4))
    if not per_grain:
        rng = np.random.default_rng(7)
        vf = np.asfortranarray(-rng.uniform(0.0, 2.0, (cfg.nx, cfg.ny, cfg.nz, cfg.ns)).astype(np.float32))
        for m in (gpu, ref):
            m.set_fall_velocity_meso(vf, per_grain=False)
    for slot in (0, 1):
        g, r = gpu.cfl_maxima_meso(slot), ref.cfl_maxima_meso(slot)
        assert np.array_equal(g, r), (slot, g, r)
    gpu.close()


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn", "tiny_latlon", "tiny_periodic", "tiny_subgrid",
                                  "tiny_stretch"])
@pytest.mark.parametrize("subgrid", [False, True])
def test_fast_dt_run_bitwise(name, subgrid):
    cfg = dataclasses.replace(syn.make_config(name), fast_dt=True, fast_subgrid=subgrid)
    cfg.sim_hours = max(cfg.sim_hours, 1.5)  # past the second met-step load
    gpu, ref = _pair(cfg)
    sg = driver.run(gpu, cfg)
    sr = driver.run(ref, cfg)
    assert sg.hour >= 1 and len(sg.history) > 10  # crossed at least one met-step load
    _assert_same_run(sg, sr, gpu, ref)
    gpu.close()


def test_fast_dt_umbrella_suppressed_while_spreading():
    """FastDt_suppress (src/MesoInterpolater.f90:233-248): the umbrella's own
    winds set dt with Adjust_DT(.false.) while the eruption lasts, FAST_DT
    afterwards."""
    cfg = dataclasses.replace(syn.make_config("tiny_umbrella"), fast_dt=True)
    gpu, ref = _pair(cfg)
    sg = driver.run(gpu, cfg)
    sr = driver.run(ref, cfg)
    assert sg.history[-1].time > cfg.duration_h
    _assert_same_run(sg, sr, gpu, ref)
    gpu.close()


def test_c1_default_build_full_run_bitwise():
    cfg = dataclasses.replace(syn.make_config("C1"), fast_dt=True, fast_subgrid=True)
    gpu, ref = _pair(cfg)
    sg = driver.run(gpu, cfg)
    sr = driver.run(ref, cfg)
    assert len(sg.history) > 50
    _assert_same_run(sg, sr, gpu, ref)
    last = sg.history[-1]
    assert abs(last.tot - last.source_cum) <= 1e-12 * last.source_cum
    gpu.close()


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn", "tiny_latlon"])
def test_fast_dt_pipeline_matches_plain_loop(name):
    cfg = dataclasses.replace(syn.make_config(name), fast_dt=True)
    gpu, ref = _pair(cfg)
    sg = driver.run_pipelined(gpu, cfg)
    sr = driver.run(ref, cfg)
    assert sg.hour >= 1
    _assert_same_run(sg, sr, gpu, ref)
    gpu.close()


def test_c2_slab_default_build_across_a_met_load():
    cfg = dataclasses.replace(syn.make_config("C2"), fast_dt=True, fast_subgrid=True)
    cfg.ny, cfg.jvent = 24, 12
    gpu, ref = _pair(cfg)
    rng = np.random.default_rng(6)
    q = np.asfortranarray(rng.uniform(0.0, 100.0, (cfg.nx, cfg.ny, cfg.nz, cfg.ns)))
    out = []
    for m in (gpu, ref):
        m.set_interior(q)
        st = driver.new_state(cfg)
        st.time = 0.97  # the first steps cross 1 h: hour 1's met step loads inside the run
        for _ in range(4):
            driver.step(m, st)
        out.append(st)
    sg, sr = out
    assert sg.hour == 1
    _assert_same_run(sg, sr, gpu, ref)
    gpu.close()
