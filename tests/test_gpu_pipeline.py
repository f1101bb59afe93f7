"""The lag-one host loop (driver.Pipeline: dt kept on the device and read
back late, the source scheduled on the device, the totals collected a step
later) against the oracle's plain loop: the same dt sequence, the state and
the outflow accumulators bit for bit, the totals to 1e-13 and the erupted
volume exactly, through the end of the eruption."""
import dataclasses

import numpy as np
import pytest

import ash3d_oracle as orc
from volcano_ash3d_b200 import driver
from volcano_ash3d_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _cfg(name, **over):
    return dataclasses.replace(syn.make_config(name), **over)


@pytest.mark.parametrize("cfg", [
    _cfg("tiny_proj"), _cfg("tiny_cn", duration_h=0.3), _cfg("tiny_latlon"), _cfg("tiny_periodic"),
    _cfg("tiny_tall"), _cfg("tiny_proj", zscaling_id=2, topo_km=1.5)], ids=lambda c: f"{c.name}-{c.zscaling_id}")
def test_pipeline_matches_plain_loop(cfg):
    from volcano_ash3d_b200.model import Ash3dGPU
    geo = syn.geometry(cfg)
    gpu, ref = Ash3dGPU(cfg, geo=geo), orc.OracleModel(cfg, geo=geo)
    sg = driver.run_pipelined(gpu, cfg, max_steps=24, geo=geo)
    sr = driver.run(ref, cfg, max_steps=24, geo=geo)
    assert [h.dt for h in sg.history] == [h.dt for h in sr.history]
    assert np.array_equal(gpu.interior(), ref.interior())
    og, orf = gpu.outflows(), ref.outflows()
    for key in og:
        assert np.array_equal(og[key], orf[key]), key
    for a, b in zip(sg.history, sr.history):
        assert a.source_cum == b.source_cum
        np.testing.assert_allclose([a.aloft, a.dep, a.outflow], [b.aloft, b.dep, b.outflow], rtol=1e-13, atol=1e-30)
    gpu.close()


def test_pipeline_rejects_subgrid_and_umbrella():
    from volcano_ash3d_b200.model import Ash3dGPU
    cfg = syn.make_config("tiny_subgrid")
    gpu = Ash3dGPU(cfg)
    with pytest.raises(ValueError):
        driver.Pipeline(gpu, cfg)
    gpu.close()
