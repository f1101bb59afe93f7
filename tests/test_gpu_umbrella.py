"""The umbrella-cloud source on the GPU (C-ABI) against the oracle, bit for
bit: the radial winds added on the umbrella levels (and the dt they set),
the 3x3 patch smoothing and insertion, on every advection variant, with CN
and explicit diffusion, and with terrain bound (vh is formed from the winds
that include the umbrella's)."""
import dataclasses

import numpy as np
import pytest

import ash3d_oracle as orc
from volcano_ash3d_b200 import driver
from volcano_ash3d_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _run(cfg, variant, steps=20):
    from volcano_ash3d_b200.model import Ash3dGPU
    geo = syn.geometry(cfg)
    gpu, ref = Ash3dGPU(cfg, geo=geo), orc.OracleModel(cfg, geo=geo)
    for d in range(3):
        gpu.set_variant(d, (4 if variant == 5 else variant) if d == 0 else (5 if variant == 5 else min(variant, 2)))
    sg = driver.run(gpu, cfg, max_steps=steps, geo=geo)
    sr = driver.run(ref, cfg, max_steps=steps, geo=geo)
    assert [h.dt for h in sg.history] == [h.dt for h in sr.history]
    bad = np.argwhere(gpu.interior() != ref.interior())
    assert bad.size == 0, f"{len(bad)} cells differ, first {bad[:3].tolist()}"
    og, orf = gpu.outflows(), ref.outflows()
    for key in og:
        assert np.array_equal(og[key], orf[key]), key
    for a, b in zip(sg.history, sr.history):
        np.testing.assert_allclose([a.aloft, a.dep, a.outflow], [b.aloft, b.dep, b.outflow], rtol=1e-13, atol=1e-30)
    gpu.close()
    return sg


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5])
def test_umbrella_run_bitwise(variant):
    sg = _run(syn.make_config("tiny_umbrella"), variant)
    h = sg.history[-1]
    np.testing.assert_allclose(h.tot, h.source_cum, rtol=1e-11)


def test_umbrella_explicit_diffusion_bitwise():
    _run(dataclasses.replace(syn.make_config("tiny_umbrella"), use_cn=False), 4)


@pytest.mark.parametrize("z", [1, 2])
def test_umbrella_with_terrain_bitwise(z):
    _run(dataclasses.replace(syn.make_config("tiny_umbrella"), zscaling_id=z, topo_km=1.5), 4)
