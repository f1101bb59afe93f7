"""Output products of Gen_Output_Vars on the GPU (a3g_output_vars) against
the oracle's restatement, bit for bit: cloud load, cloud top and bottom,
peak concentration, the masks, deposit thickness, the arrival marks and the
areas, after steps that leave settling, deposit and (FAST_SUBGRID) a strict
subgrid box."""
import numpy as np
import pytest

from gpu_common import pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn", "tiny_latlon", "tiny_subgrid", "tiny_stretch"])
def test_output_vars_match_oracle(name):
    from volcano_ash3d_b200 import driver
    cfg, gpu, ref = pair(name)
    sg, sr = driver.new_state(cfg), driver.new_state(cfg)
    for m in (gpu, ref):
        m.output_reset()
    # low thresholds so that masks, heights and deposit are non-trivial on a tiny run
    thr = dict(cloudcon_thresh=1.0e-6, cloudload_thresh=1.0e-4, depo_thresh=1.0e-9)
    gpu.set_output_params(**thr)
    for _ in range(12):
        driver.step(gpu, sg)
        driver.step(ref, sr)
        og = gpu.output_vars(sg.time)
        orf = ref.output_vars(sr.time, **thr)
        for key in ("cloud_load", "max_height", "min_height", "max_conc", "mask_cloud", "dep_thick",
                    "mask_dep", "cloud_arrival", "dep_arrival", "cloud_load_area"):
            assert np.array_equal(og[key], orf[key]), key
        assert og["cloud_area"] == orf["cloud_area"] and og["dep_area"] == orf["dep_area"]
    assert og["mask_cloud"].any() and og["mask_dep"].any()
    gpu.close()


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_latlon", "tiny_umbrella"])
def test_vprofiles_match_oracle(name):
    """Calc_vprofile at the vent, near it, and at a corner far from the cloud
    (below CLOUDCON_THRESH: its profile keeps the previous values)."""
    from volcano_ash3d_b200 import driver
    cfg, gpu, ref = pair(name)
    pts = [(cfg.ivent, cfg.jvent), (cfg.ivent + 1, cfg.jvent - 1), (1, cfg.ny)]
    sg, sr = driver.new_state(cfg), driver.new_state(cfg)
    pg = np.full((cfg.nz, len(pts)), -7.0, order="F")
    pr = pg.copy(order="F")
    gpu.set_output_params(cloudcon_thresh=1.0e-3)
    for _ in range(6):
        driver.step(gpu, sg)
        driver.step(ref, sr)
        pg, wg = gpu.vprofiles(pts, pg)
        pr, wr = ref.vprofiles(pts, pr, thresh=1.0e-3)
        assert np.array_equal(wg, wr)
        assert np.array_equal(pg, pr)
    assert wg[0] == 1 and pg[:, 0].max() > 0.0
    gpu.close()
