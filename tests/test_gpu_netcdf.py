"""The NetCDF output arrays and the restart load on the GPU
(a3g_output_ashcon / a3g_restart_load) against the oracle, bit for bit:
ashcon and depocon after steps that leave settling and deposit, through host
and device pointers and with either array left out; a run restarted from the
arrays continues exactly like the oracle restarted from them."""
import copy

import numpy as np
import pytest

import ash3d_oracle as orc
from gpu_common import pair
from volcano_ash3d_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _same_f32(a, b):
    # numerically equal (an exact zero's sign is the one sanctioned difference)
    assert a.dtype == np.float32 and b.dtype == np.float32 and a.shape == b.shape
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn", "tiny_latlon", "tiny_subgrid", "tiny_stretch"])
def test_output_arrays_match_oracle(name):
    from volcano_ash3d_b200 import driver
    cfg, gpu, ref = pair(name)
    sg, sr = driver.new_state(cfg), driver.new_state(cfg)
    for _ in range(10):
        driver.step(gpu, sg)
        driver.step(ref, sr)
    ag, dg = gpu.output_ashcon()
    ar, dr = ref.output_ashcon()
    _same_f32(ag, ar)
    _same_f32(dg, dr)
    assert ag.max() > 0.0
    gpu.close()


def test_device_pointers_and_null_arrays():
    import torch
    from volcano_ash3d_b200 import driver
    from volcano_ash3d_b200._lib import check
    cfg, gpu, ref = pair("tiny_proj")
    st = driver.new_state(cfg)
    for _ in range(12):
        driver.step(gpu, st)
    ah, dh = gpu.output_ashcon()
    assert dh.max() > 0.0
    nx, ny, nz, ns = cfg.nx, cfg.ny, cfg.nz, cfg.ns
    # device tensors laid out like the Fortran arrays: x fastest
    ad = torch.full((ns, nz, ny, nx), -1.0, dtype=torch.float32, device="cuda")
    dd = torch.full((ns, ny, nx), -1.0, dtype=torch.float32, device="cuda")
    check(gpu.lib.a3g_output_ashcon(gpu.ctx, ad.data_ptr(), dd.data_ptr()))
    assert np.array_equal(ad.cpu().numpy().transpose(3, 2, 1, 0), ah)
    assert np.array_equal(dd.cpu().numpy().transpose(2, 1, 0), dh)
    # either array alone
    a1 = np.full_like(ah, -1.0)
    check(gpu.lib.a3g_output_ashcon(gpu.ctx, a1.ctypes.data, None))
    assert np.array_equal(a1, ah)
    d1 = np.full_like(dh, -1.0)
    check(gpu.lib.a3g_output_ashcon(gpu.ctx, None, d1.ctypes.data))
    assert np.array_equal(d1, dh)
    # restart from device memory, then from host memory: the same state
    gpu2 = pair("tiny_proj")[1]
    check(gpu2.lib.a3g_restart_load(gpu2.ctx, ad.data_ptr(), dd.data_ptr()))
    assert np.array_equal(gpu2.interior(), ah.astype(np.float64))
    assert np.array_equal(gpu2.outflows()["xy1"], dh.astype(np.float64))
    gpu3 = pair("tiny_proj")[1]
    gpu3.restart_load(ah, dh)
    assert np.array_equal(gpu3.interior(), gpu2.interior())
    assert np.array_equal(gpu3.outflows()["deposit"], dh.astype(np.float64))
    for m in (gpu, gpu2, gpu3):
        m.close()


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn", "tiny_latlon"])
def test_restarted_run_matches_oracle(name):
    from volcano_ash3d_b200 import driver
    cfg, gpu, ref = pair(name)
    writer = orc.OracleModel(cfg, geo=syn.geometry(cfg))  # wrote the arrays; ref starts fresh like gpu
    st = driver.new_state(cfg)
    for _ in range(8):
        driver.step(writer, st)
    ash, dep = writer.output_ashcon()
    for m in (gpu, ref):
        m.restart_load(ash, dep)
    sg, sr = copy.deepcopy(st), copy.deepcopy(st)
    sg.hour = sr.hour = -1  # the restarted models upload their met pair on the first step
    for _ in range(6):
        rg = driver.step(gpu, sg)
        rr = driver.step(ref, sr)
        assert rg.dt == rr.dt
    assert np.array_equal(gpu.interior(), ref.interior())
    og, orf = gpu.outflows(), ref.outflows()
    for key in ("xy1", "xy2", "yz1", "yz2", "xz1", "xz2"):
        assert np.array_equal(og[key], orf[key]), key
    ag, dg = gpu.output_ashcon()
    ar, dr = ref.output_ashcon()
    _same_f32(ag, ar)
    _same_f32(dg, dr)
    gpu.close()
