"""GPU (C-ABI) vs oracle parity on seeded inputs.

The library is compiled with --fmad=false and restates every expression in
the reference's operation order, so the sweeps are compared BIT-EXACTLY
(np.array_equal) against the oracle; only the mass totals, which the
reference sums sequentially and the GPU sums in double-double, are compared
with a relative tolerance of 1e-13.
"""
import numpy as np
import pytest

from gpu_common import pair, prime, random_state
from volcano_ash3d_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

CONFIGS = ["tiny_proj", "tiny_cn", "tiny_latlon", "tiny_periodic", "tiny_subgrid", "tiny_wide",
           "tiny_tall", "tiny_deep", "tiny_stretch"]
OPS = ["advect_x", "advect_y", "AdvectVert", "DiffuseHorz_even", "DiffuseHorz_odd", "DiffuseVert"]


def _apply(m, op):
    if op == "advect_x":
        m.advect_x()
    elif op == "advect_y":
        m.advect_y()
    elif op == "AdvectVert":
        m.AdvectVert()
    elif op == "DiffuseHorz_even":
        m.DiffuseHorz(2)
    elif op == "DiffuseHorz_odd":
        m.DiffuseHorz(1)
    elif op == "DiffuseVert":
        m.DiffuseVert()


def _assert_outflows_equal(gpu, ref):
    og, orf = gpu.outflows(), ref.outflows()
    for key in og:
        assert np.array_equal(og[key], orf[key]), key


ADVECTION = ("advect_x", "advect_y", "AdvectVert")


def _variants(op):
    # advection: march / block-4 / block-8 / x warp-tiled / x warp-row / y, z
    # column march; diffusion: the CN x solve warp-tiled / one thread per line
    # and the y, z solves one / two / four grains per thread / TMA tiles
    return (0, 1, 2, 3, 4, 5, 6) if op in ADVECTION else (0, 1, 2, 3)


def _adv_variant(d, variant):
    """The variant a direction takes for a parametrised advection variant:
    3 and 4 exist for x only, 5 and 6 (the column marches, from global memory
    and from TMA chunks) for y and z only; 6 takes x's warp rows fed by TMA
    (x variant 5)."""
    if d == 0:
        return {5: 4, 6: 5}.get(variant, variant)
    return variant if variant in (5, 6) else min(variant, 2)


def _set_variant(gpu, op, variant):
    if op in ADVECTION:
        for d in range(3):
            gpu.set_variant(d, _adv_variant(d, variant))
    else:
        gpu.set_variant(3, variant % 3)
        gpu.set_variant(4, variant)


@pytest.mark.parametrize("name", CONFIGS)
@pytest.mark.parametrize("op,variant", [(o, v) for o in OPS for v in _variants(o)])
def test_single_operator_bitwise(name, op, variant):
    cfg, gpu, ref = pair(name)
    _set_variant(gpu, op, variant)
    box = None
    if cfg.fast_subgrid:  # a strict sub-box: cells outside it must come back as zero
        box = (4, cfg.nx - 5, 3, cfg.ny - 4, 2, cfg.nz - 3)
    prime(cfg, gpu, ref, seed=7, box=box)
    _apply(gpu, op)
    _apply(ref, op)
    qg, qr = gpu.interior(), ref.interior()
    bad = np.argwhere(qg != qr)
    assert bad.size == 0, f"{len(bad)} cells differ, first {bad[:3].tolist()}"
    _assert_outflows_equal(gpu, ref)
    gpu.close()


@pytest.mark.parametrize("name", CONFIGS)
def test_adjust_dt_bitwise(name):
    cfg, gpu, ref = pair(name)
    dt = prime(cfg, gpu, ref, seed=3)
    assert dt > 0
    # clipping to the next write time and to the end of the run, Adjust_dt.f90:325-332
    assert gpu.Adjust_DT(0.5, 0.5 + 0.3 * dt, 10.0) == ref.Adjust_DT(0.5, 0.5 + 0.3 * dt, 10.0)
    assert gpu.Adjust_DT(0.5, 10.0, 0.5 + 0.25 * dt) == ref.Adjust_DT(0.5, 10.0, 0.5 + 0.25 * dt)
    gpu.close()


@pytest.mark.parametrize("name", CONFIGS)
def test_minmax_index(name):
    cfg, gpu, ref = pair(name)
    q = random_state(cfg, 5)
    q[:3] = 0.0
    q[-4:] = 0.0
    q[:, :2] = 0.0
    q[:, :, -3:] = 0.0
    gpu.set_interior(q)
    ref.set_interior(q)
    assert gpu.get_minmax_index() == ref.get_minmax_index()
    gpu.close()


@pytest.mark.parametrize("name", CONFIGS)
def test_timestep_totals(name):
    cfg, gpu, ref = pair(name)
    prime(cfg, gpu, ref, seed=9)
    for m in (gpu, ref):
        m.advect_x(); m.advect_y(); m.AdvectVert()
    vg, mg = gpu.TimeStepTotals()
    vr, mr = ref.TimeStepTotals()
    np.testing.assert_allclose(vg, vr, rtol=1e-13, atol=0)
    np.testing.assert_allclose(mg, mr, rtol=1e-13, atol=0)
    gpu.close()


@pytest.mark.parametrize("name", CONFIGS)
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6])
def test_run_bitwise(name, variant):
    from volcano_ash3d_b200 import driver
    cfg, gpu, ref = pair(name)
    for d in range(3):
        gpu.set_variant(d, _adv_variant(d, variant))
    gpu.set_variant(3, variant % 3)
    gpu.set_variant(4, variant if variant <= 3 else 3 - variant % 2 if variant < 6 else 1)
    sg = driver.run(gpu, cfg, max_steps=16)
    sr = driver.run(ref, cfg, max_steps=16)
    assert [h.dt for h in sg.history] == [h.dt for h in sr.history]
    assert np.array_equal(gpu.interior(), ref.interior())
    _assert_outflows_equal(gpu, ref)
    for a, b in zip(sg.history, sr.history):
        np.testing.assert_allclose([a.aloft, a.dep, a.outflow, a.tot],
                                   [b.aloft, b.dep, b.outflow, b.tot], rtol=1e-13, atol=1e-30)
    gpu.close()


def test_error_codes():
    from volcano_ash3d_b200 import A3GError
    cfg, gpu, ref = pair("tiny_proj")
    with pytest.raises(A3GError) as e:
        gpu.Set_BC(3)
    assert e.value.code == 4  # "ERROR BC code not recognized", Set_BC.f90:119-123
    with pytest.raises(A3GError):
        gpu.set_subgrid((0, 5, 1, 5, 1, 5))
    gpu.close()


def test_c1_full_run_bitwise():
    """The whole 6-hour projected workload (100x100x40, 4 grains, explicit
    diffusion, Suzuki source) against the oracle, every step."""
    from volcano_ash3d_b200 import driver
    cfg, gpu, ref = pair("C1")
    sg = driver.run(gpu, cfg)
    sr = driver.run(ref, cfg)
    assert len(sg.history) == len(sr.history) > 50
    assert [h.dt for h in sg.history] == [h.dt for h in sr.history]
    assert np.array_equal(gpu.interior(), ref.interior())
    _assert_outflows_equal(gpu, ref)
    last_g, last_r = sg.history[-1], sr.history[-1]
    np.testing.assert_allclose([last_g.aloft, last_g.dep, last_g.outflow, last_g.tot],
                               [last_r.aloft, last_r.dep, last_r.outflow, last_r.tot], rtol=1e-13)
    # mass conservation of the run itself (MassConsErr, src/Ash3d.F90:611-617)
    assert abs(last_g.tot - last_g.source_cum) <= 1e-12 * last_g.source_cum
    gpu.close()


def test_exact_division_matches_ieee():
    """The sweeps' division (exact_div.cuh) returns the IEEE quotient bit for
    bit on 2^26 seeded operand pairs of mixed magnitude, sign and structure."""
    import ctypes as C
    from volcano_ash3d_b200 import _lib
    lib = _lib.load()
    bad = C.c_uint64(99)
    _lib.check(lib.a3g_selftest_div(0, 1 << 26, 12345, C.byref(bad)))
    assert bad.value == 0


@pytest.mark.parametrize("name", ["tiny_cn", "tiny_latlon", "tiny_subgrid"])
def test_cn_tables_follow_dt_and_box(name):
    """The CN factor tables are kept between steps while dt, the box, the
    geometry and the diffusivity stay the same; changing dt back and forth,
    and the box, must rebuild them (bitwise against the oracle)."""
    cfg, gpu, ref = pair(name)
    dt0 = prime(cfg, gpu, ref, seed=31)
    boxes = [(1, cfg.nx, 1, cfg.ny, 1, cfg.nz), (3, cfg.nx - 2, 2, cfg.ny - 3, 2, cfg.nz - 1)]
    for n, (dt, box) in enumerate([(dt0, 0), (dt0, 0), (0.5 * dt0, 0), (dt0, 0), (dt0, 1), (dt0, 1), (dt0, 0)]):
        for m in (gpu, ref):
            m.set_dt(dt)
            m.set_subgrid(boxes[box])
            m.Set_BC(2)
            m.DiffuseHorz(n)
            m.DiffuseVert()
        bad = np.argwhere(gpu.interior() != ref.interior())
        assert bad.size == 0, (n, f"{len(bad)} cells differ, first {bad[:3].tolist()}")
    gpu.close()


def test_totals_follow_the_state():
    """TimeStepTotals after a CN z solve, after a new state and after a
    source insertion each describe the state of that moment (totals
    against the oracle at 1e-13)."""
    cfg, gpu, ref = pair("tiny_cn")
    prime(cfg, gpu, ref, seed=41)
    for m in (gpu, ref):
        m.Set_BC(2)
        m.DiffuseHorz(1)
        m.DiffuseVert()

    def same_totals():
        vg, mg = gpu.TimeStepTotals()
        vr, mr = ref.TimeStepTotals()
        np.testing.assert_allclose(vg, vr, rtol=1e-13, atol=0)
        np.testing.assert_allclose(mg, mr, rtol=1e-13, atol=0)

    same_totals()
    q = random_state(cfg, 77)
    for m in (gpu, ref):
        m.set_interior(q)
    same_totals()
    for m in (gpu, ref):
        m.Set_BC(2)
        m.DiffuseVert()
        m.add_source(np.full((cfg.nz + 1, cfg.ns), 3.0e4, order="F"), 0.1)
    same_totals()
    gpu.close()


# Sub-boxes with odd and even first cells along every direction, on lines of
# several TMA tiles or chunks in each direction (x: 100 cells = 4 CN x tiles,
# whose loads start on the even cell at or before the tile; y: 70 cells = 5
# CN y chunks; z: 40-cell columns), so that the default kernels' staged tiles
# meet every start parity and a ragged last tile.
TILE_BOXES = [(5, 93, 4, 66, 3, 37), (6, 96, 3, 61, 2, 38), (1, 100, 2, 70, 1, 39)]


@pytest.mark.parametrize("box", TILE_BOXES)
@pytest.mark.parametrize("op", OPS)
def test_default_kernels_on_sub_boxes_bitwise(op, box):
    cfg = syn.Config("tile_boxes", 100, 70, 40, 2, dx=4.0, dy=5.0, dz=0.5, ivent=50, jvent=35,
                     fall_mps=(0.2, 1.5), bin_mass=(0.5, 0.5), plume_km=8.0, volume_km3=1.0e-3,
                     duration_h=1.0, use_cn=True, sim_hours=1.0, winds="random", seed=23,
                     fast_subgrid=True)
    cfg, gpu, ref = pair(cfg)
    prime(cfg, gpu, ref, seed=29, box=box)
    _apply(gpu, op)
    _apply(ref, op)
    qg, qr = gpu.interior(), ref.interior()
    bad = np.argwhere(qg != qr)
    assert bad.size == 0, f"{len(bad)} cells differ, first {bad[:3].tolist()}"
    _assert_outflows_equal(gpu, ref)
    gpu.close()
