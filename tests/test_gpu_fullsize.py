"""Full-size checks that do not need the oracle at full size.

* C2 at full size (720x360x60, 10 grains, CN, lon/lat): from a clean
  atmosphere with the Suzuki source, the airborne + deposited + outflowed
  mass equals the mass inserted to 1e-12 (MassConsErr of src/Ash3d.F90:
  611-617), and no cell goes negative beyond round-off.
* A C2 slab (the full 720-cell rows, 24 latitudes) against the oracle, bit
  for bit, over 3 steps from a filled state.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_c2_full_size_mass_conservation():
    from volcano_ash3d_b200 import driver
    from volcano_ash3d_b200 import synthetic as syn
    from volcano_ash3d_b200.model import Ash3dGPU
    cfg = syn.make_config("C2")
    gpu = Ash3dGPU(cfg)
    gpu.set_interior(np.zeros((cfg.nx, cfg.ny, cfg.nz, cfg.ns), order="F"))
    st = driver.run(gpu, cfg, max_steps=8)
    last = st.history[-1]
    assert last.source_cum > 0
    assert abs(last.tot - last.source_cum) <= 1e-12 * last.source_cum
    q = gpu.interior()
    assert q.min() >= -1e-12 * q.max()
    gpu.close()


def test_c2_slab_bitwise():
    import ash3d_oracle as orc
    from volcano_ash3d_b200 import driver
    from volcano_ash3d_b200 import synthetic as syn
    from volcano_ash3d_b200.model import Ash3dGPU
    cfg = syn.make_config("C2")
    cfg.ny, cfg.jvent = 24, 12
    geo = syn.geometry(cfg)
    gpu, ref = Ash3dGPU(cfg, geo=geo), orc.OracleModel(cfg, geo=geo)
    rng = np.random.default_rng(5)
    q = np.asfortranarray(rng.uniform(0.0, 100.0, (cfg.nx, cfg.ny, cfg.nz, cfg.ns)))
    for m in (gpu, ref):
        m.set_interior(q)
    sg = driver.run(gpu, cfg, max_steps=3)
    sr = driver.run(ref, cfg, max_steps=3)
    assert [h.dt for h in sg.history] == [h.dt for h in sr.history]
    assert np.array_equal(gpu.interior(), ref.interior())
    gpu.close()
