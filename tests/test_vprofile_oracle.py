"""Calc_vprofile (src/Output_Vars.f90:1308-1360) in the oracle against numpy
on the scratch level after a step: column totals against CLOUDCON_THRESH,
per-level grain sums in mg/m3, untouched columns below the threshold."""
import numpy as np

import ash3d_oracle as orc
from volcano_ash3d_b200 import driver
from volcano_ash3d_b200 import synthetic as syn


def test_vprofile_restated():
    cfg = syn.make_config("tiny_proj")
    m = orc.OracleModel(cfg, threads=1)
    driver.run(m, cfg, max_steps=6)
    pts = [(cfg.ivent, cfg.jvent), (1, 1)]
    out, w = m.vprofiles(pts, np.full((cfg.nz, 2), -1.0, order="F"))
    ts1 = m.concen[2:cfg.nx + 2, 2:cfg.ny + 2, 2:cfg.nz + 2, :, 1]
    assert np.array_equal(ts1, m.interior())  # after a step the scratch level equals the state
    col = ts1[cfg.ivent - 1, cfg.jvent - 1]
    assert w.tolist() == [1, 0]
    np.testing.assert_allclose(out[:, 0], col.sum(axis=1) * 1.0e6 / 1.0e9, rtol=1e-14)
    assert (out[:, 1] == -1.0).all()
