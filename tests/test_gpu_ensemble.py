"""Concurrent ensemble members (one context, stream and host thread each)
give the bits of their runs alone; the autotuner only changes speed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_concurrent_equals_sequential():
    from volcano_ash3d_b200 import ensemble as ens
    from volcano_ash3d_b200 import synthetic as syn
    cfgs = [syn.make_config(n) for n in ("tiny_proj", "tiny_cn", "tiny_latlon", "tiny_stretch",
                                         "tiny_periodic", "tiny_wide")]
    e = ens.Ensemble(cfgs, tune=True, keep_state=True)
    seq, _ = e.run_sequential(0.4)
    con, _ = e.run_concurrent(0.4)
    for a, b in zip(seq, con):
        assert a.steps == b.steps > 0
        assert np.array_equal(a.state, b.state), a.name
        assert a.final_tot == b.final_tot


def test_c3_members_shapes():
    from volcano_ash3d_b200 import ensemble as ens
    cfgs = ens.c3_members(64, seed=3)
    assert len(cfgs) == 64
    for c in cfgs:
        assert 80 <= c.nx <= 400 and 80 <= c.ny <= 400 and 30 <= c.nz <= 80 and 2 <= c.ns <= 10
        assert 5.0 <= c.plume_km <= 30.0 and 1.0 <= c.duration_h <= 12.0
