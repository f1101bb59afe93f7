"""The eruption schedule restated for the lag-one loop
(synthetic.scheduled_source_flux, the host mirror of the device's
a3g_add_source_scheduled): CheckEruptivePulses + TephraSourceNodes
(src/Source.f90:613-783) give the same SourceNodeFlux, bit for bit, as the
per-step source of the plain loop over a whole eruption, including the step
that ends it; and the reference's pulse quirks on several pulses."""
import numpy as np

from volcano_ash3d_b200 import synthetic as syn


def test_matches_plain_source_over_an_eruption():
    cfg = syn.make_config("tiny_proj")
    geo = syn.geometry(cfg)
    col = syn.suzuki_column(cfg)
    pulses = syn.eruption_pulses(cfg)
    state = [1, 1]
    t, dt = 0.0, 0.137
    seen_end = False
    while t < cfg.duration_h + 0.5:
        f = syn.scheduled_source_flux(cfg, pulses, col, geo["kappa"], state, t, dt)
        frac = syn.pulse_fraction(cfg, t, dt)
        if frac > 0.0:
            ref = syn.source_flux(cfg, col, geo["kappa"], frac)
            assert f is not None and np.array_equal(f, ref)
            seen_end = seen_end or frac < 1.0
        else:
            assert f is None
        t = t + dt
    assert seen_end


def test_pulse_quirks():
    cfg = syn.make_config("tiny_proj")
    geo = syn.geometry(cfg)
    col = np.concatenate([syn.suzuki_column(cfg)] * 2)  # NormSourceColumn(2, nz+1), pulse-major rows
    pulses = [(0.0, 1.0, 1.0e9), (1.05, 2.0, 2.0e9)]
    # a step that ends inside pulse 2 but starts after pulse 1: the loop exits
    # at pulse 2 before forming its fraction (src/Source.f90:646-651)
    state = [2, 2]
    assert syn.scheduled_source_flux(cfg, pulses, col.reshape(2, -1), geo["kappa"], state, 1.0, 0.1) is None
    assert state == [2, 2]
    # a step inside pulse 1 advances nothing
    state = [1, 1]
    f = syn.scheduled_source_flux(cfg, pulses, col.reshape(2, -1), geo["kappa"], state, 0.5, 0.1)
    assert f is not None and state == [1, 1] and f.sum() > 0.0
