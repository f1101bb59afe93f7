"""The oracle's discrete adjoint (CPU): dot-product tests of every sweep.

Each sweep is piecewise linear in the concentration, so with the limiter
branches fixed by the state it is a linear map J.  For a state with no
limiter branch near a switch, the central difference
(F(c + e*d) - F(c - e*d)) / (2e) equals J d up to rounding, and the
transpose must satisfy <J d, lam> = <d, J^T lam>.  The state is strictly
positive and the perturbation relative (d = c * N(0,1)), so the tiny-value
branches (|dq| <= EPS_THRESH) stay where they are.  A limiter kink within
e of the state still bends the difference quotient, and cancellation in
F(c + e*d) - F(c - e*d) leaves noise near 1e-8, so the advection sweeps are
held to 1e-6 relative with e = 1e-8; the diffusion sweeps, linear outright,
to 1e-8 with e = 1e-6.
"""
import numpy as np
import pytest

import ash3d_oracle as orc
from volcano_ash3d_b200 import synthetic as syn

CONFIGS = ["tiny_proj", "tiny_cn", "tiny_latlon", "tiny_periodic", "tiny_stretch"]
OPS = ["advect_x", "advect_y", "AdvectVert", "DiffuseHorz_even", "DiffuseHorz_odd", "DiffuseVert"]
LIMITERS = ["superbee", "minmod", "mc", "fromm", "laxwen", "bw", "none"]


def smooth_state(cfg, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz, ns = cfg.nx, cfg.ny, cfg.nz, cfg.ns
    x = np.linspace(-1, 1, nx)[:, None, None, None]
    y = np.linspace(-1, 1, ny)[None, :, None, None]
    z = np.linspace(0, 1, nz)[None, None, :, None]
    g = np.arange(ns)[None, None, None, :]
    q = 1.0e4 * np.exp(-((x - 0.1 * g) ** 2 + y ** 2) * 6.0 - (z - 0.4) ** 2 * 8.0) + 1.0
    return np.asfortranarray(q * rng.uniform(0.5, 1.5, q.shape))


def winds(cfg, seed):
    rng = np.random.default_rng(seed)
    shp = (cfg.nx + 4, cfg.ny + 4, cfg.nz + 4)
    return tuple(np.asfortranarray(v) for v in (60.0 * rng.standard_normal(shp) + 20.0,
                                                50.0 * rng.standard_normal(shp) - 10.0,
                                                5.0 * rng.standard_normal(shp)))


def model(name, limiter=None):
    cfg = syn.make_config(name)
    m = orc.OracleModel(cfg, limiter=limiter, threads=1)
    m.set_winds(*winds(cfg, 5))
    m.Adjust_DT(0.0, 1.0e9, 1.0e9)
    return cfg, m


def forward(m, op, c):
    m.set_interior(c)
    m.zero_outflows()
    {"advect_x": m.advect_x, "advect_y": m.advect_y, "AdvectVert": m.AdvectVert,
     "DiffuseHorz_even": lambda: m.DiffuseHorz(2), "DiffuseHorz_odd": lambda: m.DiffuseHorz(1),
     "DiffuseVert": m.DiffuseVert}[op]()
    return m.interior(), m.outflows()["deposit"]


def adjoint(m, op, c, lam, lam_dep):
    m.set_interior(c)
    if op == "advect_x":
        return m.adj_advect_x(lam)
    if op == "advect_y":
        return m.adj_advect_y(lam)
    if op == "AdvectVert":
        return m.adj_advect_z(lam, lam_dep)
    if op == "DiffuseHorz_even":
        return m.adj_diffuse_horz(lam, 2)
    if op == "DiffuseHorz_odd":
        return m.adj_diffuse_horz(lam, 1)
    return m.adj_diffuse_vert(lam)


def dot_test(m, cfg, op, seed, e):
    rng = np.random.default_rng(seed)
    c = smooth_state(cfg, seed)
    d = np.asfortranarray(c * rng.standard_normal(c.shape))
    lam = np.asfortranarray(rng.standard_normal(c.shape))
    lam_dep = np.asfortranarray(rng.standard_normal((cfg.nx, cfg.ny, cfg.ns)))
    fp, dp = forward(m, op, c + e * d)
    fm, dm = forward(m, op, c - e * d)
    jd, jd_dep = (fp - fm) / (2 * e), (dp - dm) / (2 * e)
    lhs = np.sum(jd * lam) + np.sum(jd_dep * lam_dep)
    rhs = np.sum(d * adjoint(m, op, c, lam, lam_dep))
    return lhs, rhs


@pytest.mark.parametrize("name", CONFIGS)
@pytest.mark.parametrize("op", OPS)
def test_sweep_adjoint_dot_product(name, op):
    cfg, m = model(name)
    advect = op in ("advect_x", "advect_y", "AdvectVert")
    lhs, rhs = dot_test(m, cfg, op, seed=21, e=1e-8 if advect else 1e-6)
    tol = 1e-6 if advect else 1e-8
    assert abs(lhs - rhs) <= tol * (abs(lhs) + abs(rhs)), (lhs, rhs)


@pytest.mark.parametrize("limiter", LIMITERS)
@pytest.mark.parametrize("op", ["advect_x", "AdvectVert"])
def test_limiter_adjoint_dot_product(limiter, op):
    cfg, m = model("tiny_latlon", limiter)
    lhs, rhs = dot_test(m, cfg, op, seed=33, e=1e-8)
    assert abs(lhs - rhs) <= 1e-6 * (abs(lhs) + abs(rhs)), (lhs, rhs)


@pytest.mark.parametrize("limiter", ["superbee", "minmod", "mc", "fromm"])
def test_limiter_coefficients(limiter):
    """a*dq + b*dqu reproduces the forward limited slope on every branch."""
    lib = orc.load()
    import ctypes as C
    from volcano_ash3d_b200._lib import LIMITERS
    lib.orc_lim_coef.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lid = LIMITERS[limiter]
    rng = np.random.default_rng(3)
    for _ in range(2000):
        dq, dqu = rng.standard_normal(2) * 10.0 ** rng.uniform(-3, 3, 2)
        a, b = C.c_double(), C.c_double()
        lib.orc_lim_coef(lid, dq, dqu, 1e-10, C.byref(a), C.byref(b))
        clamp = abs(dqu) > 3 * abs(dq)
        th = np.copysign(3.0, dqu * dq) if clamp else dqu / dq
        phi = {"superbee": max(max(0, min(1, 2 * th)), min(2, th)),
               "minmod": max(0, min(1, th)),
               "mc": max(0, min(min((1 + th) / 2, 2), 2 * th)),
               "fromm": 0.5 * (1 + th)}[limiter]
        np.testing.assert_allclose(a.value * dq + b.value * (0.0 if clamp else dqu), dq * phi,
                                   rtol=1e-12, atol=1e-300)


def _step_map(m, cfg, itime, c):
    """One transport step (no source, no prologue) from state c."""
    m.set_interior(c)
    m.zero_outflows()
    m.Set_BC(1)
    m.AdvectHorz(itime)
    m.AdvectVert()
    if cfg.use_diffusion:
        m.Set_BC(2)
        m.DiffuseHorz(itime)
        m.DiffuseVert()
    return m.interior(), m.outflows()["deposit"]


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn", "tiny_latlon", "tiny_periodic"])
@pytest.mark.parametrize("itime", [1, 2])
def test_step_adjoint_dot_product(name, itime):
    """adj_step is the transpose of the whole step (both toggle parities),
    deposit adjoint included."""
    cfg, m = model(name)
    rng = np.random.default_rng(40 + itime)
    c = smooth_state(cfg, 8)
    d = np.asfortranarray(c * rng.standard_normal(c.shape))
    lam = np.asfortranarray(rng.standard_normal(c.shape))
    lam_dep = np.asfortranarray(rng.standard_normal((cfg.nx, cfg.ny, cfg.ns)))
    e = 1e-8
    fp, dp = _step_map(m, cfg, itime, c + e * d)
    fm, dm = _step_map(m, cfg, itime, c - e * d)
    lhs = np.sum((fp - fm) / (2 * e) * lam) + np.sum((dp - dm) / (2 * e) * lam_dep)
    m.set_interior(c)
    m.set_lambda(lam)
    m.set_lambda_dep(lam_dep)
    m.adj_step(itime)
    rhs = np.sum(d * m.get_lambda())
    assert abs(lhs - rhs) <= 1e-6 * (abs(lhs) + abs(rhs)), (lhs, rhs)


def test_source_gradient_matches_finite_differences():
    """dJ/dp of the source inversion (checkpointed reverse sweep, K=4 on a
    39-step run) against central differences of J on 8 seeded components of
    the active source (step 1e-4 of the component)."""
    from volcano_ash3d_b200 import adjoint as adj
    cfg = syn.make_config("tiny_proj")
    inv = adj.SourceInversion(cfg, hours=2)
    m = orc.OracleModel(cfg, threads=1)
    _, loads, logs, _ = inv.forward(m, inv.prior(seed=1, lognormal_sigma=0.5))
    obs = {h: loads[h] * (1 + 0.05 * np.random.default_rng(h).standard_normal(loads[h].shape))
           for h in loads}
    p = inv.prior()
    J, g = inv.gradient(m, p, obs, K=4)
    assert J > 0 and np.all(np.isfinite(g))
    rng = np.random.default_rng(5)
    active = np.argwhere(p > 0)  # at a zero source, +-h crosses the limiter kinks at c = 0
    for _ in range(8):
        i = tuple(int(v) for v in active[rng.integers(0, len(active))])
        h = 1e-4 * p[i]
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (inv.forward(m, pp, obs)[0] - inv.forward(m, pm, obs)[0]) / (2 * h)
        assert abs(g[i] - fd) <= 1e-4 * abs(fd), (i, g[i], fd)


@pytest.mark.parametrize("fast_dt", [False, True])
def test_deposit_misfit_gradient_matches_finite_differences(fast_dt):
    """dJ/dp with the deposit term (the thickness of the deposit laid down
    after hour 1, AshThicknessCalculator unmasked) and the column loads of
    hour 1 on, with FAST_DT off and on, against central differences of J."""
    from volcano_ash3d_b200 import adjoint as adj
    cfg = syn.make_config("tiny_proj")
    inv = adj.SourceInversion(cfg, hours=2)
    m = orc.OracleModel(cfg, threads=1)
    zero_dep = np.zeros((cfg.nx, cfg.ny))
    _, loads, _, _ = inv.forward(m, inv.prior(seed=2, lognormal_sigma=0.5), fast_dt=fast_dt, obs_dep=zero_dep,
                                 dep_from=1)
    rng = np.random.default_rng(9)
    obs = {h: loads[h] * (1 + 0.05 * rng.standard_normal(loads[h].shape)) for h in loads if h != "dep"}
    obs_dep = loads["dep"] * (1 + 0.05 * rng.standard_normal(loads["dep"].shape))
    assert np.abs(loads["dep"]).max() > 0.0
    p = inv.prior()
    kw = dict(fast_dt=fast_dt, obs_dep=obs_dep, dep_from=1, load_from=1)
    J, g = inv.gradient(m, p, obs, K=5, **kw)
    assert J > 0 and np.all(np.isfinite(g))
    active = np.argwhere(p > 0)
    for _ in range(6):
        i = tuple(int(v) for v in active[rng.integers(0, len(active))])
        h = 1e-4 * p[i]
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (inv.forward(m, pp, obs, **kw)[0] - inv.forward(m, pm, obs, **kw)[0]) / (2 * h)
        assert abs(g[i] - fd) <= 1e-4 * abs(fd), (i, g[i], fd)
