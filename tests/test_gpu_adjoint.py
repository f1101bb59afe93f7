"""GPU discrete adjoint (C-ABI a3g_adj_*) against the oracle's adjoint.

The two are transposes of the same linearised sweeps with the limiter
branches fixed by the same state (identical forward arithmetic, so identical
branch choices); they sum their terms in different orders, so they are
compared to 1e-12 of the field's largest value.  The column load (H) is
compared bit for bit.  The checkpointed source gradient of the GPU is
compared with the oracle's (1e-10) and with central differences of the GPU
forward run.
"""
import numpy as np
import pytest

from gpu_common import pair, random_state, random_winds

pytestmark = pytest.mark.gpu

CONFIGS = ["tiny_proj", "tiny_cn", "tiny_latlon", "tiny_periodic", "tiny_stretch", "tiny_wide"]
OPS = ["advect_x", "advect_y", "AdvectVert", "DiffuseHorz_even", "DiffuseHorz_odd", "DiffuseVert"]


def _prime(cfg, gpu, ref, seed):
    q = random_state(cfg, seed)
    vx, vy, vz = random_winds(cfg, seed + 1)
    for m in (gpu, ref):
        m.set_interior(q)
        m.set_winds(vx, vy, vz)
    assert gpu.Adjust_DT(0.0, 1e9, 1e9) == ref.Adjust_DT(0.0, 1e9, 1e9)
    return q


def _adj(m, op, lam, lam_dep):
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


def _close(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max()
    assert err <= 1e-12 * scale, f"max |diff| {err:.3e} vs scale {scale:.3e}"


@pytest.mark.parametrize("name", CONFIGS)
@pytest.mark.parametrize("op", OPS)
def test_adjoint_sweep_matches_oracle(name, op):
    cfg, gpu, ref = pair(name)
    _prime(cfg, gpu, ref, seed=17)
    rng = np.random.default_rng(3)
    lam = np.asfortranarray(rng.standard_normal((cfg.nx, cfg.ny, cfg.nz, cfg.ns)))
    lam_dep = np.asfortranarray(rng.standard_normal((cfg.nx, cfg.ny, cfg.ns)))
    _close(_adj(gpu, op, lam, lam_dep), _adj(ref, op, lam, lam_dep))
    gpu.close()


@pytest.mark.parametrize("limiter", ["minmod", "mc", "fromm", "laxwen", "bw", "none"])
def test_adjoint_limiters_match_oracle(limiter):
    from volcano_ash3d_b200 import synthetic as syn
    cfg = syn.make_config("tiny_latlon")
    cfg.limiter = limiter
    cfg, gpu, ref = pair(cfg)
    _prime(cfg, gpu, ref, seed=19)
    rng = np.random.default_rng(4)
    lam = np.asfortranarray(rng.standard_normal((cfg.nx, cfg.ny, cfg.nz, cfg.ns)))
    for op in ("advect_x", "advect_y", "AdvectVert"):
        _close(_adj(gpu, op, lam, None), _adj(ref, op, lam, None))
    gpu.close()


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn", "tiny_periodic"])
@pytest.mark.parametrize("itime", [1, 2])
def test_adjoint_step_matches_oracle(name, itime):
    cfg, gpu, ref = pair(name)
    q = _prime(cfg, gpu, ref, seed=23)
    rng = np.random.default_rng(itime)
    lam = np.asfortranarray(rng.standard_normal(q.shape))
    lam_dep = np.asfortranarray(rng.standard_normal((cfg.nx, cfg.ny, cfg.ns)))
    for m in (gpu, ref):
        m.set_lambda(lam)
        m.set_lambda_dep(lam_dep)
        m.adj_step(itime)
    _close(gpu.get_lambda(), ref.get_lambda())
    # the forward state is left as it was
    assert np.array_equal(gpu.interior(), q)
    gpu.close()


def test_cloud_load_bitwise():
    cfg, gpu, ref = pair("tiny_stretch")
    _prime(cfg, gpu, ref, seed=29)
    assert np.array_equal(gpu.cloud_load(), ref.cloud_load())
    w = np.asfortranarray(np.random.default_rng(1).standard_normal((cfg.nx, cfg.ny)))
    for m in (gpu, ref):
        m.adj_zero()
        m.adj_add_cloud_load(w)
    assert np.array_equal(gpu.get_lambda(), ref.get_lambda())
    gpu.close()


def test_adjoint_needs_full_box():
    from volcano_ash3d_b200 import A3GError
    cfg, gpu, ref = pair("tiny_subgrid")
    _prime(cfg, gpu, ref, seed=2)
    with pytest.raises(A3GError):
        gpu.adj_advect_x(np.zeros((cfg.nx, cfg.ny, cfg.nz, cfg.ns), order="F"))
    gpu.close()


def _inversion(name, hours):
    from volcano_ash3d_b200 import adjoint as adj
    from volcano_ash3d_b200 import synthetic as syn
    cfg = syn.make_config(name)
    return cfg, adj.SourceInversion(cfg, hours=hours)


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn"])
def test_source_gradient_matches_oracle(name):
    cfg, inv = _inversion(name, 2)
    _, gpu, ref = pair(cfg)
    _, loads, logs, _ = inv.forward(ref, inv.prior(seed=1, lognormal_sigma=0.5))
    obs = {h: loads[h] * (1 + 0.05 * np.random.default_rng(h).standard_normal(loads[h].shape))
           for h in loads}
    p = inv.prior()
    Jg, gg = inv.gradient(gpu, p, obs, K=5)
    Jr, gr = inv.gradient(ref, p, obs, K=5)
    np.testing.assert_allclose(Jg, Jr, rtol=1e-12)
    assert np.abs(gg - gr).max() <= 1e-10 * np.abs(gr).max()
    gpu.close()


def test_source_gradient_gpu_finite_differences():
    cfg, inv = _inversion("tiny_cn", 2)
    _, gpu, _ = pair(cfg)
    _, loads, _, _ = inv.forward(gpu, inv.prior(seed=2, lognormal_sigma=0.5))
    obs = {h: loads[h] * 1.05 for h in loads}
    p = inv.prior()
    J, g = inv.gradient(gpu, p, obs, K=8)
    rng = np.random.default_rng(9)
    active = np.argwhere(p > 0)  # at a zero source, +-h crosses the limiter kinks at c = 0
    for _ in range(6):
        i = tuple(int(v) for v in active[rng.integers(0, len(active))])
        h = 1e-4 * p[i]
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (inv.forward(gpu, pp, obs)[0] - inv.forward(gpu, pm, obs)[0]) / (2 * h)
        assert abs(g[i] - fd) <= 1e-4 * abs(fd), (i, g[i], fd)
    gpu.close()


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_latlon", "tiny_tall", "tiny_stretch", "tiny_wide"])
@pytest.mark.parametrize("limiter", ["superbee", "minmod", "mc", "fromm", "laxwen", "bw", "none"])
def test_adjoint_block_form_equals_gather_form(name, limiter):
    """The four-cell block form of the adjoint advection sweep (the default)
    and the cell-per-thread gather form give the same bits, deposit adjoint
    included (variant direction 5: 0 blocks, 1 gather)."""
    from volcano_ash3d_b200 import synthetic as syn
    cfg = syn.make_config(name)
    cfg.limiter = limiter
    cfg, gpu, ref = pair(cfg)
    _prime(cfg, gpu, ref, seed=31)
    rng = np.random.default_rng(8)
    lam = np.asfortranarray(rng.standard_normal((cfg.nx, cfg.ny, cfg.nz, cfg.ns)))
    lam_dep = np.asfortranarray(rng.standard_normal((cfg.nx, cfg.ny, cfg.ns)))
    for op in ("advect_x", "advect_y", "AdvectVert"):
        gpu.set_variant(5, 0)
        blk = _adj(gpu, op, lam, lam_dep)
        gpu.set_variant(5, 1)
        gat = _adj(gpu, op, lam, lam_dep)
        assert np.array_equal(blk, gat), op
    gpu.close()
