"""The source inversion through the C-ABI pair (a3g_inv_setup,
a3g_forward_checkpointed, a3g_adjoint, a3g_tangent_linear), on B200:

* the library's forward run gives the host loop's observations bit for bit
  (SourceInversion.forward on the same GPU model) and the oracle's to 1e-12;
* its gradient equals the oracle's reverse sweep to 1e-10 of the gradient's
  scale, for the column-load misfit, the deposit misfit over the last hour,
  both, and with FAST_DT;
* the gradient is the same bits whatever the checkpoint budget (every state,
  a few slots, one slot), and the recomputed step counts follow the binomial
  schedule;
* tangent-linear dot-product test: <J dp, w> = <dp, J^T w> to 1e-12 for
  random dp and w, and J p = F(p) (the transport is positively homogeneous
  and piecewise linear in the source, so the tangent-linear run at p in the
  direction p returns the observations themselves);
* central differences of J agree with the gradient to 1e-6 relative (step
  1e-5 of the component);
* the torch.autograd.Function gives the adjoint's gradient for a torch loss;
* with the device met cache off, met steps go through the context's three
  slots (one upload per hour a run moves on or back) and every result is the
  same bits as with the cache.
"""
import ctypes as C

import numpy as np
import pytest

import ash3d_oracle as orc
from volcano_ash3d_b200 import adjoint as adj
from volcano_ash3d_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

HOURS = 2


def _problem(name="tiny_proj", fast_dt=False, seed=1):
    cfg = syn.make_config(name)
    inv = adj.SourceInversion(cfg, hours=HOURS)
    ref = orc.OracleModel(cfg, threads=1)
    zero = np.zeros((cfg.nx, cfg.ny))
    _, loads, _, _ = inv.forward(ref, inv.prior(seed=seed, lognormal_sigma=0.5), fast_dt=fast_dt,
                                 obs_dep=zero, dep_from=1)
    rng = np.random.default_rng(seed + 10)
    obs = {h: loads[h] * (1 + 0.05 * rng.standard_normal(loads[h].shape)) for h in loads if h != "dep"}
    obs_dep = loads["dep"] * (1 + 0.05 * rng.standard_normal(loads["dep"].shape))
    return cfg, inv, ref, obs, obs_dep


def _gpu(cfg, inv, obs=None, obs_dep=None, **kw):
    from volcano_ash3d_b200.model import Ash3dGPU
    gpu = Ash3dGPU(cfg)
    return gpu, adj.InversionGPU(gpu, cfg, HOURS, obs=obs, obs_dep=obs_dep, **kw)


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn", "tiny_latlon"])
def test_forward_matches_host_loop(name):
    cfg, inv, ref, obs, _ = _problem(name)
    p = inv.prior(seed=3, lognormal_sigma=0.3)
    gpu, ig = _gpu(cfg, inv, obs=obs)
    J, loads, _ = ig.forward(p)
    Jh, lh, logs, _ = inv.forward(gpu, p, obs)        # the host loop on the same GPU model
    Jr, lr, _, _ = inv.forward(ref, p, obs)           # the oracle
    assert ig.nsteps == len(logs)
    for h in range(HOURS):
        assert np.array_equal(loads[h], lh[h]), h
        np.testing.assert_allclose(loads[h], lr[h], rtol=1e-12, atol=1e-12 * np.abs(lr[h]).max())
    assert abs(J - Jr) <= 1e-12 * abs(Jr)
    gpu.close()


@pytest.mark.parametrize("case", ["load", "deposit", "both", "both_fast_dt", "cn"])
def test_gradient_matches_oracle(case):
    fast = case == "both_fast_dt"
    cfg, inv, ref, obs, obs_dep = _problem("tiny_cn" if case == "cn" else "tiny_proj", fast_dt=fast)
    use_load = case != "deposit"
    use_dep = case in ("deposit", "both", "both_fast_dt")
    kw = dict(fast_dt=fast, obs_dep=obs_dep if use_dep else None, dep_from=1, load_from=1 if use_dep else 0)
    p = inv.prior()
    Jr, gr = inv.gradient(ref, p, obs if use_load else {}, K=5, **kw)
    gpu, ig = _gpu(cfg, inv, obs=obs if use_load else None, obs_dep=kw["obs_dep"], load_from=kw["load_from"],
                   dep_from=1, fast_dt=fast)
    J, _, _ = ig.forward(p)
    g = ig.adjoint()
    assert abs(J - Jr) <= 1e-12 * abs(Jr)
    scale = np.abs(gr).max()
    assert scale > 0
    np.testing.assert_allclose(g, gr, rtol=0, atol=1e-10 * scale)
    gpu.close()


def test_gradient_independent_of_checkpoint_budget():
    from volcano_ash3d_b200 import _lib
    cfg, inv, ref, obs, obs_dep = _problem()
    p = inv.prior()
    grads, stats = [], []
    from volcano_ash3d_b200.model import Ash3dGPU
    gpu = Ash3dGPU(cfg)
    P = -(-cfg.nx // 8) * 8  # the device row pitch
    level = 8.0 * P * cfg.ny * cfg.nz * cfg.ns
    for slots in (0, 2, 3, 1):  # 0: every state
        ig = adj.InversionGPU(gpu, cfg, HOURS, obs=obs, obs_dep=obs_dep, dep_from=1,
                              snapshot_bytes=(slots + 0.5) * level if slots else 0.0)
        ig.forward(p)
        grads.append(ig.adjoint())
        stats.append(dict(ig.stats))
    N = stats[0]["steps"]
    assert stats[0]["slots"] == N and stats[0]["recomputed"] == 0
    for g in grads[1:]:
        assert np.array_equal(g, grads[0])
    # the recomputed steps: the binomial schedule's total less the first run's share
    for st in stats[1:]:
        assert st["slots"] < N and st["recomputed"] > 0
        r, k = C.c_int64(), C.c_int32()
        _lib.check(gpu.lib.a3g_checkpoint_cost(N, st["slots"] - 1, C.byref(r), C.byref(k)))
        assert st["recomputed"] <= r.value
    assert stats[3]["recomputed"] >= stats[1]["recomputed"] >= stats[2]["recomputed"]
    gpu.close()


@pytest.mark.parametrize("name", ["tiny_proj", "tiny_cn"])
def test_tangent_linear_dot_product(name):
    cfg, inv, ref, obs, obs_dep = _problem(name)
    p = inv.prior()
    gpu, ig = _gpu(cfg, inv, obs=obs, obs_dep=obs_dep, dep_from=1)
    rng = np.random.default_rng(11)
    dp = np.where(p > 0, p * rng.standard_normal(p.shape), 0.0)
    dl, dd = ig.tangent_linear(p, dp)
    wl = rng.standard_normal(dl.shape)
    wd = rng.standard_normal(dd.shape)
    ig.forward(p)
    g = ig.adjoint(wl, wd)
    lhs = float(np.sum(dl * wl) + np.sum(dd * wd))
    rhs = float(np.sum(dp * g))
    assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + abs(rhs)), (lhs, rhs)
    # J p = F(p): the observations themselves
    J, loads, dep = ig.forward(p)
    tl, td = ig.tangent_linear(p, p)
    np.testing.assert_allclose(tl, loads, rtol=0, atol=1e-12 * np.abs(loads).max())
    np.testing.assert_allclose(td, dep, rtol=0, atol=1e-12 * np.abs(dep).max())
    gpu.close()


def test_gradient_matches_central_differences():
    cfg, inv, ref, obs, obs_dep = _problem()
    p = inv.prior()
    gpu, ig = _gpu(cfg, inv, obs=obs, obs_dep=obs_dep, dep_from=1)
    ig.forward(p)
    g = ig.adjoint()
    rng = np.random.default_rng(21)
    active = np.argwhere(p > 0)
    errs = []
    for _ in range(10):
        i = tuple(int(v) for v in active[rng.integers(0, len(active))])
        h = 1e-5 * p[i]
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (ig.forward(pp)[0] - ig.forward(pm)[0]) / (2 * h)
        errs.append(abs(g[i] - fd) / abs(fd))
    assert max(errs) <= 1e-6, errs
    gpu.close()


def test_autograd_function():
    import torch
    cfg, inv, ref, obs, obs_dep = _problem()
    p = inv.prior()
    gpu, ig = _gpu(cfg, inv, obs=obs, obs_dep=obs_dep, dep_from=1, load_from=1)
    fn = adj.TransportObservations()
    pt = torch.tensor(p, dtype=torch.float64, requires_grad=True)
    loads, dep = fn.apply(pt, ig)
    y = torch.tensor(np.stack([obs[h] for h in range(HOURS)]))
    loss = 0.5 * ((loads[1:] - y[1:]) ** 2).sum() + 0.5 * ((dep - torch.tensor(obs_dep)) ** 2).sum()
    loss.backward()
    J, _, _ = ig.forward(p)
    g = ig.adjoint()
    assert abs(float(loss.detach()) - J) <= 1e-12 * J
    np.testing.assert_allclose(pt.grad.numpy(), g, rtol=0, atol=1e-12 * np.abs(g).max())
    gpu.close()


def test_reversal_window():
    """adj_from = 1: the reverse run covers the steps of the second hour only;
    the bins of those steps equal the whole run's bit for bit (their adjoint
    does not depend on earlier steps) and the first hour's bins stay zero."""
    cfg, inv, ref, obs, obs_dep = _problem()
    p = inv.prior(active_hours=HOURS)
    gpu, ig = _gpu(cfg, inv, obs=obs, obs_dep=obs_dep, dep_from=1)
    ig.forward(p)
    g_full = ig.adjoint()
    iw = adj.InversionGPU(gpu, cfg, HOURS, obs=obs, obs_dep=obs_dep, dep_from=1, adj_from=1)
    iw.forward(p)
    g_win = iw.adjoint()
    assert np.any(g_full[:, 1, :] != 0.0)
    assert np.array_equal(g_win[:, 1, :], g_full[:, 1, :])
    assert not np.any(g_win[:, 0, :])
    assert iw.stats["slots"] < ig.stats["slots"]
    gpu.close()


class _CountingMet:
    """The synthetic met source, recording the hours asked for."""

    def __init__(self, cfg):
        self.src = syn.MetSource(cfg)
        self.calls = []

    def step(self, hour):
        self.calls.append(int(hour))
        return self.src.step(hour)


@pytest.mark.parametrize("fast", [False, True])
def test_met_slots_without_cache(fast):
    from volcano_ash3d_b200.model import Ash3dGPU
    cfg, inv, ref, obs, obs_dep = _problem(fast_dt=fast)
    p = inv.prior()
    P = -(-cfg.nx // 8) * 8
    level = 8.0 * P * cfg.ny * cfg.nz * cfg.ns
    gpu = Ash3dGPU(cfg)
    out = []
    for cache in (True, False):
        met = _CountingMet(cfg)
        # two slots: the reversal recomputes across the hour boundary
        ig = adj.InversionGPU(gpu, cfg, HOURS, obs=obs, obs_dep=obs_dep, dep_from=1, fast_dt=fast,
                              snapshot_bytes=2.5 * level, met=met, met_cache=cache)
        n_setup = len(met.calls)
        J, loads, dep = ig.forward(p)
        n_fwd = len(met.calls) - n_setup
        g = ig.adjoint()
        out.append(dict(J=J, loads=loads, dep=dep, g=g, setup=n_setup, fwd=n_fwd,
                        adj=len(met.calls) - n_setup - n_fwd, stats=dict(ig.stats)))
    c, n = out
    assert c["fwd"] == 0 and c["adj"] == 0 and c["setup"] == HOURS + 2  # every step cached once
    assert n["fwd"] == HOURS + 1  # hours 0, 1, ..., HOURS, each uploaded once
    assert n["stats"]["recomputed"] > 0 and n["adj"] >= 1
    assert n["J"] == c["J"]
    assert np.array_equal(n["dep"], c["dep"])
    for h in range(HOURS):
        assert np.array_equal(n["loads"][h], c["loads"][h]), h
    assert np.array_equal(n["g"], c["g"])
    gpu.close()
