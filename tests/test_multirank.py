"""Grain-sharded runs over torch.distributed (gloo, world size 2, CPU).

The multi-GPU path shards the grain bins; each rank runs the full transport
step on its bins, and the ranks exchange only the CFL maxima (all-reduce MAX)
and the totals (all-reduce SUM).  These tests run that host logic with the
oracle as each rank's model, so they need no GPU: the sharded run must give
the single-process run's dt sequence bitwise, each rank's concentration must
equal the matching grains of the single-process field bitwise, and the summed
totals must agree to 1e-13.
"""
import os
import pathlib
import socket
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pipelined_oracle(orc, syn):
    """The oracle with the entry points of the lag-one loop (driver.Pipeline)
    that the device provides: the scheduled source, the queued totals, and
    the CFL maxima in a buffer the ranks all-reduce in place."""

    class PipelinedOracle(orc.OracleModel):
        def set_source_pulses(self, ivent, jvent, pulses, norm_col):
            self._pulses, self._norm_col, self._state = pulses, norm_col, [1, 1]
            self._kappa = syn.geometry(self.cfg)["kappa"]

        def add_source_scheduled(self, time):
            dt = self._dt_pending
            flux = syn.scheduled_source_flux(self.cfg, self._pulses, self._norm_col, self._kappa, self._state,
                                             time, dt)
            if flux is not None:
                self.add_source(flux, dt)

        def totals_async(self):  # the totals of this state, kept under a ticket
            self._tots = getattr(self, "_tots", {})
            t = self._ticket = getattr(self, "_ticket", -1) + 1
            self._tots[t] = self.TimeStepTotals()
            return t

        def totals_get(self, ticket):
            return self._tots.pop(ticket)

        def cfl_maxima_device(self):
            self._vmax = self.cfl_maxima()
            return self._vmax

        def adjust_dt_device_maxima_async(self, n_gs_aloft_total, time, next_write_time, simtime):
            self._dt_pending = self.adjust_dt_from_maxima(self._vmax, n_gs_aloft_total, time, next_write_time,
                                                          simtime)

    return PipelinedOracle


def _rank_main(rank: int, world: int, port: int, cfg_name: str, steps: int, out_dir: str, fast: bool = False,
               pipelined: bool = False):
    sys.path.insert(0, str(ROOT / "tests"))
    sys.path.insert(0, str(ROOT / "oracle"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import conftest
        import ash3d_oracle as orc
        mod = conftest._load_pkg()
        pkg, syn = mod.driver, mod.synthetic
        import dataclasses
        gcfg = dataclasses.replace(syn.make_config(cfg_name), fast_dt=fast)
        cfg = pkg.split_grains(gcfg, rank, world)
        model = (_pipelined_oracle(orc, mod.synthetic) if pipelined else orc.OracleModel)(cfg, threads=1)

        class CountingComm(pkg.Comm):
            max_calls = 0

            def max(self, a):
                CountingComm.max_calls += 1
                return super().max(a)

            def max_inplace(self, buf):
                CountingComm.max_calls += 1
                return super().max_inplace(buf)

        comm = CountingComm()
        if pipelined:
            st = pkg.run_pipelined(model, cfg, max_steps=steps, comm=comm, n_gs_aloft_total=gcfg.ns)
        else:
            st = pkg.run(model, cfg, max_steps=steps, comm=comm, n_gs_aloft_total=gcfg.ns)
        hist = np.array([[r.time, r.dt, r.aloft, r.dep, r.outflow, r.tot] for r in st.history])
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), hist=hist, conc=model.interior(),
                 dep=model.outflows()["deposit"], max_calls=CountingComm.max_calls, hour=st.hour)
    finally:
        dist.destroy_process_group()


def _sharded(cfg_name: str, world: int, steps: int, tmp_path, fast: bool = False, pipelined: bool = False):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, cfg_name, steps, str(tmp_path), fast, pipelined))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
        assert p.exitcode == 0, f"rank process exit code {p.exitcode}"
    return [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]


@pytest.mark.parametrize("cfg_name,steps,fast,pipelined", [
    ("tiny_proj", 12, False, False), ("tiny_latlon", 8, False, False),
    ("tiny_proj", None, True, False), ("tiny_latlon", None, True, False),
    ("tiny_proj", 12, False, True), ("tiny_latlon", None, True, True)])
def test_grain_sharded_matches_single(pkg, oracle_mod, cfg_name, steps, fast, pipelined, tmp_path):
    """With FAST_DT the ranks exchange the CFL maxima only at the met-step
    loads (the first pair: two, then one per later load), not every step.
    The pipelined sharded loop (driver.Pipeline with a Comm: maxima all-
    reduced in place, the totals summed when a record is collected) gives the
    same bits as the plain single-process loop."""
    import dataclasses
    syn, drv = pkg.synthetic, pkg.driver
    gcfg = dataclasses.replace(syn.make_config(cfg_name), fast_dt=fast)
    world = 2
    ranks = _sharded(cfg_name, world, steps, tmp_path, fast, pipelined)

    ref = oracle_mod.OracleModel(gcfg, threads=1)
    st = drv.run(ref, gcfg, max_steps=steps)
    ref_hist = np.array([[r.time, r.dt, r.aloft, r.dep, r.outflow, r.tot] for r in st.history])
    ref_c = ref.interior()
    ref_dep = ref.outflows()["deposit"]

    for r in range(world):
        h = ranks[r]["hist"]
        assert h.shape == ref_hist.shape
        # identical dt sequence and clock on every rank (bitwise)
        assert np.array_equal(h[:, :2], ref_hist[:, :2])
        lo, hi = drv.grain_range(gcfg.ns, r, world)
        assert np.array_equal(ranks[r]["conc"], ref_c[..., lo:hi])
        assert np.array_equal(ranks[r]["dep"], ref_dep[..., lo:hi])
        # totals are all-reduced: every rank holds the global sums
        np.testing.assert_allclose(h[:, 2:], ref_hist[:, 2:], rtol=1e-13, atol=1e-300)
        if fast:
            assert int(ranks[r]["hour"]) >= 1
            assert int(ranks[r]["max_calls"]) == 2 + int(ranks[r]["hour"])
        else:
            assert int(ranks[r]["max_calls"]) == len(h)


def test_split_grains_partition(pkg):
    syn, drv = pkg.synthetic, pkg.driver
    cfg = syn.make_config("C2")
    for world in (1, 2, 3, 4, 7, 10):
        got = []
        for r in range(world):
            c = drv.split_grains(cfg, r, world)
            lo, hi = drv.grain_range(cfg.ns, r, world)
            assert c.ns == hi - lo and c.fall_mps == cfg.fall_mps[lo:hi]
            got.extend(c.fall_mps)
        assert tuple(got) == cfg.fall_mps
    with pytest.raises(ValueError):
        drv.split_grains(cfg, 0, 11)


def _rank_netcdf(rank: int, world: int, port: int, cfg_name: str, steps: int, out_dir: str):
    sys.path.insert(0, str(ROOT / "tests"))
    sys.path.insert(0, str(ROOT / "oracle"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import conftest
        import ash3d_oracle as orc
        mod = conftest._load_pkg()
        pkg, syn = mod.driver, mod.synthetic
        gcfg = syn.make_config(cfg_name)
        cfg = pkg.split_grains(gcfg, rank, world)
        comm = pkg.Comm()
        model = orc.OracleModel(cfg, threads=1)
        pkg.run(model, cfg, max_steps=steps, comm=comm, n_gs_aloft_total=gcfg.ns)
        ash, dep = pkg.gather_netcdf(model, comm, gcfg.ns)
        fresh = orc.OracleModel(cfg, threads=1)
        pkg.scatter_restart(fresh, comm, cfg, gcfg.ns, ash, dep)
        save = dict(conc=fresh.interior(), xy1=fresh.outflows()["xy1"])
        if rank == 0:
            save.update(ash=ash, dep=dep)
        else:
            assert ash is None and dep is None
        np.savez(os.path.join(out_dir, f"nc{rank}.npz"), **save)
    finally:
        dist.destroy_process_group()


def test_sharded_netcdf_gather_and_restart(pkg, oracle_mod, tmp_path):
    """The ranks' ashcon/depocon blocks assemble on rank 0 into the
    single-process run's arrays bitwise (uneven blocks: 3 bins over 2 ranks),
    and a restart scattered from rank 0 gives each rank its own bins."""
    import torch.multiprocessing as mp
    syn, drv = pkg.synthetic, pkg.driver
    cfg_name, steps, world = "tiny_proj", 10, 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_netcdf, args=(r, world, port, cfg_name, steps, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
        assert p.exitcode == 0, f"rank process exit code {p.exitcode}"
    ranks = [np.load(tmp_path / f"nc{r}.npz") for r in range(world)]

    gcfg = syn.make_config(cfg_name)
    ref = oracle_mod.OracleModel(gcfg, threads=1)
    drv.run(ref, gcfg, max_steps=steps)
    ash, dep = ref.output_ashcon()
    assert np.array_equal(ranks[0]["ash"], ash) and np.array_equal(ranks[0]["dep"], dep)
    assert ash.max() > 0.0 and dep.max() > 0.0
    for r in range(world):
        lo, hi = drv.grain_range(gcfg.ns, r, world)
        assert np.array_equal(ranks[r]["conc"], ash[..., lo:hi].astype(np.float64))
        assert np.array_equal(ranks[r]["xy1"], dep[..., lo:hi].astype(np.float64))
