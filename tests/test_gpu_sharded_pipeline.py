"""The lag-one loop of a grain-sharded run on B200, one rank over NCCL: the CFL
maxima go through a3g_cfl_maxima_device, an in-place NCCL all-reduce (MAX)
ordered on the context's stream, and a3g_adjust_dt_device_maxima_async, with
no host read-back; with FAST_DT they are exchanged only at met-step loads.
The run gives the oracle's plain loop the same dt sequence, state and
outflows bit for bit and the totals to 1e-13, and the maxima the device
buffer holds equal a3g_cfl_maxima's.  (More ranks need more GPUs; the host
logic of two ranks is covered with gloo on the CPU.)"""
import os
import pathlib
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(port: int, name: str, fast: bool, steps: int, out: str):
    sys.path.insert(0, str(ROOT / "tests"))
    sys.path.insert(0, str(ROOT / "oracle"))
    import dataclasses
    import datetime

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        import conftest
        import ash3d_oracle as orc
        pkg = conftest._load_pkg()
        drv, syn = pkg.driver, pkg.synthetic
        from volcano_ash3d_b200.model import Ash3dGPU
        cfg = dataclasses.replace(syn.make_config(name), fast_dt=fast)
        geo = syn.geometry(cfg)
        gpu = Ash3dGPU(cfg, geo=geo)

        class CountingComm(drv.Comm):
            host_max = inplace_max = 0

            def max(self, a):
                CountingComm.host_max += 1
                return super().max(a)

            def max_inplace(self, buf):
                CountingComm.inplace_max += 1
                return super().max_inplace(buf)

        comm = CountingComm(device=torch.device("cuda", 0))
        sg = drv.run_pipelined(gpu, cfg, max_steps=steps, geo=geo, comm=comm, n_gs_aloft_total=cfg.ns)
        # the device buffer of the maxima against the host-returning entry point
        dev = torch.as_tensor(gpu.cfl_maxima_device(), device="cuda").cpu().numpy().copy()
        host = gpu.cfl_maxima()
        ref = orc.OracleModel(cfg, geo=geo)
        sr = drv.run(ref, cfg, max_steps=steps, geo=geo)
        hg = np.array([[r.time, r.dt, r.aloft, r.dep, r.outflow, r.tot, r.source_cum] for r in sg.history])
        hr = np.array([[r.time, r.dt, r.aloft, r.dep, r.outflow, r.tot, r.source_cum] for r in sr.history])
        og, orf = gpu.outflows(), ref.outflows()
        np.savez(out, hg=hg, hr=hr, cg=gpu.interior(), cr=ref.interior(), dev=dev, host=host,
                 og=np.concatenate([og[k].ravel() for k in sorted(og)]),
                 orf=np.concatenate([orf[k].ravel() for k in sorted(orf)]),
                 host_max=CountingComm.host_max, inplace_max=CountingComm.inplace_max, hour=sg.hour)
        gpu.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,fast,steps", [("tiny_proj", False, 16), ("tiny_latlon", False, 12),
                                             ("tiny_cn", True, None)])
def test_sharded_pipeline_one_rank(name, fast, steps, tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "r.npz")
    p = mp.get_context("spawn").Process(target=_rank, args=(_free_port(), name, fast, steps, out))
    p.start()
    p.join(timeout=300)
    if p.is_alive():
        p.kill()
        p.join()
    assert p.exitcode == 0
    r = np.load(out)
    hg, hr = r["hg"], r["hr"]
    assert hg.shape == hr.shape
    assert np.array_equal(hg[:, :2], hr[:, :2])          # time and dt, bitwise
    assert np.array_equal(hg[:, 6], hr[:, 6])            # SourceCumulativeVol
    np.testing.assert_allclose(hg[:, 2:6], hr[:, 2:6], rtol=1e-13, atol=1e-30)
    assert np.array_equal(r["cg"], r["cr"])
    assert np.array_equal(r["og"], r["orf"])
    assert np.array_equal(r["dev"], r["host"])
    if fast:  # maxima only at the met-step loads, through the host
        assert int(r["inplace_max"]) == 0 and int(r["host_max"]) == 2 + int(r["hour"])
    else:     # every step on the device, never through the host
        assert int(r["inplace_max"]) == len(hg) and int(r["host_max"]) == 0
