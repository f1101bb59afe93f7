"""GPU test of a3g_mass_aloft_noalloc, the entry point for callers that
cannot allocate device memory when they need the airborne mass: hosts that
reserve all GPU memory up front and forbid allocation later, and hosts that
pass buffers from their own memory manager.

It must agree with the context path (a3g_timestep_totals' mass_aloft) within
the tolerance the totals tests use (1e-13 relative), and with the oracle's
mass_aloft, on two calls in a row.  The second call runs on a non-default
stream with fewer grain bins and a padded row pitch, so it reads the
library's fixed scratch array over the larger first call's leftovers.  The
caller's current device must be the same after each call.  The file name
makes pytest collect it last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))


def test_noalloc_mass_matches_context_path_on_two_calls():
    import torch
    import ash3d_oracle as orc
    from volcano_ash3d_b200 import _lib, synthetic as syn
    from volcano_ash3d_b200.model import Ash3dGPU

    lib = _lib.load()
    cfg = syn.make_config("tiny_latlon")  # cell volumes vary with j and k
    nx, ny, nz, ns = cfg.nx, cfg.ny, cfg.nz, cfg.ns
    assert ns >= 2
    gpu = Ash3dGPU(cfg)
    ref = orc.OracleModel(cfg)
    kap = gpu.geo["kappa"][2:nx + 2, 2:ny + 2, 2:nz + 2]
    kap_d = torch.tensor(np.ascontiguousarray(kap.transpose(2, 1, 0)), dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(2024)
    side = torch.cuda.Stream()
    # call 0: all grains, default stream, tight rows; call 1: one grain fewer,
    # a caller's stream, padded rows
    for call, (pitch, nsc, stream) in enumerate(((nx, ns, None), (nx + 3, ns - 1, side))):
        q = np.asfortranarray(rng.uniform(0.0, 1.0e3, (nx, ny, nz, ns)) * (call + 1))
        gpu.set_interior(q)
        _, mass_ctx = gpu.TimeStepTotals()
        ref.set_interior(q)
        _, mass_orc = ref.TimeStepTotals()
        host = np.zeros((ns, nz, ny, pitch))
        host[:, :, :, :nx] = q.transpose(3, 2, 1, 0)
        conc_d = torch.tensor(host, dtype=torch.float64, device="cuda")
        out = torch.full((ns,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        handle = None if stream is None else C.c_void_p(stream.cuda_stream)
        _lib.check(lib.a3g_mass_aloft_noalloc(0, _ptr(conc_d), _ptr(kap_d), nx, ny, nz, nsc, pitch,
                                              _ptr(out), handle))
        assert torch.cuda.current_device() == 0
        if stream is not None:
            stream.synchronize()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got[:nsc], mass_ctx[:nsc], rtol=1e-13, atol=0)
        np.testing.assert_allclose(got[:nsc], mass_orc[:nsc], rtol=1e-13, atol=0)
        # grain bins past nsc are not written
        assert np.all(np.isnan(got[nsc:]))
    # more grain bins than the fixed scratch array holds: a clear error
    out = torch.zeros(65, dtype=torch.float64, device="cuda")
    rc = lib.a3g_mass_aloft_noalloc(0, _ptr(conc_d), _ptr(kap_d), nx, ny, nz, 65, nx, _ptr(out), None)
    assert rc == 1 and b"64" in lib.a3g_last_error()
    gpu.close()
