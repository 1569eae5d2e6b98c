"""The allocation-free transmittance entry point (dr_transmittance_noalloc).

It is for callers that cannot let the library allocate device memory: an
application that owns the GPU's memory budget, or one whose other streams
cannot absorb the synchronisation cudaMalloc/cudaFree can cause.  The caller
supplies device buffers for the rays and the result; the library's per-ray
counters live in a fixed device array.

The test calls it through the C ABI twice in a row on the caller's torch
stream, then once on the context's own stream, and checks each result against
the existing entry point (dr_probe_transmittance) on the same rays and random
streams.  Both count the same delta-tracked samples, so the tolerance is the
transmittance test's 1e-4 relative (they agree exactly in practice).  The
second call also shows that a call clears the counters the previous one left.
This file is collected last so that a failure here cannot hide earlier ones.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import c0_cfg, golden_octree, settings_from_cfg

pytestmark = pytest.mark.gpu


def test_noalloc_transmittance_matches_existing_entry_point():
    import torch

    from droplet_b200 import _native as N
    from droplet_b200.renderer import Renderer, stream_handle
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    rng = np.random.default_rng(2027)
    n = 300
    ro = rng.uniform(-1.5, 2.5, (n, 3))
    ro[:, 2] = rng.uniform(-1.0, -0.5, n)  # below the volume, looking up through it
    rd = (0.5 + rng.uniform(-0.3, 0.3, (n, 3))) - ro
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    ro = ro.astype(np.float32)
    rd = rd.astype(np.float32)
    nsamp, seed = 4096, 17
    with Renderer(0) as r:
        r.upload(Octree(nodes, bricks, mlevel))
        r.set_params(settings_from_cfg(c0_cfg(64, 64)))
        expected = r.probe_transmittance(ro, rd, nsamp, seed)
        assert (expected < 0.999).sum() > 50  # many rays cross the medium

        ro_d = torch.as_tensor(ro, device="cuda").contiguous()
        rd_d = torch.as_tensor(rd, device="cuda").contiguous()
        # Two calls in a row on the caller's own stream (the entry point's main
        # use): the fills below are queued on that stream too, so they come
        # before the clear / track / finish kernels of the call.
        ts = torch.cuda.current_stream()
        for _ in range(2):
            out_d = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
            rc = N.lib().dr_transmittance_noalloc(r.handle, C.c_void_p(ro_d.data_ptr()), C.c_void_p(rd_d.data_ptr()),
                                                  n, nsamp, seed, C.c_void_p(out_d.data_ptr()),
                                                  C.c_void_p(stream_handle(ts)))
            N.check(rc)
            ts.synchronize()
            got = out_d.cpu().numpy()
            assert np.allclose(got, expected, rtol=1e-4, atol=0.0), np.abs(got - expected).max()

        # One call on the context's own stream (NULL): torch's fill must have
        # finished before it starts, so synchronise the device first.
        out_d = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = N.lib().dr_transmittance_noalloc(r.handle, C.c_void_p(ro_d.data_ptr()), C.c_void_p(rd_d.data_ptr()),
                                              n, nsamp, seed, C.c_void_p(out_d.data_ptr()), None)
        N.check(rc)
        r.synchronize()
        got = out_d.cpu().numpy()
        assert np.allclose(got, expected, rtol=1e-4, atol=0.0), np.abs(got - expected).max()

        too_many = N.DR_NOALLOC_MAX_RAYS + 1
        rc = N.lib().dr_transmittance_noalloc(r.handle, C.c_void_p(ro_d.data_ptr()), C.c_void_p(rd_d.data_ptr()),
                                              too_many, nsamp, seed, C.c_void_p(out_d.data_ptr()), None)
        assert rc == N.DR_ERR_INVALID
        assert b"DR_NOALLOC_MAX_RAYS" in N.lib().dr_last_error()
