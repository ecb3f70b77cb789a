"""The allocation-free trace entry point, liar_gpu_trace_device_noalloc, called through the C ABI.

It serves callers that cannot call cudaMalloc while tracing (an application whose pool
allocator owns all device memory, a frame loop that must not stall its other streams, a
plugin with a fixed memory budget). Its results must equal those of liar_gpu_trace_device,
bit for bit, on two calls in a row (the second call reuses the device scratch array the first
one left behind), and neither call may change the free device memory. This file is collected
last on purpose."""
import ctypes as C

import numpy as np
import pytest

from liar_b200 import scenes
from liar_b200._native import lib
from liar_b200.trace import Context, Mesh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = Context(0)
    v, f = scenes.displaced_icosphere(levels=6, seed=11)
    mesh = Mesh(ctx, v, f)
    rays = scenes.random_rays(v, 300007, seed=12)
    rays[::3, 7] = 0.6
    d_rays = torch.from_numpy(rays).cuda()
    yield torch, ctx, mesh, d_rays
    mesh.close()
    ctx.close()


def reference_hits(torch, ctx, mesh, d_rays, any_hit):
    out = torch.empty((d_rays.shape[0], 2), dtype=torch.int32, device="cuda")
    rc = lib().liar_gpu_trace_device(ctx.handle, mesh.handle, C.c_void_p(d_rays.data_ptr()), d_rays.shape[0],
                                     C.c_void_p(out.data_ptr()), int(any_hit), None)
    assert rc == 0
    ctx.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("any_hit", [0, 1])
def test_noalloc_matches_existing_entry_point_twice(setup, any_hit):
    torch, ctx, mesh, d_rays = setup
    ref = reference_hits(torch, ctx, mesh, d_rays, any_hit)
    assert (ref[:, 0] >= 0).mean() > 0.1
    stream = torch.cuda.Stream()
    for call in range(2):
        out = torch.full((d_rays.shape[0], 2), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib().liar_gpu_trace_device_noalloc(mesh.handle, C.c_void_p(d_rays.data_ptr()), d_rays.shape[0],
                                                 C.c_void_p(out.data_ptr()), any_hit, C.c_void_p(stream.cuda_stream))
        assert rc == 0, f"call {call}: status {rc}"
        # nothing allocated on the device, on the first call (which does the per-device set-up)
        # as on the second
        assert torch.cuda.mem_get_info()[0] == free_before, f"call {call} changed free device memory"
        got = out.cpu().numpy()
        if any_hit:
            np.testing.assert_array_equal(got[:, 0] >= 0, ref[:, 0] >= 0)
        else:
            np.testing.assert_array_equal(got[:, 0], ref[:, 0])
            hit = ref[:, 0] >= 0
            np.testing.assert_array_equal(got[hit, 1], ref[hit, 1])  # t, bit pattern


def test_noalloc_rejects_oversized_and_bad_arguments(setup):
    torch, ctx, mesh, d_rays = setup
    out = torch.empty((16, 2), dtype=torch.int32, device="cuda")
    L = lib()
    # more rays than the per-call maximum (2^31): rejected before anything is read
    assert L.liar_gpu_trace_device_noalloc(mesh.handle, C.c_void_p(d_rays.data_ptr()), (1 << 31) + 1,
                                           C.c_void_p(out.data_ptr()), 0, None) == -1
    assert L.liar_gpu_trace_device_noalloc(None, C.c_void_p(d_rays.data_ptr()), 16, C.c_void_p(out.data_ptr()), 0,
                                           None) == -1
    assert L.liar_gpu_trace_device_noalloc(mesh.handle, C.c_void_p(d_rays.data_ptr() + 4), 16,
                                           C.c_void_p(out.data_ptr()), 0, None) == -1
    assert L.liar_gpu_trace_device_noalloc(mesh.handle, None, 0, None, 0, None) == 0
