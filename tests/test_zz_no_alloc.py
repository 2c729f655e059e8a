"""mt_render_accumulate_device_noalloc: the path-tracing entry point for
callers that cannot allocate device memory while rendering (an application
whose own pool allocator owns the whole device budget, or a loop that must not
pay cudaMalloc's device-wide synchronisation). It must give the same image as
mt_render_accumulate_device, call after call, although every call reuses one
fixed scratch array inside the library.

This file is collected last on purpose: a run that stops at the first failure
has run every other test before it.
"""
import numpy as np
import pytest
import torch

import marmel_trace_b200 as mt
from marmel_trace_b200 import _capi, scenes

pytestmark = pytest.mark.gpu

W, H, DEPTH = 96, 72, 6   # 6912 pixels, under the 16384-pixel limit


def _render(fn, g, cam, s0, s1, acc_tensor, accumulate):
    if fn.__name__ == "mt_render_accumulate_device":  # the allocating entry point takes a mode (0 = path tracer)
        rc = fn(g.h, cam.ref, W, H, s0, s1, DEPTH, 0, acc_tensor.data_ptr(), accumulate, None)
    else:
        rc = fn(g.h, cam.ref, W, H, s0, s1, DEPTH, acc_tensor.data_ptr(), accumulate, None)
    _capi.check(rc, fn.__name__)
    torch.cuda.synchronize()
    return acc_tensor.cpu().numpy().copy()


def test_noalloc_matches_allocating_entry_point_two_calls(mtlib):
    d = scenes.torus_field_scene(n_instances=256, area=30.0)
    cam = d.make_camera(W, H)
    with mt.GpuScene(d, precision="fp32", integrator="wavefront") as g:
        ref_acc = torch.zeros((H, W, 3), dtype=torch.float32, device="cuda")
        new_acc = torch.zeros((H, W, 3), dtype=torch.float32, device="cuda")
        for call, (s0, s1, accumulate) in enumerate([(0, 4, 0), (4, 8, 1)]):
            want = _render(mtlib.mt_render_accumulate_device, g, cam, s0, s1, ref_acc, accumulate)
            got = _render(mtlib.mt_render_accumulate_device_noalloc, g, cam, s0, s1, new_acc, accumulate)
            err = np.abs(got - want)
            tol = 1e-4 * np.maximum(1.0, np.abs(want))
            assert (err <= tol).mean() > 0.999, f"call {call}: max {err.max()}, mean {err.mean()}"
            assert want.mean() > 0


def test_noalloc_rejects_images_beyond_its_limit(mtlib):
    d = scenes.spheres_scene()
    cam = d.make_camera(256, 256)
    with mt.GpuScene(d, precision="fp32") as g:
        acc = torch.zeros((256, 256, 3), dtype=torch.float32, device="cuda")
        rc = mtlib.mt_render_accumulate_device_noalloc(g.h, cam.ref, 256, 256, 0, 1, 4, acc.data_ptr(), 0, None)
        assert rc == _capi.MT_ERR_INVALID
        assert b"16384" in mtlib.mt_last_error()
