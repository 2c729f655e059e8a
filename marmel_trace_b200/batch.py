"""Many images in one CUDA-graph launch (mt_batch_* of the C ABI).

    br = BatchRenderer(lanes=8)
    images, item_ms, total_ms = br.render([(scene, camera, width, height, spp, depth), ...])

Each item renders samples [s0, s0 + spp) of its own scene (a GpuScene, FP32)
into a device tensor (height, width, 3) of mean linear RGB. The batch context
keeps `lanes` sets of wavefront queues; items are spread over the lanes
longest first and all lanes run concurrently inside one graph launch.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _capi


class BatchRenderer:
    def __init__(self, lanes: int = 8, queue_capacity: int = 0, device: int = 0):
        self.lib = _capi.load()
        self.h = C.c_void_p()
        _capi.check(self.lib.mt_batch_create(lanes, queue_capacity, device, C.byref(self.h)), "mt_batch_create")
        self.device = device

    def render(self, items, s0: int = 0, timed: bool = True, out=None):
        """items: (GpuScene, Camera, width, height, spp, depth) tuples.
        Returns (list of device images, per-item ms, total ms); the times are
        None when timed is False (then the call does not wait)."""
        n = len(items)
        arr = (_capi.MtBatchItem * n)()
        imgs = out if out is not None else [
            torch.empty((it[3], it[2], 3), dtype=torch.float32, device=f"cuda:{self.device}") for it in items]
        for i, (scene, cam, w, h, spp, depth) in enumerate(items):
            a = arr[i]
            a.scene = scene.h.value
            a.cam = C.cast(C.pointer(cam.c), C.c_void_p)
            a.width, a.height, a.s0, a.spp, a.depth = w, h, s0, spp, depth
            a.out_dev = imgs[i].data_ptr()
        item_ms = (C.c_float * n)()
        total = C.c_float()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        rc = self.lib.mt_batch_render(self.h, n, arr, stream, item_ms if timed else None,
                                      C.byref(total) if timed else None)
        _capi.check(rc, "mt_batch_render")
        if not timed:
            return imgs, None, None
        return imgs, list(item_ms), total.value

    def release(self):
        if self.h:
            self.lib.mt_batch_release(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
