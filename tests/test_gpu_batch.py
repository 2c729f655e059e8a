"""Batched rendering: many uneven images in one graph launch (mt_batch_*)."""
import numpy as np
import pytest
import torch

import marmel_trace_b200 as mt
from marmel_trace_b200 import scenes
from marmel_trace_b200.batch import BatchRenderer

pytestmark = pytest.mark.gpu


def _small_workload(n=7, seed=11):
    rng = np.random.default_rng(seed)
    sizes = [(64, 48), (96, 64), (40, 40), (128, 72), (72, 96), (32, 24), (80, 80)]
    out = []
    for i in range(n):
        d = scenes.mixed_scene(rng, int(rng.integers(500, 4000)))
        w, h = sizes[i % len(sizes)]
        out.append(dict(desc=d, width=w, height=h, spp=int(rng.choice([1, 3, 4, 6])), depth=int(rng.integers(2, 9))))
    return out


def test_batch_matches_single_image_renders(mtlib):
    """Each image of the batch is bit-identical to the same image rendered on
    its own: the per-sample values do not depend on the batch split and the
    pixel sums run in sample order either way."""
    wl = _small_workload()
    gs = [mt.GpuScene(it["desc"], integrator="wavefront") for it in wl]
    cams = [it["desc"].make_camera(it["width"], it["height"]) for it in wl]
    items = [(g, c, it["width"], it["height"], it["spp"], it["depth"]) for g, c, it in zip(gs, cams, wl)]
    br = BatchRenderer(lanes=3, queue_capacity=1 << 14)
    imgs, item_ms, total_ms = br.render(items)
    assert len(item_ms) == len(items) and all(0.0 < t <= total_ms + 1e-3 for t in item_ms)
    for g, c, it, img in zip(gs, cams, wl, imgs):
        ref = g.linear(c, it["width"], it["height"], it["spp"], it["depth"])
        assert np.array_equal(img.cpu().numpy(), ref)
    # a second call reuses the captured graph (same shapes, new cameras)
    cams2 = [it["desc"].make_camera(it["width"], it["height"]) for it in wl]
    items2 = [(g, c, it["width"], it["height"], it["spp"], it["depth"]) for g, c, it in zip(gs, cams2, wl)]
    imgs2, _, _ = br.render(items2)
    for a, b in zip(imgs, imgs2):
        assert torch.equal(a, b)
    br.release()
    for g in gs:
        g.release()


def test_batch_rejects_bad_items(mtlib):
    d = scenes.spheres_scene(n_spheres=8)
    g = mt.GpuScene(d, precision="fp64")
    cam = d.make_camera(16, 16)
    br = BatchRenderer(lanes=2)
    with pytest.raises(RuntimeError):
        br.render([(g, cam, 16, 16, 2, 3)])  # FP64 scene
    g.release()
    g = mt.GpuScene(d)
    with pytest.raises(RuntimeError):
        br.render([(g, cam, 0, 16, 2, 3)])  # zero width
    with pytest.raises(RuntimeError):
        br.render([(g, cam, 16, 16, 0, 3)])  # no samples
    br.release()
    g.release()
