"""The BVH built on the device (mt_bvh_build_device, the reference's
binned-SAH algorithm run breadth-first) against the host build, which is the
reference's tree node for node (tests/test_host.py).

Split decisions depend only on each node's set of primitives, so the device
tree has the host tree's nodes, bounds, leaves, links and preorder numbering;
only the order of the primitives inside each node differs, so leaves are
compared as sets. Scenes built either way render identical images.
"""
import time

import numpy as np
import pytest
import torch

import marmel_trace_b200 as mt
from marmel_trace_b200 import scenes
from marmel_trace_b200.api import bvh_build_device, bvh_build_host

pytestmark = pytest.mark.gpu


def _scene(name):
    if name == "spheres":
        return scenes.spheres_scene()
    if name == "torus":
        return scenes.torus_field_scene(n_instances=512)
    rng = np.random.default_rng(7)
    return scenes.mixed_scene(rng, 20000)


@pytest.mark.parametrize("name", ["spheres", "torus", "mixed"])
def test_device_tree_is_the_reference_tree(mtlib, name):
    d = _scene(name)
    hb, hl, ho, hd = bvh_build_host(d.prims)
    db, dl, do, dd, ms = bvh_build_device(d.prims)
    assert len(hb) == len(db) and hd == dd
    assert np.array_equal(hl, dl)           # links, leaf first / count
    assert np.array_equal(hb, db)           # bounds (-0.0 == 0.0)
    assert sorted(ho.tolist()) == sorted(do.tolist())
    leaves = np.nonzero(hl[:, 3] > 0)[0]
    for i in leaves:
        f, c = hl[i, 2], hl[i, 3]
        assert sorted(ho[f:f + c].tolist()) == sorted(do[f:f + c].tolist())


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_scene_built_on_device_renders_the_same_image(mtlib, precision):
    d = scenes.torus_field_scene(n_instances=128)
    W, H, SPP, DEPTH = 96, 64, 2, 5
    cam = d.make_camera(W, H)
    imgs = []
    for builder in (0, 1):
        with mt.GpuScene(d, precision=precision, integrator="wavefront", bvh_builder=builder) as g:
            imgs.append(g.linear(cam, W, H, SPP, DEPTH))
    assert np.array_equal(imgs[0], imgs[1])


def test_device_build_time(mtlib):
    """The 1M-triangle torus field: device build time next to the host's."""
    d = scenes.torus_field_scene()
    t0 = time.perf_counter()
    hb, _, _, _ = bvh_build_host(d.prims)
    host_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    db, dl, _, _, ms = bvh_build_device(d.prims)
    dev_wall = time.perf_counter() - t0
    print(f"host build {host_s:.2f} s; device build {ms:.1f} ms device time, {dev_wall:.2f} s wall per call")
    assert len(hb) == len(db)


def test_large_scene_shape_matches_reference(mtlib, oracle):
    """A scaled-down version of the large configuration (water heightfield,
    trees, spheres, emitters, soft sun) built on the device: the FP64 image
    equals the reference's except where rays meet the water near the
    critical angle (last-ulp cos / sin differences amplified by refraction)."""
    d = scenes.large_scene(grid=64, n_trees=2, n_spheres=20)
    w, h = 96, 64
    cam = d.make_camera(w, h)
    rs = oracle.RefScene.from_desc(d, cam)
    want = rs.pathtrace_render(w, h, 4, 12)
    rs.free()
    with mt.GpuScene(d, precision="fp64", integrator="wavefront", bvh_builder=1) as g:
        got = g.pathtrace(cam, w, h, 4, 12)
    assert (got != want).mean() < 2e-3
