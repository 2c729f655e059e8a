"""GPU parity against the oracle (the reference renderer) through the C ABI.

FP64 device path: the reference's double-precision arithmetic restated
operation by operation, so primary rays, hits, distances, occlusion and the
8-bit images must agree exactly.
FP32 device path (production): primary-hit prim ids equal outside the FP32
ambiguity band with t within 1e-5 relative; Whitted bytes within 1/255 on at
least 99.9% of channels; path-traced means within 3 Monte-Carlo standard
errors per pixel.
"""
import numpy as np
import pytest

import marmel_trace_b200 as mt
from marmel_trace_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1(oracle, mtlib):
    d = scenes.spheres_scene()
    return d


def _ref_and_cam(oracle, d, w, h):
    cam = d.make_camera(w, h)
    rs = oracle.RefScene.from_desc(d, cam)
    return rs, cam


@pytest.mark.parametrize("mode", ["pathtrace", "whitted"])
def test_primary_rays_fp64_exact(oracle, c1, mode):
    w, h, spp = 40, 30, 4
    rs, cam = _ref_and_cam(oracle, c1, w, h)
    with mt.GpuScene(c1, precision="fp64") as g:
        got = g.primary_rays(cam, w, h, spp, mode)
    want = rs.primary_rays(w, h, spp, mode)
    assert np.array_equal(got, want)


def test_primary_rays_fp32_close(oracle, c1):
    w, h, spp = 40, 30, 4
    rs, cam = _ref_and_cam(oracle, c1, w, h)
    with mt.GpuScene(c1, precision="fp32") as g:
        got = g.primary_rays(cam, w, h, spp)
    want = rs.primary_rays(w, h, spp)
    assert np.max(np.abs(got - want)) < 1e-5


def _hits(oracle, d, w, h, spp, precision):
    rs, cam = _ref_and_cam(oracle, d, w, h)
    rays = rs.primary_rays(w, h, spp)
    with mt.GpuScene(d, precision=precision) as g:
        got = g.intersect(rays[:, :3], rays[:, 3:], 1e-4, 1e30)
    want = rs.intersect(rays[:, :3], rays[:, 3:], 1e-4, 1e30)
    return got, want, rays


def test_primary_hits_fp64_exact(oracle, c1):
    (gp, gt, gn, gf, gm), (rp, rt, rn, rf, rm), _ = _hits(oracle, c1, 160, 120, 2, "fp64")
    assert np.array_equal(gp, rp)
    assert np.array_equal(gt, rt)
    assert np.array_equal(gn, rn)
    assert np.array_equal(gf, rf)
    assert np.array_equal(gm, rm)


def test_primary_hits_fp32(oracle, c1):
    (gp, gt, *_), (rp, rt, *_), rays = _hits(oracle, c1, 160, 120, 2, "fp32")
    same = gp == rp
    # FP32 ambiguity band: rays that graze a silhouette within FP32 resolution
    assert same.mean() > 0.9995, f"{(~same).sum()} of {len(same)} prim ids differ"
    hit = same & (rp >= 0)
    rel = np.abs(gt[hit] - rt[hit]) / np.maximum(np.abs(rt[hit]), 1e-30)
    assert rel.max() < 1e-5


def test_occluded_fp64_exact(oracle, c1):
    rng = np.random.default_rng(7)
    n = 20000
    o = np.stack([rng.uniform(-12, 12, n), rng.uniform(0.01, 4, n), rng.uniform(-12, 12, n)], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rs, _ = _ref_and_cam(oracle, c1, 32, 24)
    want = rs.occluded(o, d, 1e-3, 1e30)
    with mt.GpuScene(c1, precision="fp64") as g:
        got = g.occluded(o, d, 1e-3, 1e30)
    assert np.array_equal(got, want)
    assert 0.05 < want.mean() < 0.95


def test_pathtrace_fp64_bytes_exact(oracle, c1):
    w, h, spp, depth = 160, 120, 4, 5
    rs, cam = _ref_and_cam(oracle, c1, w, h)
    want = rs.pathtrace_render(w, h, spp, depth)
    with mt.GpuScene(c1, precision="fp64") as g:
        got = g.pathtrace(cam, w, h, spp, depth)
    diff = got.astype(int) - want.astype(int)
    assert (diff == 0).mean() > 0.9999, f"{(diff != 0).sum()} channels differ, max {np.abs(diff).max()}"


def test_whitted_fp64_bytes_exact(oracle, c1):
    w, h, spp, depth = 160, 120, 4, 5
    rs, cam = _ref_and_cam(oracle, c1, w, h)
    want = rs.whitted_render(w, h, spp, depth)
    with mt.GpuScene(c1, precision="fp64") as g:
        got = g.whitted(cam, w, h, spp, depth)
    diff = got.astype(int) - want.astype(int)
    assert (diff == 0).mean() > 0.9999, f"{(diff != 0).sum()} channels differ, max {np.abs(diff).max()}"


def test_whitted_fp32_within_one_level(oracle, c1):
    w, h, spp, depth = 160, 120, 4, 5
    rs, cam = _ref_and_cam(oracle, c1, w, h)
    want = rs.whitted_render(w, h, spp, depth)
    with mt.GpuScene(c1, precision="fp32") as g:
        got = g.whitted(cam, w, h, spp, depth)
    diff = np.abs(got.astype(int) - want.astype(int))
    frac = (diff <= 1).mean()
    assert frac >= 0.999, f"only {frac:.5f} of channels within 1/255"


def test_radiance_fp64_exact(oracle, c1):
    w, h, spp = 64, 48, 1
    rs, cam = _ref_and_cam(oracle, c1, w, h)
    rays = rs.primary_rays(w, h, spp)
    seeds = ((np.arange(len(rays), dtype=np.uint64) * 2654435761) % (2**32)).astype(np.uint32)
    want = rs.radiance(rays[:, :3], rays[:, 3:], 5, seeds)
    with mt.GpuScene(c1, precision="fp64") as g:
        got = g.radiance(rays[:, :3], rays[:, 3:], 5, seeds)
    # Same random stream, same decisions: the only differences left are the
    # last-ulp differences of CUDA's double sin/cos/pow/exp versus glibc's.
    close = np.all(np.abs(got - want) <= 1e-9 * np.abs(want) + 1e-12, axis=1)
    assert close.mean() > 0.998, f"{(~close).sum()} of {len(close)} paths diverge"


def test_whitted_trace_fp64_exact(oracle, c1):
    w, h, spp = 48, 36, 1
    rs, cam = _ref_and_cam(oracle, c1, w, h)
    rays = rs.primary_rays(w, h, spp, "whitted")
    seeds = ((np.arange(len(rays), dtype=np.uint64) * 2246822519) % (2**32)).astype(np.uint32)
    want = rs.radiance(rays[:, :3], rays[:, 3:], 5, seeds, mode="whitted")
    with mt.GpuScene(c1, precision="fp64") as g:
        got = g.radiance(rays[:, :3], rays[:, 3:], 5, seeds, mode="whitted")
    close = np.all(np.abs(got - want) <= 1e-9 * np.abs(want) + 1e-12, axis=1)
    assert close.mean() > 0.998, f"{(~close).sum()} of {len(close)} Whitted samples diverge"


def test_default_scene_whitted_matches_reference_bytes(oracle, mtlib):
    """The SHA-256-pinned Whitted frame (320x180, 4 spp, depth 4) of the
    reference's built-in default scene (plane, water box, 121 tapered
    cylinders, 1163 spheres), rendered through the reference-side binding."""
    rs = oracle.RefScene.from_text(None, 320, 180)
    want = rs.whitted_render(320, 180, 4, 4)
    desc, cam = rs.export()
    with mt.GpuScene(desc, precision="fp64") as g:
        got = g.whitted(cam, 320, 180, 4, 4)
    diff = got.astype(int) - want.astype(int)
    assert (diff == 0).mean() > 0.9999, f"{(diff != 0).sum()} channels differ, max {np.abs(diff).max()}"


def test_torus_field_hits_fp64_exact(oracle, mtlib):
    d = scenes.torus_field_scene(n_instances=256)
    (gp, gt, *_), (rp, rt, *_), _ = _hits(oracle, d, 96, 54, 1, "fp64")
    assert np.array_equal(gp, rp)
    assert np.array_equal(gt, rt)
    assert (rp > 0).mean() > 0.05


def test_error_codes(mtlib, c1):
    with mt.GpuScene(c1) as g:
        cam = c1.make_camera(8, 8)
        buf = np.zeros((8, 8, 3), np.uint8)
        assert mt.pathtrace_render(None, cam, 8, 8, 1, 1, buf) == 1
        assert mt.pathtrace_render(g, None, 8, 8, 1, 1, buf) == 1
        assert mt.pathtrace_render(g, cam, 8, 8, 1, 1, None) == 1
        assert mt.pathtrace_render(g, cam, 0, 8, 1, 1, buf) == 2
        assert mt.pathtrace_render(g, cam, 8, -1, 1, 1, buf) == 2
        assert mt.pathtrace_render(g, cam, 8, 8, 0, 1, buf) == 3
        assert mt.pathtrace_render(g, cam, 8, 8, 1, -1, buf) == 3
        assert mt.render_image_ex(g, cam, 8, 8, None, buf) == 1
        assert mt.render_image_ex(g, cam, 8, 8, dict(samples_per_pixel=0, max_depth=1), buf) == 3
        assert mt.pathtrace_render(g, cam, 8, 8, 1, 1, buf) == 0
