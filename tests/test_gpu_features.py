"""Scene content beyond the benchmark configurations, against the oracle:
every texture kind (procedural, UV checker, image; hit (u, v) on spheres,
planes, boxes, cylinders and triangles with and without vertex UVs), fog
(analytic height fog with noise; marched with sun shadow segments), volumetric
clouds (sky and sun transmittance) and the marched underwater segment.

FP64 device images must match the reference's bytes (the only differences
are last-ulp ones between CUDA's and glibc's exp / pow / sin / atan2, which
move a channel across a rounding edge at most rarely). The FP32 wavefront
integrator must equal the FP32 megakernel bit for bit, as on every other
scene, and stay within one level of the reference on most channels.
"""
import numpy as np
import pytest

import marmel_trace_b200 as mt
from marmel_trace_b200 import scenes

pytestmark = pytest.mark.gpu

W, H = 96, 72


def _mismatch(a, b):
    return (a.astype(int) != b.astype(int)).mean()


def _close(got, want, frac=0.999):
    diff = got.astype(int) - want.astype(int)
    same = (diff == 0).mean()
    assert same > frac, f"{(diff != 0).sum()} of {diff.size} channels differ, max {np.abs(diff).max()}"


def _case(oracle, fog, clouds):
    d = scenes.feature_scene(fog=fog, clouds=clouds)
    cam = d.make_camera(W, H)
    return d, cam, oracle.RefScene.from_desc(d, cam)


CASES = [(None, False), ("analytic", False), ("marched", False), (None, True), ("marched", True)]


@pytest.mark.parametrize("fog,clouds", CASES)
@pytest.mark.parametrize("integrator", ["megakernel", "wavefront"])
def test_pathtrace_fp64_matches_reference(oracle, mtlib, fog, clouds, integrator):
    d, cam, rs = _case(oracle, fog, clouds)
    want = rs.pathtrace_render(W, H, 2, 4)
    with mt.GpuScene(d, precision="fp64", integrator=integrator) as g:
        got = g.pathtrace(cam, W, H, 2, 4)
    _close(got, want)


@pytest.mark.parametrize("fog,clouds", [(None, False), ("analytic", False), (None, True)])
def test_whitted_fp64_matches_reference(oracle, mtlib, fog, clouds):
    d, cam, rs = _case(oracle, fog, clouds)
    want = rs.whitted_render(W, H, 2, 4)
    with mt.GpuScene(d, precision="fp64") as g:
        got = g.whitted(cam, W, H, 2, 4)
    _close(got, want)


def test_features_change_the_image(oracle, mtlib):
    """Textures, fog and clouds each change the image (the parity above is not
    vacuous)."""
    cam = scenes.feature_scene().make_camera(W, H)
    plain = scenes.feature_scene()
    plain.materials["texture_kind"] = 0
    imgs = {}
    for name, d in (("plain", plain), ("tex", scenes.feature_scene()),
                    ("fog", scenes.feature_scene(fog="analytic")), ("clouds", scenes.feature_scene(clouds=True))):
        with mt.GpuScene(d, precision="fp64") as g:
            imgs[name] = g.whitted(cam, W, H, 1, 2)
    assert _mismatch(imgs["plain"], imgs["tex"]) > 0.05
    assert _mismatch(imgs["tex"], imgs["fog"]) > 0.05
    assert _mismatch(imgs["tex"], imgs["clouds"]) > 0.01


@pytest.mark.parametrize("fog,clouds", [("marched", True), ("analytic", False)])
def test_fp32_wavefront_equals_megakernel(oracle, mtlib, fog, clouds):
    d = scenes.feature_scene(fog=fog, clouds=clouds)
    cam = d.make_camera(W, H)
    with mt.GpuScene(d, precision="fp32", integrator="megakernel") as g:
        mk = g.pathtrace(cam, W, H, 4, 4)
    with mt.GpuScene(d, precision="fp32", integrator="wavefront") as g:
        wf = g.pathtrace(cam, W, H, 4, 4)
    assert np.array_equal(mk, wf)


def test_fp32_close_to_reference(oracle, mtlib):
    d, cam, rs = _case(oracle, "analytic", True)
    want = rs.whitted_render(W, H, 2, 3)
    with mt.GpuScene(d, precision="fp32") as g:
        got = g.whitted(cam, W, H, 2, 3)
    diff = np.abs(got.astype(int) - want.astype(int))
    assert (diff <= 1).mean() > 0.995, f"{(diff > 1).sum()} channels differ by more than one level"


def test_marched_water_matches_reference(oracle, mtlib):
    """fog.shadow_steps > 0 marches water media with sun shadow segments
    (pt_water_segment) even without fog density. The water scene's FP64 paths
    already diverge from the reference on a few pixels (near-critical-angle
    refraction amplifies last-ulp libm differences in the wave normal); the
    marched render may differ no more than the plain one does."""
    plain = scenes.water_scene()
    marched = scenes.water_scene()
    marched.fog = dict(shadow_steps=5)
    cam = plain.make_camera(W, H)
    want = {k: oracle.RefScene.from_desc(d, cam).pathtrace_render(W, H, 2, 5) for k, d in
            (("plain", plain), ("marched", marched))}
    assert _mismatch(want["plain"], want["marched"]) > 0.01  # marching changes the image
    for integrator in ("megakernel", "wavefront"):
        miss = {}
        for k, d in (("plain", plain), ("marched", marched)):
            with mt.GpuScene(d, precision="fp64", integrator=integrator) as g:
                miss[k] = _mismatch(g.pathtrace(cam, W, H, 2, 5), want[k])
        assert miss["marched"] <= max(2.0 * miss["plain"], 0.003), (integrator, miss)


def test_adjoint_rejects_the_new_content(mtlib):
    import torch

    from marmel_trace_b200 import _capi

    d = scenes.feature_scene(fog="analytic")
    cam = d.make_camera(16, 16)
    with mt.GpuScene(d, precision="fp32", integrator="wavefront") as g:
        dl = torch.zeros((16, 16, 3), dtype=torch.float32, device="cuda")
        grad = torch.zeros(g.lib.mt_scene_param_count(g.h), dtype=torch.float64, device="cuda")
        rc = g.lib.mt_adjoint_backward_device(g.h, cam.ref, 16, 16, 0, 1, 2, dl.data_ptr(), grad.data_ptr(), 0, None)
        assert rc == _capi.MT_ERR_UNSUPPORTED


def test_glass_scene_fp64_matches_reference(oracle, mtlib):
    """A mixed scene with glass tori and spheres: shadow segments pass
    through transparent hits (pt_occluded_segment's chain). The wavefront runs
    the chain link by link across launches (k_wf_shadow, k_wf_shadow_link),
    the megakernel in one loop: their FP64 bytes are equal. Against the
    reference both differ in the same handful of channels (22 of 20,736 at
    this size), paths through glass where, as with water near the critical
    angle, refraction magnifies last-ulp differences."""
    d = scenes.mixed_scene(np.random.default_rng(11), 4000)
    assert ((d.materials["transparency"] > 0.8) | (d.materials["is_water"] != 0)).any()
    cam = d.make_camera(W, H)
    rs = oracle.RefScene.from_desc(d, cam)
    want = rs.pathtrace_render(W, H, 4, 6)
    rs.free()
    got = {}
    for integrator in ("megakernel", "wavefront"):
        with mt.GpuScene(d, precision="fp64", integrator=integrator) as g:
            got[integrator] = g.pathtrace(cam, W, H, 4, 6)
    assert np.array_equal(got["megakernel"], got["wavefront"])
    _close(got["wavefront"], want, frac=0.998)
