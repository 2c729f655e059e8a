"""Host-side logic of the GPU library, on CPU: the C-ABI library loads and
exports every declared symbol, the host BVH builder reproduces the reference
builder node for node, the camera matches camera_create bit for bit, and the
seeded scenes round-trip through the reference's scene parser."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import marmel_trace_b200 as mt
from marmel_trace_b200 import _capi, api, scenes

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    text = (ROOT / "include" / "mtgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(mtlib):
    names = _declared()
    assert len(names) >= 20
    lib = C.CDLL(str(_capi.LIB_PATH))
    for n in names:
        assert hasattr(lib, n), f"{n} declared in mtgpu.h but not exported"
    assert set(names) <= set(_capi.SIGNATURES), "ctypes signatures missing for some entry points"
    assert mtlib.mt_version().startswith(b"mtgpu")


def test_no_device_is_an_error_not_a_fallback(mtlib):
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    d = scenes.spheres_scene()
    cd = d.c_desc()
    h = C.c_void_p()
    rc = mtlib.mt_scene_create(C.byref(cd), None, C.byref(h))
    assert rc == _capi.MT_ERR_NO_DEVICE
    assert not h.value


def test_argument_codes_without_scene(mtlib):
    # NULL scene -> reference code 1 before any device work (src/pathtrace.c:1260)
    buf = np.zeros(12, np.uint8)
    cam = mt.camera_create((0, 0, 0), (0, 0, -1), (0, 1, 0), 40, 1.0)
    assert mtlib.mt_pathtrace_render(None, cam.ref, 2, 2, 1, 1, buf.ctypes.data) == 1
    assert mtlib.mt_render_image(None, cam.ref, 2, 2, 1, 1, buf.ctypes.data) == 1


def test_unsupported_content_is_rejected(mtlib):
    """CSG / SDF primitives, bump maps and the star / nebula / galaxy sky
    terms stay off the GPU path (MT_ERR_UNSUPPORTED, no CPU fallback)."""
    for mutate in ("csg", "bump", "stars"):
        dd = scenes.spheres_scene()
        if mutate == "csg":
            dd.prims["kind"][3] = 5
        elif mutate == "bump":
            dd.materials["bump_strength"][1] = 0.5
        cd = dd.c_desc()
        if mutate == "stars":
            cd.sky.star_intensity = 1.0
        h = C.c_void_p()
        assert mtlib.mt_scene_create(C.byref(cd), None, C.byref(h)) == _capi.MT_ERR_UNSUPPORTED


def test_feature_fields_reach_the_descriptor(mtlib):
    """Fog, clouds and image textures travel through mt_scene_desc; an image
    pointer without an image size is an argument error (before any device
    work)."""
    dd = scenes.feature_scene(fog="marched", clouds=True)
    cd = dd.c_desc()
    assert cd.fog_shadow_steps == 6 and cd.sky.cloud_thickness == 40.0 and cd.fog_density > 0
    img = [i for i in range(len(dd.materials)) if dd.materials["texture_kind"][i] == _capi.TEXTURE_IMAGE][0]
    assert dd.materials["texture_rgb"][img] != 0 and dd.materials["texture_width"][img] == 8
    bad = scenes.spheres_scene()
    bad.materials["texture_rgb"][1] = 1  # a pointer with no image size
    h = C.c_void_p()
    assert mtlib.mt_scene_create(C.byref(bad.c_desc()), None, C.byref(h)) == _capi.MT_ERR_INVALID


def test_feature_scene_round_trips_through_the_reference(oracle):
    """The reference scene built from the descriptor exports the same fog,
    cloud, texture and UV fields back (harness + binding)."""
    d = scenes.feature_scene(fog="analytic", clouds=True)
    rs = oracle.RefScene.from_desc(d)
    d2, _ = rs.export()
    assert np.array_equal(d.prims, d2.prims)
    for f in ("texture_kind", "texture_scale", "texture_color_a", "texture_color_b", "albedo"):
        assert np.array_equal(d.materials[f], d2.materials[f]), f
    for k, v in d.fog.items():
        assert np.allclose(d2.fog[k], v), k
    assert d2.sky["cloud_thickness"] == 40.0 and d2.sky["cloud_steps"] == 16
    (i, img), = d.images.items()
    assert np.array_equal(d2.images[i], img)


def test_camera_matches_reference(oracle):
    from marmel_trace_b200._capi import MtCamera

    for args in [((0.0, 2.0, -10.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 45.0, 4 / 3),
                 ((-18.0, 6.0, 22.0), (0.0, 5.0, -20.0), (0.0, 1.0, 0.0), 40.0, 16 / 9),
                 ((0.0, 5.0, 0.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 60.0, 1.0)]:
        mine = mt.camera_create(*args)
        theirs = MtCamera()
        e, t, u = (np.asarray(v, np.float64) for v in args[:3])
        oracle.load().mtref_camera_create(e.ctypes.data, t.ctypes.data, u.ctypes.data, args[3], args[4],
                                          C.byref(theirs))
        for f, _ in MtCamera._fields_:
            a, b = getattr(mine.c, f), getattr(theirs, f)
            assert (list(a) if hasattr(a, "__len__") else a) == (list(b) if hasattr(b, "__len__") else b), f


def _coincident_scene():
    d = scenes.spheres_scene()
    prims = np.concatenate([d.prims, np.repeat(d.prims[5:6], 11)])  # 12 spheres with one centroid
    return api.SceneDesc(prims=prims, materials=d.materials, sky=d.sky)


@pytest.mark.parametrize("name", ["c1", "torus", "default", "coincident"])
def test_host_bvh_equals_reference_builder(oracle, mtlib, name):
    if name == "c1":
        rs_desc = scenes.spheres_scene()
        rs = oracle.RefScene.from_desc(rs_desc)
    elif name == "torus":
        rs_desc = scenes.torus_field_scene(n_instances=128)
        rs = oracle.RefScene.from_desc(rs_desc)
    elif name == "coincident":
        rs_desc = _coincident_scene()
        rs = oracle.RefScene.from_desc(rs_desc)
    else:
        rs = oracle.RefScene.from_text(None, 64, 36)
        rs_desc, _ = rs.export()
    b, l, o, dep = api.bvh_build_host(rs_desc.prims)
    rb, rl, ro, rpl, rdep = rs.bvh_export()
    assert np.array_equal(b, rb)
    assert np.array_equal(l, rl)
    assert np.array_equal(o, ro)
    assert dep == rdep


def test_scene_text_round_trip(oracle):
    for d in (scenes.spheres_scene(), scenes.torus_field_scene(n_instances=16)):
        txt = scenes.to_scene_text(d)
        rs = oracle.RefScene.from_text(txt, 64, 48)
        d2, cam = rs.export()
        assert np.array_equal(d.prims, d2.prims)
        assert np.array_equal(d.materials, d2.materials)
        for k, v in d.sky.items():
            assert np.array_equal(np.asarray(v), np.asarray(d2.sky[k])), k
        mine = d.make_camera(64, 48)
        for f in ("position", "lower_left", "horizontal", "vertical"):
            assert list(getattr(mine.c, f)) == list(getattr(cam.c, f))


def test_emissive_light_list_matches_reference(oracle):
    d = scenes.torus_field_scene(n_instances=8)
    rs = oracle.RefScene.from_desc(d)
    want = rs.lights()
    assert len(want) == 8
    # the library collects the same list on upload (mt_scene_get_info); on CPU,
    # restate the rule from the descriptor (src/scene.c:1384-1426)
    got = [i for i, p in enumerate(d.prims) if p["kind"] == 0 and d.materials[p["material"]]["pbr"]
           and np.any(d.materials[p["material"]]["emissive"] != 0) and p["v"][3] > 0][:8]
    assert list(want) == got
