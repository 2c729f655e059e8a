"""The oracle and its restatement, pinned before they are trusted.

* The reference compiled by oracle/Makefile reproduces the reference's own
  SHA-256 pins of the Whitted renderer (tests/test_integration_pathtrace.c:99-106
  of the reference; docs/validation_report_pathtrace.md:586).
* oracle/restate.py reproduces the reference's known-answer intersection
  vectors (tests/test_math.c:276-360) and agrees with the compiled reference
  on hashes, cameras, primary rays and nearest hits.
* The reference BVH equals a linear scan (tests/test_math.c:769-831).
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from marmel_trace_b200 import scenes
from marmel_trace_b200._capi import PRIM_DTYPE
from oracle import restate


def _cli_sha(oracle, tmp_path, args):
    out = tmp_path / "img.bmp"
    env = dict(os.environ, RAYTRACER_NO_PROGRESS="1")
    subprocess.run([str(oracle.CLI), *args, "--out", str(out)], check=True, env=env, stdout=subprocess.DEVNULL)
    return hashlib.sha256(out.read_bytes()).hexdigest()


def test_whitted_fixed_sha_pin(oracle, tmp_path):
    sha = _cli_sha(oracle, tmp_path, ["--no-pathtrace", "--no-adaptive", "--width", "320", "--height", "180",
                                      "--samples", "4", "--depth", "4"])
    assert sha == "f9f4551a12c4c73f85c7954ce7e00adebd768798c2471def03df0e97c818ffcb"


def test_whitted_adaptive_sha_pin(oracle, tmp_path):
    sha = _cli_sha(oracle, tmp_path, ["--no-pathtrace", "--width", "160", "--height", "90", "--samples", "4",
                                      "--depth", "4"])
    assert sha == "419d5d72ff00c51c794509f8dbece04dc67ff0ff8109e23f70cb516192890496"


def test_harness_render_image_matches_cli_pin(oracle):
    """render_image through the harness gives the pinned frame's pixels."""
    rs = oracle.RefScene.from_text(None, 320, 180)
    rgb = rs.whitted_render(320, 180, 4, 4)
    # bmp_write (src/bmp.c:38): 54-byte header, bottom-up BGR rows padded to 4 bytes
    row = 320 * 3
    body = b"".join(rgb[y, :, ::-1].tobytes() for y in range(179, -1, -1))
    size = 54 + len(body)
    hdr = b"BM" + size.to_bytes(4, "little") + b"\0\0\0\0" + (54).to_bytes(4, "little")
    hdr += (40).to_bytes(4, "little") + (320).to_bytes(4, "little", signed=True) + (180).to_bytes(4, "little", signed=True)
    hdr += (1).to_bytes(2, "little") + (24).to_bytes(2, "little") + b"\0" * 4 + len(body).to_bytes(4, "little")
    hdr += (2835).to_bytes(4, "little") * 2 + b"\0" * 8
    assert row % 4 == 0
    sha = hashlib.sha256(hdr + body).hexdigest()
    assert sha == "f9f4551a12c4c73f85c7954ce7e00adebd768798c2471def03df0e97c818ffcb"


def test_hash_kat(oracle):
    rng = np.random.default_rng(3)
    a, b, c = (rng.integers(0, 2**32, 2000, dtype=np.uint64) for _ in range(3))
    want = np.array([oracle.pt_hash3(int(x), int(y), int(z)) for x, y, z in zip(a, b, c)], np.uint64)
    assert np.array_equal(restate.hash3(a, b, c), want)
    r = np.array([oracle.pt_rand01(int(x), int(y), int(z)) for x, y, z in zip(a[:200], b[:200], c[:200])])
    assert np.array_equal(restate.rand01(a[:200], b[:200], c[:200]), r)


def test_to_byte_kat(oracle):
    xs = np.concatenate([np.linspace(-0.5, 1.5, 4001), [np.nan, np.inf, -np.inf, 1e-300]])
    want = np.array([oracle.to_byte(float(x)) for x in xs], np.uint8)
    assert np.array_equal(restate.to_byte(xs), want)


def _one(kind, v, mat=0):
    p = np.zeros(1, PRIM_DTYPE)
    p["kind"] = kind
    p["material"] = mat
    p["v"][0, : len(v)] = v
    return p


def test_sphere_kats():
    """tests/test_math.c:276-332 of the reference."""
    c, r = (0.0, 0.0, -5.0), 1.0
    O = lambda *v: np.array([v], np.float64)
    assert restate.sphere_t(c, r, O(0, 0, 0), O(0, 0, -1), 1e-4, 1e30)[0] == 4.0
    assert np.isnan(restate.sphere_t(c, r, O(0, 0, 0), O(0, 1, 0), 1e-4, 1e30)[0])
    assert restate.sphere_t(c, r, O(0, 0, -5), O(0, 0, -1), 1e-4, 1e30)[0] == 1.0
    assert abs(restate.sphere_t(c, r, O(1, 0, 0), O(0, 0, -1), 1e-4, 1e30)[0] - 5.0) < 1e-9
    assert np.isnan(restate.sphere_t(c, r, O(0, 0, 0), O(0, 0, -1), 1e-4, 3.0)[0])
    assert np.isnan(restate.sphere_t(c, r, O(0, 0, 0), O(0, 0, -1), 4.5, 5.5)[0])
    assert restate.sphere_t(c, r, O(0, 0, 0), O(0, 0, -1), 1e-4, 4.5)[0] == 4.0
    assert restate.sphere_t(c, r, O(0, 0, 0), O(0, 0, -1), 5.0, 1e30)[0] == 6.0
    assert np.isnan(restate.sphere_t((0, 0, 5.0), 1.0, O(0, 0, 0), O(0, 0, -1), 1e-4, 1e30)[0])


def test_plane_kats():
    """tests/test_math.c:336-360 of the reference."""
    O = lambda *v: np.array([v], np.float64)
    assert restate.plane_t((0, 1, 0), (0, 1, 0), O(0, 5, 0), O(0, -1, 0), 1e-4, 1e30)[0] == 4.0
    assert np.isnan(restate.plane_t((0, 1, 0), (0, 1, 0), O(0, 5, 0), O(1, 0, 0), 1e-4, 1e30)[0])
    assert np.isnan(restate.plane_t((0, 1, 0), (0, 1, 0), O(0, 5, 0), O(0, 1, 0), 1e-4, 1e30)[0])


def test_restatement_matches_reference_camera_and_hits(oracle):
    d = scenes.spheres_scene()
    w, h, spp = 48, 36, 2
    cam = restate.camera_create((0.0, 2.0, -10.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 45.0, w / h)
    import marmel_trace_b200 as mt

    mcam = mt.camera_create((0.0, 2.0, -10.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 45.0, w / h)
    for k in ("position", "lower_left", "horizontal", "vertical"):
        assert tuple(getattr(mcam.c, k)) == cam[k]
    rs = oracle.RefScene.from_desc(d, mcam)
    rays = restate.pt_primary_rays(cam, w, h, spp)
    assert np.array_equal(rays, rs.primary_rays(w, h, spp))
    p_r, t_r = restate.nearest_linear(d.prims, rays[:, :3], rays[:, 3:])
    p_o, t_o, *_ = rs.intersect(rays[:, :3], rays[:, 3:])
    assert np.array_equal(p_r, p_o)
    assert np.array_equal(t_r, t_o)


def test_reference_bvh_equals_linear_scan(oracle):
    """bvh_intersect == geometry_intersect on random rays (test_math.c:769-831)."""
    d = scenes.torus_field_scene(n_instances=64, area=20.0)
    rs = oracle.RefScene.from_desc(d)
    rng = np.random.default_rng(11)
    n = 4000
    o = np.stack([rng.uniform(-12, 12, n), rng.uniform(0.1, 5, n), rng.uniform(-12, 12, n)], 1)
    dd = rng.normal(size=(n, 3))
    dd /= np.linalg.norm(dd, axis=1, keepdims=True)
    p1, t1, *_ = rs.intersect(o, dd)
    p2, t2 = rs.intersect_linear(o, dd)
    assert np.array_equal(p1, p2) and np.array_equal(t1, t2)
    assert (p1 > 0).mean() > 0.05
