"""Adaptive Whitted refinement (render_image_adaptive, src/render.c:1128-1500)
on the GPU against the oracle, through mt_render_image_ex.

FP64: the per-pixel sums, the relative-error test and the resolve are the
reference's double arithmetic, so the bytes (and hence every refinement
decision) match the reference exactly; the drop-in CLI reproduces the
reference's SHA-256 pin of its adaptive default. FP32: a sample near the
refinement threshold can flip a pixel's pass count, so the bytes are compared
with a tolerance.
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import marmel_trace_b200 as mt
from marmel_trace_b200 import api, scenes

pytestmark = pytest.mark.gpu

ADAPTIVE_PIN = "419d5d72ff00c51c794509f8dbece04dc67ff0ff8109e23f70cb516192890496"


def _gpu(d, cam, w, h, params, precision):
    out = np.zeros((h, w, 3), np.uint8)
    with mt.GpuScene(d, precision=precision) as g:
        rc = api.render_image_ex(g, cam, w, h, params, out)
    assert rc == 0
    return out


@pytest.mark.parametrize("params", [dict(samples_per_pixel=4, max_depth=5, adaptive=1),
                                    dict(samples_per_pixel=2, max_depth=4, adaptive=1, adaptive_max_spp=9,
                                         adaptive_tau=0.01),
                                    dict(samples_per_pixel=1, max_depth=3, adaptive=1, adaptive_max_spp=5)])
def test_adaptive_fp64_bytes_match_reference(oracle, mtlib, params):
    d = scenes.spheres_scene()
    w, h = 128, 96
    cam = d.make_camera(w, h)
    rs = oracle.RefScene.from_desc(d, cam)
    want = rs.render_image_ex(w, h, params["samples_per_pixel"], params["max_depth"], 1,
                              params.get("adaptive_max_spp", 0), params.get("adaptive_tau", 0.0))
    rs.free()
    got = _gpu(d, cam, w, h, params, "fp64")
    diff = got.astype(int) - want.astype(int)
    assert (diff == 0).mean() > 0.9999, f"{(diff != 0).sum()} channels differ, max {np.abs(diff).max()}"


def test_adaptive_fp32_close_to_reference(oracle, mtlib):
    d = scenes.spheres_scene()
    w, h = 160, 120
    params = dict(samples_per_pixel=4, max_depth=5, adaptive=1)
    cam = d.make_camera(w, h)
    rs = oracle.RefScene.from_desc(d, cam)
    want = rs.render_image_ex(w, h, 4, 5)
    rs.free()
    got = _gpu(d, cam, w, h, params, "fp32")
    diff = np.abs(got.astype(int) - want.astype(int))
    assert (diff <= 1).mean() >= 0.995, f"only {(diff <= 1).mean():.5f} of channels within 1/255"


def test_adaptive_refines_more_than_fixed(mtlib):
    """The adaptive image spends extra samples: with tau tiny and a cap of
    4 x n0, every pixel not yet converged takes the extra passes, so the
    result differs from the fixed-spp image."""
    d = scenes.spheres_scene()
    w, h = 64, 48
    cam = d.make_camera(w, h)
    fixed = _gpu(d, cam, w, h, dict(samples_per_pixel=2, max_depth=4), "fp64")
    adapt = _gpu(d, cam, w, h, dict(samples_per_pixel=2, max_depth=4, adaptive=1, adaptive_tau=1e-6), "fp64")
    assert (fixed != adapt).any()


def test_gpu_cli_reproduces_adaptive_pin(oracle, mtlib, tmp_path):
    exe = oracle.HERE / "_ref" / "raytracer_gpu"
    if not exe.exists():
        pytest.skip(f"{exe} not built")
    out = tmp_path / "adaptive.bmp"
    env = dict(os.environ, RAYTRACER_NO_PROGRESS="1", MT_PRECISION="fp64")
    subprocess.run([str(exe), "--no-pathtrace", "--width", "160", "--height", "90", "--samples", "4", "--depth", "4",
                    "--out", str(out)], check=True, env=env, stdout=subprocess.DEVNULL)
    assert hashlib.sha256(out.read_bytes()).hexdigest() == ADAPTIVE_PIN
