"""Monte-Carlo parity of the path tracer (the north-star criterion).

A 16,384-spp FP64 image of the 64-sphere scene is the converged reference. It
is first checked against the CPU oracle (the reference's own
pathtrace_radiance) on disjoint samples: within 3 standard errors per pixel.
Then the production FP32 wavefront image at 256 spp must lie within 3 of its
own standard errors of the converged image per pixel, and its RMSE against the
converged image must fall as 1/sqrt(spp). Standard errors come from 16
independent sample windows.
"""
import numpy as np
import pytest
import torch

import marmel_trace_b200 as mt
from marmel_trace_b200 import _capi, scenes

pytestmark = pytest.mark.gpu

W, H, DEPTH = 64, 48, 5


def _windows(g, cam, s_base, n_windows, spp):
    """Per-window mean images (n_windows, H, W, 3)."""
    acc = torch.zeros((H, W, 3), dtype=torch.float32, device="cuda")
    out = []
    for k in range(n_windows):
        s0 = s_base + k * spp
        rc = g.lib.mt_render_accumulate_device(g.h, cam.ref, W, H, s0, s0 + spp, DEPTH, 0, acc.data_ptr(), 0, None)
        _capi.check(rc, "mt_render_accumulate_device")
        torch.cuda.synchronize()
        out.append(acc.cpu().numpy().astype(np.float64) / spp)
    return np.stack(out)


def _within_3se(est, se, truth, floor=1e-6):
    z = np.abs(est - truth) / np.maximum(se, floor)
    return (z <= 3.0).mean(), float(np.median(z))


@pytest.fixture(scope="module")
def converged(mtlib):
    d = scenes.spheres_scene()
    cam = d.make_camera(W, H)
    with mt.GpuScene(d, precision="fp64", integrator="wavefront") as g:
        img = g.linear(cam, W, H, 16384, DEPTH).astype(np.float64)
    return d, cam, img


def test_converged_image_agrees_with_oracle(oracle, converged):
    d, cam, conv = converged
    rs = oracle.RefScene.from_desc(d, cam)
    wins = np.stack([rs.pathtrace_linear(W, H, 64, DEPTH, s0=40000 + 64 * k) for k in range(16)])
    mean = wins.mean(0)
    se = wins.std(0, ddof=1) / np.sqrt(len(wins))
    frac, med = _within_3se(mean, se, conv)
    assert frac >= 0.985, f"only {frac:.4f} of channels within 3 SE (median z {med:.3f})"


def test_fp32_wavefront_within_3se_and_rmse(mtlib, converged):
    d, cam, conv = converged
    with mt.GpuScene(d, precision="fp32", integrator="wavefront") as g:
        wins = _windows(g, cam, 100000, 16, 16)   # 256 spp in 16 windows
    mean = wins.mean(0)
    se = wins.std(0, ddof=1) / np.sqrt(len(wins))
    frac, med = _within_3se(mean, se, conv)
    assert frac >= 0.985, f"only {frac:.4f} of channels within 3 SE (median z {med:.3f})"
    # RMSE against the converged image falls as 1/sqrt(spp)
    rmse16 = float(np.sqrt(np.mean((wins[0] - conv) ** 2)))
    rmse256 = float(np.sqrt(np.mean((mean - conv) ** 2)))
    print(f"RMSE vs 16k-spp converged image: 16 spp {rmse16:.5f}, 256 spp {rmse256:.5f}")
    assert 2.5 < rmse16 / rmse256 < 6.5   # ideal sqrt(16) = 4
