"""Path-replay adjoint against central finite differences with common random
numbers (the same seeds in every render).

Emissive radiance and sun radiance enter the image linearly, and the albedo of
a legacy (Lambert) material does not change any sampling decision when
Russian roulette cannot act (depth <= 2): for these parameters the adjoint
must equal the finite difference up to rounding. PBR albedo / roughness /
metallic move the lobe-selection probability, so the per-sample derivatives
differ (the adjoint holds sampling fixed) and only the expectations agree;
they are compared statistically.
"""
import numpy as np
import pytest
import torch

from marmel_trace_b200 import scenes
from marmel_trace_b200.adjoint import DiffRenderer, RenderFunction

pytestmark = pytest.mark.gpu


def _loss_weights(h, w, seed=0):
    rng = np.random.default_rng(seed)
    return torch.tensor(rng.uniform(0.5, 1.5, (h, w, 3)), dtype=torch.float32, device="cuda")


def _loss(img, wts):
    return float((img.double() * wts.double()).sum())


def _fd(r, p0, idx, h, wts):
    out = []
    for i in idx:
        hp = h * max(1.0, abs(p0[i]))
        p = p0.copy()
        p[i] += hp
        r.set_params(p)
        lp = _loss(r.render(), wts)
        p[i] -= 2 * hp
        r.set_params(p)
        lm = _loss(r.render(), wts)
        out.append((lp - lm) / (2 * hp))
    r.set_params(p0)
    return np.array(out)


def test_param_round_trip(mtlib):
    d = scenes.adjoint_scene(n_spheres=16, n_materials=8, n_emissive=2)
    r = DiffRenderer(d, 16, 12, 1, 2)
    p = r.params()
    assert np.array_equal(p, scenes.material_params(d))
    p2 = p * 0.9
    r.set_params(p2)
    assert np.allclose(r.params(), p2)
    r.release()


def test_linear_params_match_fd_exactly(mtlib):
    d = scenes.adjoint_scene(n_spheres=24, n_materials=8, n_emissive=2)
    W, H, SPP, DEPTH = 32, 24, 8, 4
    r = DiffRenderer(d, W, H, SPP, DEPTH, precision="fp64")
    wts = _loss_weights(H, W)
    p0 = r.params()
    M = len(d.materials)
    em = [8 * m + 5 + c for m in range(M) if np.any(d.materials[m]["emissive"] > 0) for c in range(3)]
    idx = em + [8 * M, 8 * M + 1, 8 * M + 2]
    g = r.backward(wts).cpu().numpy()
    # the image is linear in these parameters, so any step is exact; the
    # tolerance covers the float32 image and float32 gradient accumulation
    fd = _fd(r, p0, idx, 1e-2, wts)
    assert np.allclose(g[idx], fd, rtol=2e-4, atol=1e-7), np.c_[g[idx], fd]
    r.release()


def test_legacy_albedo_matches_fd_exactly(mtlib):
    d = scenes.spheres_scene()   # Lambert, metal (PBR) and glass materials
    W, H, SPP, DEPTH = 32, 24, 8, 2
    r = DiffRenderer(d, W, H, SPP, DEPTH, precision="fp64")
    wts = _loss_weights(H, W, 1)
    p0 = r.params()
    lam = [m for m in range(len(d.materials)) if not d.materials[m]["pbr"] and d.materials[m]["transparency"] == 0]
    idx = [8 * m + c for m in lam[:8] for c in range(3)]
    g = r.backward(wts).cpu().numpy()
    fd = _fd(r, p0, idx, 1e-2, wts)
    mask = np.abs(fd) > 1e-6
    assert mask.sum() >= 6
    assert np.allclose(g[idx], fd, rtol=2e-4, atol=1e-6), np.c_[g[idx], fd]
    r.release()


def test_pbr_params_agree_with_fd_statistically(mtlib):
    d = scenes.adjoint_scene(n_spheres=24, n_materials=6, n_emissive=1)
    W, H, SPP, DEPTH = 32, 24, 256, 3
    r = DiffRenderer(d, W, H, SPP, DEPTH, precision="fp32")
    wts = _loss_weights(H, W, 2)
    p0 = r.params()
    g = r.backward(wts).cpu().numpy()
    # largest-magnitude PBR gradients (albedo, roughness, metallic)
    cand = [8 * m + k for m in range(len(d.materials)) for k in range(5)]
    top = sorted(cand, key=lambda i: -abs(g[i]))[:6]
    fd = _fd(r, p0, top, 2e-2, wts)
    rel = np.abs(g[top] - fd) / np.maximum(np.abs(fd), 1e-9)
    print("adjoint vs FD (PBR):", np.c_[g[top], fd, rel])
    assert np.median(rel) < 0.1, np.c_[g[top], fd, rel]
    r.release()


def test_autograd_function_and_fp32_fp64_agree(mtlib):
    d = scenes.adjoint_scene(n_spheres=16, n_materials=8, n_emissive=2)
    W, H, SPP, DEPTH = 24, 16, 4, 3
    grads = []
    for prec in ("fp32", "fp64"):
        r = DiffRenderer(d, W, H, SPP, DEPTH, precision=prec)
        params = torch.tensor(r.params(), dtype=torch.float64, device="cuda", requires_grad=True)
        img = RenderFunction.apply(params, r, 0)
        loss = (img.double() ** 2).sum()
        loss.backward()
        grads.append(params.grad.cpu().numpy())
        r.release()
    g32, g64 = grads
    big = np.abs(g64) > 1e-3 * np.abs(g64).max()
    assert np.allclose(g32[big], g64[big], rtol=2e-3, atol=1e-6)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("which", ["pbr", "legacy"])
def test_wavefront_adjoint_matches_megakernel(mtlib, prec, which):
    """The wavefront replay (stage kernels, each vertex's gradient deferred
    until its NEE is resolved) and the one-thread-per-pixel replay evaluate
    the same estimator on the same random streams; only the order of the
    float gradient sums differs."""
    if which == "pbr":
        d = scenes.adjoint_scene(n_spheres=24, n_materials=8, n_emissive=2)
    else:
        d = scenes.spheres_scene()  # Lambert, metal and glass: shadow rays pass through glass
    W, H, SPP, DEPTH = 40, 30, 6, 5
    wts = _loss_weights(H, W, 3)
    g = {}
    for integ in ("wavefront", "megakernel"):
        r = DiffRenderer(d, W, H, SPP, DEPTH, precision=prec, integrator=integ)
        g[integ] = r.backward(wts, s0=17).cpu().numpy()
        r.release()
    gw, gm = g["wavefront"], g["megakernel"]
    scale = np.abs(gm).max()
    assert scale > 0
    tol = 1e-5 if prec == "fp64" else 2e-3
    assert np.allclose(gw, gm, rtol=tol, atol=tol * scale), np.c_[gw, gm][np.abs(gw - gm) > tol * scale]


@pytest.mark.parametrize("integ", ["wavefront", "megakernel"])
@pytest.mark.parametrize("which", ["pbr", "legacy", "water"])
def test_adjoint_matches_dual_number_oracle(mtlib, oracle, which, integ):
    """Every parameter's gradient (albedo, roughness, metallic, emissive per
    material, sun radiance) against forward-mode differentiation of the
    reference path tracer (oracle/ref_dual.cpp) on the same samples. FP64
    kernels: the only differences are the float gradient sums and last-ulp
    transcendentals."""
    if which == "pbr":
        d = scenes.adjoint_scene(n_spheres=24, n_materials=8, n_emissive=2)
    elif which == "legacy":
        d = scenes.spheres_scene(n_spheres=24)  # Lambert, metal and glass
    else:
        d = scenes.water_scene()  # media and shadow rays through water: absorption
    W, H, SPP, DEPTH = 24, 16, 4, 5
    adj = np.random.default_rng(5).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    ref = oracle.RefScene.from_desc(d, d.make_camera(W, H))
    r = DiffRenderer(d, W, H, SPP, DEPTH, precision="fp64", integrator=integ)
    # Compare over the pixels whose FP64 image equals the reference's: under
    # water, rays meeting the surface near the critical angle amplify last-ulp
    # differences of cos / sin (water_normal) through the refraction's square
    # root, and a few paths take another course (0.5 % of the water scene's).
    _, value_sum, _ = ref.dual_grad(W, H, 3, 3 + SPP, DEPTH, adj, idx=[0])
    same = np.all(r.render(s0=3).cpu().numpy() == (value_sum / SPP).astype(np.float32), axis=2)
    assert same.mean() > 0.95
    adj = adj * same[:, :, None].astype(np.float32)
    g = r.backward(torch.tensor(adj, device="cuda"), s0=3).cpu().numpy()
    r.release()
    gd, _, mismatches = ref.dual_grad(W, H, 3, 3 + SPP, DEPTH, adj)
    ref.free()
    assert mismatches == 0
    scale = np.abs(gd).max()
    assert (np.abs(gd) > 1e-3 * scale).sum() >= 10
    bad = ~np.isclose(g, gd, rtol=1e-4, atol=1e-6 * scale)
    assert not bad.any(), np.c_[np.nonzero(bad)[0], g[bad], gd[bad]]


def test_fp32_adjoint_close_to_dual_number_oracle(mtlib, oracle):
    d = scenes.adjoint_scene(n_spheres=24, n_materials=8, n_emissive=2)
    W, H, SPP, DEPTH = 32, 24, 8, 6
    adj = np.random.default_rng(6).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    r = DiffRenderer(d, W, H, SPP, DEPTH, precision="fp32")
    g = r.backward(torch.tensor(adj, device="cuda")).cpu().numpy()
    r.release()
    ref = oracle.RefScene.from_desc(d, d.make_camera(W, H))
    gd, _, mismatches = ref.dual_grad(W, H, 0, SPP, DEPTH, adj)
    ref.free()
    assert mismatches == 0
    big = np.abs(gd) > 1e-2 * np.abs(gd).max()
    rel = np.abs(g[big] - gd[big]) / np.abs(gd[big])
    # FP32 rounding can flip an occasional roulette or lobe decision
    assert np.median(rel) < 1e-3 and np.quantile(rel, 0.9) < 2e-2, rel


def test_absorption_gradient_matches_fd(mtlib):
    """The water's absorption gradient against central finite differences of
    the GPU renderer with common random numbers (depth 2: no roulette)."""
    d = scenes.water_scene()
    W, H, SPP, DEPTH = 32, 24, 8, 2
    r = DiffRenderer(d, W, H, SPP, DEPTH, precision="fp64")
    wts = _loss_weights(H, W, 4)
    p0 = r.params()
    M = len(d.materials)
    idx = [8 * M + 3 + 3 + c for c in range(3)]
    g = r.backward(wts).cpu().numpy()
    fd = _fd(r, p0, idx, 1e-2, wts)
    assert np.all(np.abs(fd) > 1e-5)
    # FD of exp(-a t) at h = 1e-2 carries a curvature error of O(h^2 t^2)
    assert np.allclose(g[idx], fd, rtol=2e-3), np.c_[g[idx], fd]
    r.release()
