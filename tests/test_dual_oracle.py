"""The dual-number oracle of the adjoint (oracle/ref_dual.cpp), pinned on the
CPU before the GPU adjoint is compared with it.

* Its value part is the reference's path tracer: every sample equals the
  reference's pathtrace_radiance bit for bit, and so does every restated BSDF
  weight (the oracle counts mismatches).
* Its tangents equal central finite differences of the reference renderer
  itself, with common random numbers, for the parameters the image is linear
  in (emissive, sun radiance) and for Lambert albedo where no roulette acts
  (depth <= 2): there the detached-sampling derivative is the exact one.
"""
import numpy as np
import pytest

from marmel_trace_b200 import scenes


def _ref_scene(oracle, desc, w, h):
    return oracle.RefScene.from_desc(desc, desc.make_camera(w, h))


def _ref_loss(oracle, desc, params, w, h, spp, depth, adj):
    r = _ref_scene(oracle, scenes.with_params(desc, params), w, h)
    img = r.pathtrace_linear(w, h, spp, depth, threads=1)
    r.free()
    return float((img * adj.astype(np.float64)).sum())


def _fd(oracle, desc, idx, w, h, spp, depth, adj, rel=1e-3):
    p0 = scenes.material_params(desc)
    out = []
    for i in idx:
        hp = rel * max(1.0, abs(p0[i]))
        p = p0.copy()
        p[i] += hp
        lp = _ref_loss(oracle, desc, p, w, h, spp, depth, adj)
        p[i] -= 2 * hp
        lm = _ref_loss(oracle, desc, p, w, h, spp, depth, adj)
        out.append((lp - lm) / (2 * hp))
    return np.array(out)


def _adj(h, w, seed):
    return np.random.default_rng(seed).uniform(0.5, 1.5, (h, w, 3)).astype(np.float32)


@pytest.mark.parametrize("which", ["pbr", "legacy"])
def test_dual_value_part_is_the_reference(oracle, which):
    d = (scenes.adjoint_scene(n_spheres=16, n_materials=8, n_emissive=2) if which == "pbr"
         else scenes.spheres_scene(n_spheres=24))
    W, H, SPP, DEPTH = 16, 12, 4, 6
    r = _ref_scene(oracle, d, W, H)
    g, vs, mismatches = r.dual_grad(W, H, 0, SPP, DEPTH, _adj(H, W, 0), idx=[0])
    assert mismatches == 0
    assert np.array_equal(vs / SPP, r.pathtrace_linear(W, H, SPP, DEPTH, threads=1))
    r.free()


def test_dual_matches_fd_for_linear_params(oracle):
    d = scenes.adjoint_scene(n_spheres=16, n_materials=8, n_emissive=2)
    W, H, SPP, DEPTH = 16, 12, 4, 4
    adj = _adj(H, W, 1)
    M = len(d.materials)
    em = [8 * m + 5 + c for m in range(M) if np.any(d.materials[m]["emissive"] > 0) for c in range(3)]
    idx = em + [8 * M, 8 * M + 1, 8 * M + 2]
    r = _ref_scene(oracle, d, W, H)
    g, _, mm = r.dual_grad(W, H, 0, SPP, DEPTH, adj, idx=idx)
    r.free()
    assert mm == 0
    fd = _fd(oracle, d, idx, W, H, SPP, DEPTH, adj)
    assert np.all(np.abs(fd) > 1e-6)
    assert np.allclose(g, fd, rtol=1e-7, atol=1e-10), np.c_[g, fd]


def test_dual_matches_fd_for_lambert_albedo(oracle):
    d = scenes.spheres_scene(n_spheres=24)
    W, H, SPP, DEPTH = 16, 12, 4, 2
    adj = _adj(H, W, 2)
    lam = [m for m in range(len(d.materials)) if not d.materials[m]["pbr"] and d.materials[m]["transparency"] == 0]
    idx = [8 * m + c for m in lam[:5] for c in range(3)]
    r = _ref_scene(oracle, d, W, H)
    g, _, mm = r.dual_grad(W, H, 0, SPP, DEPTH, adj, idx=idx)
    r.free()
    assert mm == 0
    fd = _fd(oracle, d, idx, W, H, SPP, DEPTH, adj)
    assert (np.abs(fd) > 1e-6).sum() >= 6
    assert np.allclose(g, fd, rtol=1e-7, atol=1e-10), np.c_[g, fd]


def test_dual_matches_fd_for_absorption(oracle):
    """Beer-Lambert absorption of the water: media on refracted paths and
    shadow rays through the surface. Depth 2 keeps roulette out, so the
    detached derivative is the exact one."""
    d = scenes.water_scene()
    W, H, SPP, DEPTH = 16, 12, 4, 2
    adj = _adj(H, W, 3)
    M = len(d.materials)
    idx = [8 * M + 3 + 3 * 1 + c for c in range(3)]  # the water material's absorption
    r = _ref_scene(oracle, d, W, H)
    g, _, mm = r.dual_grad(W, H, 0, SPP, DEPTH, adj, idx=idx)
    r.free()
    assert mm == 0
    fd = _fd(oracle, d, idx, W, H, SPP, DEPTH, adj, rel=1e-4)
    assert np.all(np.abs(fd) > 1e-6)
    assert np.allclose(g, fd, rtol=1e-5, atol=1e-9), np.c_[g, fd]
