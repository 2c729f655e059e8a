"""Inverse rendering with the path-replay adjoint: recover material and sun
parameters from a target image by gradient descent (Adam).

    python -m marmel_trace_b200.inverse --steps 200

The target is rendered from the scene's true parameters; the start point
perturbs them by N(0, 0.15) and clips to the valid ranges (albedo and
metallic in [0, 1], roughness in [0.01, 1], emissive and sun >= 0). Each step
renders a fresh sample window (so the noise decorrelates between steps),
takes the L2 image loss and its gradient through RenderFunction, and applies
an Adam update. The adjoint replays a different sample window than the one
the loss sees: with the same samples the image and its derivative are
correlated, which biases the gradient of an L2 loss (toward parameters that
lower the image's variance rather than its error). The learning rate follows
a cosine from `lr` down to lr / 20: once the loss reaches its Monte-Carlo
noise floor the gradients of weakly observed parameters (roughness,
metallic) are mostly noise, and Adam's normalised steps would otherwise walk
them at the full rate.

The parameter error is reported per group (albedo, roughness, metallic,
emissive, sun; the absorption parameters do not act on this scene, which has
no medium) over the materials some pixel of the target shows.

Two image-space figures go with it. `loss_at_truth` is the L2 loss of the
true parameters against the target, averaged over fresh windows: the floor
that the Monte-Carlo noise of a `spp` render and of the target set, below
which the loss cannot go. `image_rmse_crn` is the RMS difference between the
image of the start (or final) parameters and the image of the true ones,
both rendered at `target_spp` on the same sample window (common random
numbers), so that most of the noise cancels: it measures how far the
parameters are from reproducing the target, which one view pins down better
than the parameters themselves (the sun radiance and the albedos trade
against each other, and so do metallic and albedo on rough surfaces).
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import scenes
from .adjoint import DiffRenderer, RenderFunction

GROUPS = {"albedo": (0, 3), "roughness": (3, 4), "metallic": (4, 5), "emissive": (5, 8)}


def clip_params(p: torch.Tensor, n_mat: int) -> torch.Tensor:
    per = p[: 8 * n_mat].view(n_mat, 8)
    per[:, 0:3].clamp_(0.0, 1.0)
    per[:, 3].clamp_(0.01, 1.0)
    per[:, 4].clamp_(0.0, 1.0)
    per[:, 5:8].clamp_(min=0.0)
    p[8 * n_mat:].clamp_(min=0.0)
    return p


def group_errors(p: np.ndarray, truth: np.ndarray, n_mat: int, seen: np.ndarray) -> dict:
    """RMS error of each parameter group over the materials in `seen`, and of
    the sun radiance."""
    per_p = p[: 8 * n_mat].reshape(n_mat, 8)[seen]
    per_t = truth[: 8 * n_mat].reshape(n_mat, 8)[seen]
    out = {g: float(np.sqrt(np.mean((per_p[:, a:b] - per_t[:, a:b]) ** 2))) for g, (a, b) in GROUPS.items()}
    out["sun"] = float(np.sqrt(np.mean((p[8 * n_mat: 8 * n_mat + 3] - truth[8 * n_mat: 8 * n_mat + 3]) ** 2)))
    return out


def visible_materials(desc, width: int, height: int, device: int) -> np.ndarray:
    """Materials of the primary hits of the frame (a 1-spp ray cast)."""
    from .api import GpuScene

    cam = desc.make_camera(width, height)
    with GpuScene(desc, precision="fp32", device=device) as g:
        rays = g.primary_rays(cam, width, height, 1)
        _, _, _, _, mat = g.intersect(rays[:, :3], rays[:, 3:], 1e-4, 1e30)
    mats = np.unique(mat[mat >= 0])
    seen = np.zeros(len(desc.materials), bool)
    seen[mats] = True
    return seen


def run(steps: int = 200, width: int = 512, height: int = 512, spp: int = 32, depth: int = 6, lr: float = 0.02,
        seed: int = 4, target_spp: int = 256, log_every: int = 20, device: int = 0) -> dict:
    d = scenes.adjoint_scene(seed=seed)
    n_mat = len(d.materials)
    truth = scenes.material_params(d)
    seen = visible_materials(d, min(width, 256), min(height, 256), device)
    tgt = DiffRenderer(d, width, height, target_spp, depth, device=device)
    target = tgt.render(s0=10_000_000).detach()
    tgt.release()
    r = DiffRenderer(d, width, height, spp, depth, device=device)
    rng = np.random.default_rng(seed + 1000)
    p0 = truth + rng.normal(0.0, 0.15, truth.shape)
    params = clip_params(torch.tensor(p0, dtype=torch.float64, device="cuda"), n_mat).requires_grad_(True)
    start = params.detach().cpu().numpy()
    opt = torch.optim.Adam([params], lr=lr)
    hist = []
    t0 = time.perf_counter()
    for k in range(steps):
        for grp in opt.param_groups:
            grp["lr"] = lr * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * k / max(steps - 1, 1))))
        opt.zero_grad()
        # the loss sees window 2k, the adjoint replays window 2k + 1: an
        # unbiased estimate of the gradient of the expected L2 loss
        img = RenderFunction.apply(params, r, spp * 2 * k, spp * (2 * k + 1))
        loss = ((img - target) ** 2).mean()
        loss.backward()
        opt.step()
        with torch.no_grad():
            clip_params(params, n_mat)
        if k % log_every == 0 or k == steps - 1:
            cur = params.detach().cpu().numpy()
            hist.append({"step": k, "loss": float(loss.detach()),
                         "param_rmse": float(np.sqrt(np.mean((cur - truth) ** 2))),
                         "groups": group_errors(cur, truth, n_mat, seen)})
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    final = params.detach().cpu().numpy()
    # the loss floor: the true parameters against the target on fresh windows
    r.set_params(truth)
    floor = [float(((r.render(s0=spp * (2 * steps + 2 * j)) - target) ** 2).mean()) for j in range(4)]
    r.release()
    # start / final images against the true image on one shared sample window
    ev = DiffRenderer(d, width, height, target_spp, depth, device=device)
    imgs = {}
    for name, p in (("truth", truth), ("start", start), ("last", final)):
        ev.set_params(p)
        imgs[name] = ev.render(s0=20_000_000)
    ev.release()
    crn = {k: float(torch.sqrt(((imgs[k] - imgs["truth"]) ** 2).mean())) for k in ("start", "last")}
    return {"steps": steps, "seconds": dt, "steps_per_s": steps / dt, "history": hist,
            "loss_at_truth": float(np.mean(floor)), "image_rmse_crn": crn,
            "start_param_rmse": float(np.sqrt(np.mean((start - truth) ** 2))),
            "start_groups": group_errors(start, truth, n_mat, seen), "params": len(truth),
            "materials_seen": int(seen.sum()),
            "config": dict(width=width, height=height, spp=spp, depth=depth, lr=lr, seed=seed)}


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--lr", type=float, default=0.02)
    a = ap.parse_args()
    print(json.dumps(run(steps=a.steps, lr=a.lr)))
