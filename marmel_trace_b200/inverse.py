"""Inverse rendering with the path-replay adjoint: recover material and sun
parameters from a target image by gradient descent (Adam).

    python -m marmel_trace_b200.inverse --steps 200

The target is rendered from the scene's true parameters; the start point
perturbs them by N(0, 0.15) and clips to the valid ranges (albedo and
metallic in [0, 1], roughness in [0.01, 1], emissive and sun >= 0). Each step
renders a fresh sample window (so the noise decorrelates between steps),
takes the L2 image loss and its gradient through RenderFunction, and applies
an Adam update.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import scenes
from .adjoint import DiffRenderer, RenderFunction


def clip_params(p: torch.Tensor, n_mat: int) -> torch.Tensor:
    per = p[: 8 * n_mat].view(n_mat, 8)
    per[:, 0:3].clamp_(0.0, 1.0)
    per[:, 3].clamp_(0.01, 1.0)
    per[:, 4].clamp_(0.0, 1.0)
    per[:, 5:8].clamp_(min=0.0)
    p[8 * n_mat:].clamp_(min=0.0)
    return p


def run(steps: int = 200, width: int = 512, height: int = 512, spp: int = 32, depth: int = 6, lr: float = 0.02,
        seed: int = 4, target_spp: int = 256, log_every: int = 20, device: int = 0) -> dict:
    d = scenes.adjoint_scene(seed=seed)
    n_mat = len(d.materials)
    truth = scenes.material_params(d)
    tgt = DiffRenderer(d, width, height, target_spp, depth, device=device)
    target = tgt.render(s0=10_000_000).detach()
    tgt.release()
    r = DiffRenderer(d, width, height, spp, depth, device=device)
    rng = np.random.default_rng(seed + 1000)
    p0 = truth + rng.normal(0.0, 0.15, truth.shape)
    params = clip_params(torch.tensor(p0, dtype=torch.float64, device="cuda"), n_mat).requires_grad_(True)
    opt = torch.optim.Adam([params], lr=lr)
    hist = []
    t0 = time.perf_counter()
    for k in range(steps):
        opt.zero_grad()
        img = RenderFunction.apply(params, r, spp * k)
        loss = ((img - target) ** 2).mean()
        loss.backward()
        opt.step()
        with torch.no_grad():
            clip_params(params, n_mat)
        if k % log_every == 0 or k == steps - 1:
            err = float(np.sqrt(np.mean((params.detach().cpu().numpy() - truth) ** 2)))
            hist.append({"step": k, "loss": float(loss), "param_rmse": err})
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    r.release()
    return {"steps": steps, "seconds": dt, "steps_per_s": steps / dt, "history": hist,
            "start_param_rmse": float(np.sqrt(np.mean((p0 - truth) ** 2))), "params": len(truth),
            "config": dict(width=width, height=height, spp=spp, depth=depth, lr=lr, seed=seed)}


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--lr", type=float, default=0.02)
    a = ap.parse_args()
    print(json.dumps(run(steps=a.steps, lr=a.lr)))
