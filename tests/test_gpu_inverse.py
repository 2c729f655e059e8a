"""Inverse rendering (the adjoint configuration) end to end: Adam on the
path-replay gradients recovers the hidden material parameters. At a reduced
frame (128x128, 16 spp) 20 steps must lower the image loss and the error of
the directly observed parameters (albedo and emission of the materials the
frame shows) from the perturbed start."""
import numpy as np
import pytest

from marmel_trace_b200 import inverse

pytestmark = pytest.mark.gpu


def test_twenty_adam_steps_lower_loss_and_parameter_error(mtlib):
    res = inverse.run(steps=20, width=128, height=128, spp=16, depth=6, lr=0.02, target_spp=256, log_every=1)
    hist = res["history"]
    first = np.mean([h["loss"] for h in hist[:3]])
    last = np.mean([h["loss"] for h in hist[-3:]])
    g0, g1 = res["start_groups"], hist[-1]["groups"]
    print(f"loss {first:.5f} -> {last:.5f}; over {res['materials_seen']} visible materials: "
          + ", ".join(f"{k} {g0[k]:.4f} -> {g1[k]:.4f}" for k in g0) + f"; {res['steps_per_s']:.1f} steps/s")
    assert last < 0.8 * first
    # the directly observed parameters move toward the truth
    assert g1["albedo"] < g0["albedo"]
    assert g1["emissive"] < g0["emissive"]
