"""Differentiable path tracing on top of the C ABI's forward/backward pair.

`DiffRenderer` holds a device scene and a camera; `render(params)` is the
forward (the linear mean image over a sample window, mt_render_accumulate_device)
and `backward(dL_dimage)` the path-replay adjoint (mt_adjoint_backward_device).
`RenderFunction` wraps the pair in the torch.autograd.Function contract:
forward saves nothing but the sample window -- the backward replays every path
from its random stream instead of storing vertices.

Parameter layout (mt_scene_param_count = 11 * materials + 3): per material
albedo rgb, roughness, metallic, emissive rgb; then the sun radiance rgb; then
per material the Beer-Lambert absorption rgb. Scenes with fog, textures,
volumetric clouds or marched media are rejected (MT_ERR_UNSUPPORTED).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _capi
from .api import GpuScene, SceneDesc


class DiffRenderer:
    def __init__(self, desc: SceneDesc, width: int, height: int, spp: int, depth: int, precision: str = "fp32",
                 integrator: str = "wavefront", **opts):
        self.scene = GpuScene(desc, precision=precision, integrator=integrator, **opts)
        self.lib = self.scene.lib
        self.cam = desc.make_camera(width, height)
        self.w, self.h, self.spp, self.depth = width, height, spp, depth
        self.n_params = self.lib.mt_scene_param_count(self.scene.h)

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float64)
        _capi.check(self.lib.mt_scene_get_material_params(self.scene.h, out.ctypes.data, self.n_params), "get_params")
        return out

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(np.asarray(params, np.float64).reshape(-1))
        _capi.check(self.lib.mt_scene_set_material_params(self.scene.h, p.ctypes.data, len(p)), "set_params")

    def render(self, s0: int = 0) -> torch.Tensor:
        """Linear mean image (h, w, 3) over samples [s0, s0 + spp), on the GPU."""
        out = torch.zeros((self.h, self.w, 3), dtype=torch.float32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rc = self.lib.mt_render_accumulate_device(self.scene.h, self.cam.ref, self.w, self.h, s0, s0 + self.spp,
                                                  self.depth, 0, out.data_ptr(), 0, stream)
        _capi.check(rc, "mt_render_accumulate_device")
        return out / self.spp

    def backward(self, dL_dimage: torch.Tensor, s0: int = 0) -> torch.Tensor:
        """dL/dparams (float64, on the GPU) for the image rendered at window s0."""
        g = torch.zeros(self.n_params, dtype=torch.float64, device="cuda")
        a = dL_dimage.detach().to(device="cuda", dtype=torch.float32).contiguous()
        stream = torch.cuda.current_stream().cuda_stream
        rc = self.lib.mt_adjoint_backward_device(self.scene.h, self.cam.ref, self.w, self.h, s0, s0 + self.spp,
                                                 self.depth, a.data_ptr(), g.data_ptr(), 0, stream)
        _capi.check(rc, "mt_adjoint_backward_device")
        return g

    def release(self):
        self.scene.release()


class RenderFunction(torch.autograd.Function):
    """image = RenderFunction.apply(params, renderer, s0, s0_replay).

    The forward renders the sample window starting at s0; the backward
    replays the window starting at s0_replay (default: s0). For a loss that is
    not linear in the image (an L2 loss) the two should differ: with the same
    samples the image and its derivative are correlated, and the product in
    dL/dparams = dL/dimage . dimage/dparams is then a biased estimate of the
    gradient of the expected loss."""

    @staticmethod
    def forward(ctx, params: torch.Tensor, renderer: DiffRenderer, s0: int = 0, s0_replay: int | None = None):
        renderer.set_params(params.detach().cpu().numpy())
        ctx.renderer = renderer
        ctx.s0 = s0 if s0_replay is None else s0_replay
        ctx.dtype = params.dtype
        ctx.device = params.device
        return renderer.render(s0)

    @staticmethod
    def backward(ctx, grad_image: torch.Tensor):
        g = ctx.renderer.backward(grad_image, ctx.s0)
        return g.to(device=ctx.device, dtype=ctx.dtype), None, None, None
