"""torch.autograd.Function over the C ABI's differentiable radiative transfer.

ImageRenderer holds one device context (grid uploaded, camera from the
params).  render(m_abs, m_emis) returns the Stokes-I image as a torch tensor
whose backward is the hand-written adjoint kernel (grt_adjoint_image_I):
forward = grt_set_cell_multipliers + grt_init_image_forward_photons
(line-of-sight rays through the fluid) + grt_forward_checkpointed +
grt_get_image_products; backward = the adjoint
sweep from the checkpoints.  Nothing is computed in torch except the loss the
caller builds on the returned image.
"""

from __future__ import annotations

import numpy as np
import torch

from . import lib


class ImageRenderer:
    def __init__(self, params, grid: dict, checkpoint_interval: int = 64, back_distance: float = 60.0):
        self.ctx = lib.Context(params)
        self.ctx.upload_grid(grid)
        self.grid_shape = tuple(grid["r.npy"].shape)
        self.params = params
        self.K = int(checkpoint_interval)
        self.back = float(back_distance)
        self.last_stats = None

    def close(self):
        self.ctx.close()

    def forward_image(self, m_abs: np.ndarray, m_emis: np.ndarray) -> np.ndarray:
        self.ctx.set_cell_multipliers(m_abs, m_emis)
        self.ctx.init_image_forward_photons(self.params.image_nx, self.params.image_ny, self.back)
        self.last_stats = self.ctx.forward_checkpointed(self.K)
        return self.ctx.image_products().image_I.copy()

    def backward_image(self, dL_dI: np.ndarray):
        return self.ctx.adjoint_image_I(dL_dI, self.grid_shape)

    def render(self, m_abs: torch.Tensor, m_emis: torch.Tensor) -> torch.Tensor:
        return _RenderStokesI.apply(m_abs, m_emis, self)


class _RenderStokesI(torch.autograd.Function):
    @staticmethod
    def forward(ctx, m_abs, m_emis, renderer):
        img = renderer.forward_image(m_abs.detach().double().cpu().numpy(),
                                     m_emis.detach().double().cpu().numpy())
        ctx.renderer = renderer
        ctx.dtype = m_abs.dtype
        ctx.device = m_abs.device
        return torch.from_numpy(img).to(device=m_abs.device, dtype=m_abs.dtype)

    @staticmethod
    def backward(ctx, grad_img):
        ga, ge = ctx.renderer.backward_image(grad_img.detach().double().cpu().numpy())
        to = dict(device=ctx.device, dtype=ctx.dtype)
        return torch.from_numpy(ga).to(**to), torch.from_numpy(ge).to(**to), None
