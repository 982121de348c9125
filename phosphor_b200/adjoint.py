"""Differentiable SPPM for torch: the library's adjoint (phx_adjoint_*) as a torch.autograd.Function.

Parameters θ are laid out like the library's gradient: 4 per material (base colour r, g, b and
roughness), then 3 per light (power r, g, b).  `ParamTable` converts between θ and the scene's
phx_material / phx_light tables; `render` renders an image for θ whose backward pass is the
library's hand-written adjoint (gather adjoint + camera and photon paths replayed from their RNG
seeds).  The gradient is that of the frozen-path estimator described in include/phx.h.
"""
from __future__ import annotations

import numpy as np
import torch

from .renderer import Renderer


class ParamTable:
    """θ <-> (materials, lights) for one scene; other material and light fields stay as given."""

    def __init__(self, materials: np.ndarray, lights: np.ndarray):
        self.materials = np.array(materials, copy=True)
        self.lights = np.array(lights, copy=True)
        self.n_mat = len(self.materials)
        self.n_lights = len(self.lights)

    @property
    def size(self) -> int:
        return 4 * self.n_mat + 3 * self.n_lights

    def vector(self) -> np.ndarray:
        th = np.empty(self.size, dtype=np.float32)
        m = th[:4 * self.n_mat].reshape(self.n_mat, 4)
        b = self.materials["base_color"]
        m[:, 0], m[:, 1], m[:, 2] = b["x"], b["y"], b["z"]
        m[:, 3] = self.materials["roughness"]
        lp = th[4 * self.n_mat:].reshape(self.n_lights, 3)
        p = self.lights["power"]
        lp[:, 0], lp[:, 1], lp[:, 2] = p["x"], p["y"], p["z"]
        return th

    def tables(self, theta) -> tuple[np.ndarray, np.ndarray]:
        th = np.asarray(theta, dtype=np.float32).reshape(-1)
        if th.size != self.size:
            raise ValueError(f"theta has {th.size} entries, expected {self.size}")
        mats = self.materials.copy()
        lts = self.lights.copy()
        m = th[:4 * self.n_mat].reshape(self.n_mat, 4)
        mats["base_color"]["x"], mats["base_color"]["y"], mats["base_color"]["z"] = m[:, 0], m[:, 1], m[:, 2]
        mats["roughness"] = m[:, 3]
        lp = th[4 * self.n_mat:].reshape(self.n_lights, 3)
        if self.n_lights:
            lts["power"]["x"], lts["power"]["y"], lts["power"]["z"] = lp[:, 0], lp[:, 1], lp[:, 2]
        return mats, lts

    def apply(self, renderer: Renderer, theta) -> None:
        mats, lts = self.tables(theta)
        renderer.set_materials(mats)
        if self.n_lights:
            renderer.set_lights(lts)


class _Render(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, renderer: Renderer, table: ParamTable, rounds: int) -> torch.Tensor:
        table.apply(renderer, theta.detach().to("cpu", torch.float32).numpy())
        img = renderer.adjoint_forward(rounds)
        ctx.renderer = renderer
        ctx.theta_device = theta.device
        return torch.from_numpy(img).to(theta.device)

    @staticmethod
    def backward(ctx, grad_img: torch.Tensor):
        g = ctx.renderer.adjoint_backward(grad_img.detach().to("cpu", torch.float32).contiguous().numpy())
        return torch.from_numpy(g).to(ctx.theta_device), None, None, None


def render(theta: torch.Tensor, renderer: Renderer, table: ParamTable, rounds: int = 1) -> torch.Tensor:
    """Linear SPPM image (H, W, 3) for parameters θ, differentiable with respect to θ.  Each call
    renders `rounds` fresh rounds; the backward pass must follow before the renderer is used again."""
    return _Render.apply(theta, renderer, table, rounds)
