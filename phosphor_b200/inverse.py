"""Inverse rendering with the SPPM adjoint: recover per-material base colour and roughness and the
light power of a scene from target images (L2 loss on the linear image, Adam).

The target is the mean of `target_renders` independent one-pass renders at the true parameters, so
it carries the same SPPM radius bias as each optimisation step's render and less noise.  Each step
renders `rounds` fresh rounds at the current parameters and back-propagates through the library's
adjoint (phosphor_b200.adjoint).  Base colours and roughness are optimised directly (clamped to
[0.01, 1] and [0.02, 0.99]); light power is optimised as power / POWER_SCALE.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np
import torch

from . import _capi as A
from .adjoint import ParamTable, render
from .renderer import ArgsList, Renderer, SceneData

POWER_SCALE = 100.0


@dataclasses.dataclass
class InverseConfig:
    width: int = 512
    height: int = 512
    photons: int = 1 << 20
    depth: int = 16
    grid: int = 64
    direct_samples: int = 16
    scene_seed: int = 1
    detail: int = 0
    steps: int = 200
    lr: float = 1e-2
    rounds: int = 1
    target_renders: int = 16
    init_base: float = 0.5
    init_rough: float = 0.5
    init_power: float = 140.0


def _encode(table: ParamTable, theta: np.ndarray) -> np.ndarray:
    p = theta.astype(np.float32).copy()
    p[4 * table.n_mat:] /= POWER_SCALE
    return p


def _decode(table: ParamTable, p: torch.Tensor) -> torch.Tensor:
    n = 4 * table.n_mat
    return torch.cat([p[:n], p[n:] * POWER_SCALE])


def _clamp_(table: ParamTable, p: torch.Tensor) -> None:
    n = 4 * table.n_mat
    with torch.no_grad():
        m = p[:n].view(table.n_mat, 4)
        m[:, :3].clamp_(0.01, 1.0)
        m[:, 3].clamp_(0.02, 0.99)
        p[n:].clamp_(0.0, None)


def run(cfg: InverseConfig, device: int = 0, log_every: int = 0) -> dict:
    scene = SceneData.generate(A.PHX_SCENE_ATRIUM, seed=cfg.scene_seed, width=cfg.width, height=cfg.height,
                               detail=cfg.detail)
    args = ArgsList(width=cfg.width, height=cfg.height, photons_per_round=cfg.photons, max_photon_bounces=cfg.depth,
                    grid_res=cfg.grid, seed=cfg.scene_seed, direct_samples=cfg.direct_samples, sppm_alpha=0.7)
    table = ParamTable(scene.materials(), scene.lights())
    theta_true = table.vector()
    r = Renderer(args, device=device)
    r.set_scene(scene)
    t0 = time.perf_counter()
    target = np.zeros((cfg.height, cfg.width, 3), np.float64)
    for _ in range(cfg.target_renders):
        target += r.adjoint_forward(cfg.rounds)
    target = torch.from_numpy((target / cfg.target_renders).astype(np.float32))
    t_target = time.perf_counter() - t0

    theta0 = theta_true.copy()
    m = theta0[:4 * table.n_mat].reshape(table.n_mat, 4)
    m[:, :3] = cfg.init_base
    m[:, 3] = cfg.init_rough
    theta0[4 * table.n_mat:] = cfg.init_power
    p = torch.tensor(_encode(table, theta0), requires_grad=True)
    opt = torch.optim.Adam([p], lr=cfg.lr)
    losses, fwd_bwd = [], []
    scale = 1.0 / float(target.pow(2).mean())
    for step in range(cfg.steps):
        ts = time.perf_counter()
        img = render(_decode(table, p), r, table, cfg.rounds)
        loss = ((img - target) ** 2).mean() * scale
        opt.zero_grad()
        loss.backward()
        fwd_bwd.append(time.perf_counter() - ts)
        opt.step()
        _clamp_(table, p)
        losses.append(float(loss.detach()))
        if log_every and step % log_every == 0:
            print(f"step {step}: loss {losses[-1]:.5f}")
    theta = _decode(table, p.detach()).numpy()
    r.close()

    def errs(th):
        mm = th[:4 * table.n_mat].reshape(table.n_mat, 4)
        mt = theta_true[:4 * table.n_mat].reshape(table.n_mat, 4)
        lp = th[4 * table.n_mat:]
        lt = theta_true[4 * table.n_mat:]
        return {"base_mae": float(np.abs(mm[:, :3] - mt[:, :3]).mean()),
                "roughness_mae": float(np.abs(mm[:, 3] - mt[:, 3]).mean()),
                "light_rel_err": float(np.abs(lp - lt).sum() / max(np.abs(lt).sum(), 1e-12))}

    return {"steps": cfg.steps, "rounds_per_step": cfg.rounds, "photons_per_round": cfg.photons,
            "pixels": cfg.width * cfg.height, "n_params": int(table.size),
            "loss_first": losses[0], "loss_last": float(np.mean(losses[-10:])),
            "error_start": errs(theta0), "error_end": errs(theta),
            "ms_per_step": 1e3 * float(np.median(fwd_bwd)), "target_s": t_target,
            "loss_curve": [round(x, 5) for x in losses[:: max(1, cfg.steps // 20)]]}
