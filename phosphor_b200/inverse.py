"""Inverse rendering with the SPPM adjoint: recover per-material base colour and roughness and the
light power of a scene from target images (L2 loss on the linear image, Adam).

With common random numbers (the default) the target is one render at the true parameters and
every optimisation step renders with the same round seeds (the round-seed stream is saved once and
written back before each render, PHX_BUF_ROUND_RNG), so the loss is exactly 0 at the truth and its
gradient carries no sampling noise; otherwise the target is the mean of `target_renders`
independent renders and each step draws fresh rounds.  Each step renders `rounds` rounds at the
current parameters and back-propagates through the library's adjoint (phosphor_b200.adjoint).
Base colours and roughness are optimised directly (clamped to [0.01, 1] and [0.02, 0.99]); light
power is optimised as power / POWER_SCALE.

Most of the atrium's 32 materials cover few or no pixels, and the roughness of a non-metal only
reaches the image through its 4 % dielectric lobe, so not every parameter is observable.  Each
parameter's image sensitivity ||dI/dθ_j|| is estimated at the truth from random adjoint probes
(E[(g·dI/dθ_j)^2] = ||dI/dθ_j||^2 for g ~ N(0, 1) per pixel); parameters whose sensitivity is
below `observed_frac` of the largest of their kind are reported as unobserved, and the errors are
given over all parameters and over the observed ones.
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
    common_random_numbers: bool = True
    probes: int = 4
    observed_frac: float = 0.05


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
    rng0 = r.read("ROUND_RNG").copy()
    t0 = time.perf_counter()
    if cfg.common_random_numbers:
        target = r.adjoint_forward(cfg.rounds).astype(np.float64)
    else:
        target = np.zeros((cfg.height, cfg.width, 3), np.float64)
        for _ in range(cfg.target_renders):
            target += r.adjoint_forward(cfg.rounds)
        target /= cfg.target_renders
    # sensitivity of the image to each parameter at the truth (random adjoint probes)
    prng = np.random.default_rng(cfg.scene_seed)
    sens = np.zeros(table.size)
    for _ in range(cfg.probes):
        g = prng.standard_normal(cfg.width * cfg.height * 3).astype(np.float32)
        sens += r.adjoint_backward(g).astype(np.float64) ** 2
    sens = np.sqrt(sens / max(cfg.probes, 1))
    target = torch.from_numpy(target.astype(np.float32))
    t_target = time.perf_counter() - t0
    ms = sens[:4 * table.n_mat].reshape(table.n_mat, 4)
    base_sens = ms[:, :3].mean(axis=1)
    obs_base = base_sens >= cfg.observed_frac * base_sens.max()
    obs_rough = ms[:, 3] >= cfg.observed_frac * ms[:, 3].max()

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
        if cfg.common_random_numbers:
            r.write("ROUND_RNG", rng0)
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
                "observed_base_mae": float(np.abs(mm[obs_base, :3] - mt[obs_base, :3]).mean())
                if obs_base.any() else None,
                "observed_roughness_mae": float(np.abs(mm[obs_rough, 3] - mt[obs_rough, 3]).mean())
                if obs_rough.any() else None,
                "light_rel_err": float(np.abs(lp - lt).sum() / max(np.abs(lt).sum(), 1e-12))}

    return {"steps": cfg.steps, "rounds_per_step": cfg.rounds, "photons_per_round": cfg.photons,
            "pixels": cfg.width * cfg.height, "n_params": int(table.size),
            "common_random_numbers": cfg.common_random_numbers,
            "observed_materials_base": int(obs_base.sum()), "observed_materials_roughness": int(obs_rough.sum()),
            "loss_first": losses[0], "loss_last": float(np.mean(losses[-10:])),
            "error_start": errs(theta0), "error_end": errs(theta),
            "ms_per_step": 1e3 * float(np.median(fwd_bwd)), "target_s": t_target,
            "loss_curve": [round(x, 5) for x in losses[:: max(1, cfg.steps // 20)]]}
