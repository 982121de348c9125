"""Adjoint of the SPPM image with respect to per-material base colour / roughness and per-light power.

The function differentiated is the frozen-path estimator F(θ) (include/phx.h, oracle/phx_frozen.hpp):
paths and every discrete choice come from the scene's own parameters θ0, only weights move with θ.
The oracle evaluates F in double, and two reference gradients come from it: central finite
differences (h = 1e-3, frozen random numbers) and the analytic FP64 gradient, forward-mode dual
numbers through the same evaluation (oracle/phx_dual.hpp), which gives every one of the 131
partial derivatives exactly.  Gradients must agree within GRAD_TOL = 1e-3 relative.

CPU tests pin the oracle: its θ0 replay is bit-identical to the float render, F is smooth, and the
analytic gradient equals the finite differences.  GPU tests compare the library's adjoint
(phx_adjoint_backward) with both, the analytic one on all 131 coordinates.
"""
import numpy as np
import pytest

import oracle as O
import phosphor_b200 as P
from phosphor_b200 import _capi as A
from phosphor_b200.adjoint import ParamTable

GRAD_TOL = 1e-3  # relative, adjoint vs central finite differences of F
H = 1e-3         # finite-difference step (relative to each parameter's value)
ROUNDS = 2


def small_atrium(seed=3):
    scene = P.SceneData.generate(A.PHX_SCENE_ATRIUM, seed=seed, width=40, height=30, detail=4)
    args = P.ArgsList(width=40, height=30, photons_per_round=1 << 13, max_photon_bounces=8, grid_res=24, seed=seed,
                      direct_samples=4, sppm_alpha=0.7)
    return scene, args


def loss_of(o, args, table, theta, g):
    mats, lts = table.tables(theta)
    img, _, _ = o.frozen_render(args.params(), ROUNDS, mats, lts)
    return float(np.sum(img * g.reshape(-1, 3).astype(np.float64)))


def fd_directional(o, args, table, theta0, d, g):
    """Central difference (L(θ0 + s) - L(θ0 - s)) / 2 of L(θ) = Σ g·F(θ), s = H·|θ0|·d per
    coordinate.  Parameters are float32 in the scene tables, so the step actually taken, (θ+ - θ-)/2
    after rounding, is returned with it."""
    step = H * np.maximum(np.abs(theta0), 1e-2) * d
    tp = (theta0 + step).astype(np.float32)
    tm = (theta0 - step).astype(np.float32)
    lp = loss_of(o, args, table, tp, g)
    lm = loss_of(o, args, table, tm, g)
    return (lp - lm) / 2.0, (tp.astype(np.float64) - tm.astype(np.float64)) / 2.0


def test_param_table_round_trip():
    scene, _ = small_atrium()
    t = ParamTable(scene.materials(), scene.lights())
    th = t.vector()
    assert th.size == 4 * len(scene.materials()) + 3 * len(scene.lights())
    mats, lts = t.tables(th * 1.5)
    assert np.allclose(mats["roughness"], scene.materials()["roughness"] * 1.5)
    assert np.allclose(lts["power"]["y"], scene.lights()["power"]["y"] * 1.5)
    assert np.array_equal(mats["ior"], scene.materials()["ior"])
    assert np.array_equal(ParamTable(mats, lts).vector(), (th * 1.5).astype(np.float32))


def test_frozen_oracle_replays_the_float_render():
    scene, args = small_atrium()
    o = O.Oracle(scene)
    img, flux, rad = o.frozen_render(args.params(), ROUNDS, scene.materials(), scene.lights())
    st = o.render(args.params(), ROUNDS, prec=0)
    assert np.array_equal(st["flux"], flux) and np.array_equal(st["radiance"], rad)
    # at θ0, F differs from the float render's image only by precision and the RGBE quantisation
    area = np.pi * flux[:, 3:4]
    ref = rad[:, :3] / ROUNDS + np.where(area > 0, flux[:, :3] / np.where(area > 0, area, 1) /
                                         (args.photons_per_round * ROUNDS), 0)
    assert np.abs(img - ref).max() <= 1e-2 * np.abs(ref).max()


def test_frozen_estimator_is_smooth():
    """Central differences at h and h/2 agree to O(h^2): F has no kink at θ0."""
    scene, args = small_atrium()
    o = O.Oracle(scene)
    t = ParamTable(scene.materials(), scene.lights())
    th = t.vector().astype(np.float64)
    rng = np.random.default_rng(0)
    g = rng.standard_normal(args.width * args.height * 3)
    d = rng.standard_normal(th.size)
    d[3:4 * t.n_mat:4] *= (th[3:4 * t.n_mat:4] > 0.01) & (th[3:4 * t.n_mat:4] < 0.99)  # roughness off the clamp
    f1, _ = fd_directional(o, args, t, th, d, g)
    f2, _ = fd_directional(o, args, t, th, d / 2, g)
    assert abs(f1 - 2 * f2) <= 1e-4 * abs(f1)


def test_analytic_gradient_equals_finite_differences():
    """The forward-mode FP64 gradient of L(θ) = Σ g·F(θ) equals central differences of F along
    random directions through all parameters and along single coordinates (the finite differences
    carry an O(h^2) truncation error, about 1e-6 relative here)."""
    scene, args = small_atrium()
    o = O.Oracle(scene)
    t = ParamTable(scene.materials(), scene.lights())
    th = t.vector().astype(np.float64)
    rng = np.random.default_rng(4)
    g = rng.standard_normal(args.width * args.height * 3)
    grad, loss = o.frozen_grad(args.params(), ROUNDS, scene.materials(), scene.lights(), g)
    assert loss == pytest.approx(loss_of(o, args, t, th.astype(np.float32), g), rel=1e-12)
    assert grad.shape == (t.size,) and (grad != 0).sum() > 0.9 * t.size
    interior = (th[3:4 * t.n_mat:4] > 0.01) & (th[3:4 * t.n_mat:4] < 0.99)
    for k in range(3):
        d = rng.standard_normal(th.size)
        d[3:4 * t.n_mat:4] *= interior
        fd, step = fd_directional(o, args, t, th, d, g)
        assert abs(float(np.dot(grad, step)) - fd) <= 1e-4 * abs(fd), k
    for i in list(np.argsort(-np.abs(grad))[:4]) + [4 * t.n_mat + 2]:
        d = np.zeros(th.size)
        d[i] = 1.0
        fd, step = fd_directional(o, args, t, th, d, g)
        assert abs(grad[i] * step[i] - fd) <= 1e-4 * abs(fd) + 1e-12, i


@pytest.mark.gpu
def test_adjoint_matches_the_analytic_gradient_on_every_coordinate():
    """The library's reverse-mode adjoint against the oracle's forward-mode FP64 gradient, all 131
    coordinates: each within GRAD_TOL relative, or within GRAD_TOL of the largest partial for
    coordinates that are nearly zero (float accumulation noise)."""
    scene, args = small_atrium()
    t = ParamTable(scene.materials(), scene.lights())
    rng = np.random.default_rng(5)
    g = rng.standard_normal(args.width * args.height * 3).astype(np.float32)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        r.adjoint_forward(ROUNDS)
        grad = r.adjoint_backward(g).astype(np.float64)
    want, _ = O.Oracle(scene).frozen_grad(args.params(), ROUNDS, scene.materials(), scene.lights(),
                                          g.astype(np.float64))
    assert grad.shape == want.shape == (t.size,)
    scale = np.abs(want).max()
    err = np.abs(grad - want)
    bad = np.flatnonzero(err > GRAD_TOL * np.maximum(np.abs(want), 1e-3 * scale))
    assert len(bad) == 0, [(int(i), grad[i], want[i]) for i in bad[:8]]
    assert np.count_nonzero(want) > 0.9 * t.size


@pytest.mark.gpu
def test_adjoint_forward_is_the_render():
    scene, args = small_atrium()
    with P.Renderer(args) as r:
        r.set_scene(scene)
        img = r.adjoint_forward(ROUNDS).reshape(-1, 3)
        flux = r.read("FLUX")
        rad = r.read("RADIANCE")
    st = O.Oracle(scene).render(args.params(), ROUNDS, prec=0)
    assert np.array_equal(flux, st["flux"]) and np.array_equal(rad, st["radiance"])
    area = np.pi * flux[:, 3:4].astype(np.float64)
    want = rad[:, :3] / ROUNDS + np.where(area > 0, flux[:, :3] / np.where(area > 0, area, 1) /
                                          (args.photons_per_round * ROUNDS), 0)
    assert np.allclose(img, want, rtol=1e-5, atol=1e-7 * np.abs(want).max())


@pytest.mark.gpu
def test_adjoint_matches_finite_differences():
    scene, args = small_atrium()
    t = ParamTable(scene.materials(), scene.lights())
    th = t.vector().astype(np.float64)
    rng = np.random.default_rng(1)
    g = rng.standard_normal(args.width * args.height * 3).astype(np.float32)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        r.adjoint_forward(ROUNDS)
        grad = r.adjoint_backward(g).astype(np.float64)
        grad2 = r.adjoint_backward(g).astype(np.float64)
    assert np.allclose(grad, grad2, rtol=1e-5, atol=1e-9 * np.abs(grad).max())
    o = O.Oracle(scene)
    interior = (th[3:4 * t.n_mat:4] > 0.01) & (th[3:4 * t.n_mat:4] < 0.99)
    # random directions through every parameter
    for k in range(3):
        d = rng.standard_normal(th.size)
        d[3:4 * t.n_mat:4] *= interior
        fd, step = fd_directional(o, args, t, th, d, g)
        adj = float(np.dot(grad, step))
        assert abs(adj - fd) <= GRAD_TOL * abs(fd), (k, adj, fd)
    # the largest single coordinates: each material channel kind and the light
    big = np.argsort(-np.abs(grad))[:6]
    for i in list(big) + [4 * t.n_mat, 4 * t.n_mat + 1]:
        if i % 4 == 3 and i < 4 * t.n_mat and not interior[i // 4]:
            continue
        d = np.zeros(th.size)
        d[i] = 1.0
        fd, step = fd_directional(o, args, t, th, d, g)
        adj = float(grad[i] * step[i])
        assert abs(adj - fd) <= GRAD_TOL * abs(fd) + 1e-9 * np.abs(grad).max() * abs(step[i]), (i, adj, fd)


@pytest.mark.gpu
def test_adjoint_state_errors():
    scene, args = small_atrium()
    with P.Renderer(args) as r:
        r.set_scene(scene)
        g = np.zeros(args.width * args.height * 3, np.float32)
        with pytest.raises(A.PhxError) as e:
            r.adjoint_backward(g)
        assert e.value.code == A.PHX_E_STATE
        r.adjoint_forward(1)
        r.round()  # a round in between invalidates the recording
        with pytest.raises(A.PhxError) as e:
            r.adjoint_backward(g)
        assert e.value.code == A.PHX_E_STATE
        mats = scene.materials().copy()
        mats["diff_index"][0] = 0
        with pytest.raises(A.PhxError):
            r.set_materials(mats)


@pytest.mark.gpu
def test_torch_function_and_a_descent_step():
    """θ's base colours start off target; one step against the adjoint's gradient lowers the L2 image
    loss.  Every render starts from a fresh context, so all of them use the same random numbers."""
    import torch

    from phosphor_b200.adjoint import render
    scene, args = small_atrium()
    t = ParamTable(scene.materials(), scene.lights())
    th_true = torch.tensor(t.vector())
    with P.Renderer(args) as r:
        def img_of(th):
            r.set_scene(scene)
            return render(th, r, t, ROUNDS)

        target = img_of(th_true).detach()
        th = th_true.clone()
        th[:4 * t.n_mat:4] = 0.5  # the red base colour of every material off target
        th.requires_grad_(True)
        loss0 = ((img_of(th) - target) ** 2).sum()
        loss0.backward()
        assert th.grad is not None and th.grad.abs().sum() > 0
        with torch.no_grad():
            th1 = th - 0.02 * th.grad / th.grad.abs().max()
            loss1 = ((img_of(th1) - target) ** 2).sum()
    assert float(loss1.detach()) < float(loss0.detach())


@pytest.mark.gpu
def test_round_rng_state_replays_the_seeds():
    """PHX_BUF_ROUND_RNG holds the round-seed stream: a render after writing a saved state back
    repeats the earlier render bit for bit; without it the next render draws new seeds."""
    scene, args = small_atrium()
    with P.Renderer(args) as r:
        r.set_scene(scene)
        s0 = r.read("ROUND_RNG").copy()
        a = r.adjoint_forward(ROUNDS)
        b = r.adjoint_forward(ROUNDS)
        r.write("ROUND_RNG", s0)
        c = r.adjoint_forward(ROUNDS)
    assert not np.array_equal(a, b)
    assert np.array_equal(a.view(np.uint32), c.view(np.uint32))
