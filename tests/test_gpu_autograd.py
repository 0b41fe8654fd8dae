"""The torch.autograd binding of the differentiable rollout: a config-3
style loss (mean squared distance of the final centres to targets) over
small settled piles, with per-scene friction and per-body masses as
parameters; gradients equal the C ABI's, and a finite difference of the
loss along a random velocity direction agrees with the autograd slope."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0


def make_world(pkg, specs, settle=60):
    w = pkg.World(0)
    for s in specs:
        w.add_scene(s)
    w.step(DT, steps=settle)
    return w


def test_autograd_binding(pkg, scenes):
    import torch
    ag = importlib.import_module("fyzzxyzzy-sdk_b200.autograd")
    specs = scenes.loose_piles(3, 12, base_seed=21)
    w = make_world(pkg, specs)
    nb, ns = w.counts()["bodies"], w.counts()["shapes"]
    props = np.zeros((nb, 11))
    dyn = np.zeros(nb, bool)
    for i in range(nb):
        try:
            props[i] = w.body_mass_properties(i)
            dyn[i] = True
        except RuntimeError:
            pass
    mass = torch.tensor(np.where(dyn, 1.0 / np.where(dyn, props[:, 0], 1.0), 0.0), requires_grad=True)
    # per-scene friction mapped to the scene's shapes (floor first)
    shape_scene = np.concatenate([[k] * (1 + s.n_shapes) for k, s in enumerate(specs)])
    mu_scene = torch.tensor([float(s.shape_mat[0, 0]) for s in specs], dtype=torch.float64, requires_grad=True)
    friction = mu_scene[torch.as_tensor(shape_scene)]
    rng = np.random.default_rng(5)
    v0 = torch.tensor(rng.normal(0, 0.5, (nb, 3)) * dyn[:, None], requires_grad=True)
    w0 = torch.tensor(rng.normal(0, 0.5, (nb, 3)) * dyn[:, None], requires_grad=True)
    c_start, _ = w.read_mass_frames()
    target = torch.tensor(c_start + rng.uniform(-1, 1, (nb, 3)) * dyn[:, None])
    mask = torch.tensor(dyn)
    c, v, wv = ag.rollout(w, v0, w0, mass, friction, steps=24, every=8)
    loss = ((c - target)[mask] ** 2).sum(1).mean()
    loss.backward()
    assert v0.grad is not None and mu_scene.grad is not None and mass.grad is not None
    # same gradients as the C ABI
    n_dyn = int(dyn.sum())
    wb = make_world(pkg, specs)
    wb.write_velocities(np.ascontiguousarray(np.concatenate([v0.detach().numpy(), w0.detach().numpy()], 1),
                                             np.float32))
    wb.rollout_begin(24, 8)
    wb.rollout_forward(DT)
    cb, _ = wb.read_mass_frames()
    gc = 2.0 * (cb - target.numpy()) / n_dyn * dyn[:, None]
    g = wb.rollout_backward(grad_center=gc)
    np.testing.assert_allclose(v0.grad.numpy(), g["v0"], rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(w0.grad.numpy(), g["w0"], rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(mass.grad.numpy(), g["mass"], rtol=1e-4, atol=1e-6)
    g_mu = np.bincount(shape_scene, weights=g["static_friction"] + g["dynamic_friction"])
    np.testing.assert_allclose(mu_scene.grad.numpy(), g_mu, rtol=1e-4, atol=1e-6)
