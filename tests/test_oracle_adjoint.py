"""The f64 CPU adjoint (the checker for lum_backward) pinned by f64 finite differences.

With detach=0 the oracle adjoint is the plain derivative of the per-sample keyed estimator;
a central difference of orc_render (keyed, f64) with a tiny step and the same random numbers
must reproduce it for every parameter of a small all-planar scene (quads, rect lights) where
the estimator's derivative is exact.  With detach=1 (the device adjoint's estimator) the
emission gradients are unchanged, since emission moves no probability.
"""
import numpy as np
import pytest

import oracle as O
from luminara_b200 import workloads as W

from tests.diffparams import ALBEDO, EMISSION, ROUGHNESS, grad_of, param_list, perturb, seeded_weights


def small_scene(n_quads=12, w=20, h=20, spp=9, depth=4):
    world, cfg = W.diff_quads(width=w, height=h, spp=spp, max_depth=depth, n_quads=n_quads)
    return world, cfg


def weighted_sum(world, cfg, g):
    img, _ = O.OracleScene(world).render(cfg, mode=O.MODE_KEYED, threads=0)
    return float((g * img).sum())


def test_adjoint_primal_image_is_the_keyed_render():
    world, cfg = small_scene()
    osc = O.OracleScene(world)
    g = seeded_weights(cfg.out_shape())
    *_, img = osc.adjoint(cfg, g, world.light_material_indices())
    ref, _ = osc.render(cfg, mode=O.MODE_KEYED)
    assert ref.max() > 0.5
    np.testing.assert_allclose(img, ref, rtol=1e-12, atol=1e-14)


def test_plain_derivative_matches_tiny_step_finite_differences():
    world, cfg = small_scene()
    g = seeded_weights(cfg.out_shape())
    lm = world.light_material_indices()
    da, dr, de, _ = O.OracleScene(world).adjoint(cfg, g, lm, detach=False)
    h = 1e-7
    params = param_list(world)
    assert len(params) == 12 * 4 + 4 * 3
    grads = np.array([grad_of(k, m, c, da, dr, de) for k, m, c in params])
    scale = np.abs(grads).max()
    assert scale > 0
    fds = []
    for k, m, c in params:
        undo = perturb(world, k, m, c, h)
        lp = weighted_sum(world, cfg, g)
        undo()
        undo = perturb(world, k, m, c, -h)
        ln = weighted_sum(world, cfg, g)
        undo()
        fds.append((lp - ln) / (2 * h))
    fds = np.array(fds)
    err = np.abs(fds - grads)
    bad = err > 1e-5 * scale + 1e-5 * np.abs(grads)
    assert not bad.any(), [(params[i], fds[i], grads[i]) for i in np.nonzero(bad)[0]]
    # every kind of parameter carries signal in this scene
    kinds = np.array([k for k, _, _ in params])
    for kind in (ALBEDO, ROUGHNESS, EMISSION):
        assert np.abs(grads[kinds == kind]).max() > 1e-3 * scale


def test_detached_estimator_keeps_emission_gradients_and_is_linear():
    world, cfg = small_scene(n_quads=8, w=12, h=12, spp=4)
    osc = O.OracleScene(world)
    lm = world.light_material_indices()
    g1 = seeded_weights(cfg.out_shape(), 1)
    g2 = seeded_weights(cfg.out_shape(), 2)
    a0, r0, e0, _ = osc.adjoint(cfg, g1, lm, detach=False)
    a1, r1, e1, _ = osc.adjoint(cfg, g1, lm, detach=True)
    np.testing.assert_allclose(e1, e0, rtol=1e-12, atol=1e-14)
    assert not np.allclose(a1, a0)                   # RR / lobe probabilities move with albedo
    a2, r2, e2, _ = osc.adjoint(cfg, g2, lm, detach=True)
    a12, r12, e12, _ = osc.adjoint(cfg, g1 + 2 * g2, lm, detach=True)
    np.testing.assert_allclose(a12, a1 + 2 * a2, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(r12, r1 + 2 * r2, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(e12, e1 + 2 * e2, rtol=1e-9, atol=1e-12)


def test_light_without_material_routes_no_emission_gradient():
    world, cfg = small_scene(n_quads=8, w=12, h=12, spp=4)
    osc = O.OracleScene(world)
    g = np.ones(cfg.out_shape())
    _, _, with_lm, _ = osc.adjoint(cfg, g, world.light_material_indices())
    _, _, without, _ = osc.adjoint(cfg, g, None)
    emissive = [m for m, mat in enumerate(world.materials) if mat.kind == 4]
    # NEE light terms add to the light's material only when light_material names it
    assert (with_lm[emissive].sum() > without[emissive].sum()) and without[emissive].sum() >= 0
