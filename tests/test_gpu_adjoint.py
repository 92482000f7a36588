"""GPU tests of the path-replay adjoint (lum_forward / lum_backward).

1. Against the f64 CPU adjoint of the same keyed estimator (oracle, probabilities held plus
   the survival score term) on small all-planar scenes: per parameter kind, the gradient
   vectors agree within 2e-2 relative (L2), and 90% of the significant parameters within 5e-2
   each.  The device traces paths in f32, so a path whose discrete decision (RR, lobe, hit)
   flips against the f64 replay moves its few parameters; the aggregate is insensitive to that.
2. Against central finite differences with common random numbers on the differentiable
   workload (1000 GGX quads + 4 emissive quads, 512x512, 64 spp, depth 6, L2 loss against a
   render at parameters + N(0, 0.05)):
   - every emission parameter, per seed, step 1e-3, within 1e-2 relative (emission moves no
     sampling decision, so the per-seed difference is smooth);
   - albedo and roughness along fixed unit directions (each parameter stepped by ~1e-3),
     averaged over 2048 seeds: a per-seed difference of albedo or roughness also contains the
     jumps of paths whose Russian-roulette, lobe or visibility decision flips, whose mean is
     what the adjoint's held-probability and score terms account for.  The bar is 1e-2
     relative on the expectation; the seed means carry sampling error (standard error about
     0.3% for albedo and 1.1% for roughness at 2048 seeds), so the test requires the measured
     difference to lie within 1e-2 plus two standard errors.  A 4096-seed run measured
     -0.66% +- 0.22% (albedo) and -0.06% +- 0.77% (roughness).
"""
import numpy as np
import pytest

import luminara_b200 as L
import oracle as O
from luminara_b200 import workloads as W

from tests.diffparams import (ALBEDO, EMISSION, ROUGHNESS, directional, grad_of, param_list, perturb,
                              seeded_weights)

pytestmark = pytest.mark.gpu


def gpu_grads(world, cfg, g):
    sc = L.GpuScene(world)
    da, dr, de, st = sc.backward(cfg, g, world.light_material_indices())
    assert st.error_flags == 0
    return da.astype(np.float64), dr.astype(np.float64), de.astype(np.float64), st


def compare_kinds(world, ga, go):
    params = param_list(world)
    out = {}
    for kind in (ALBEDO, ROUGHNESS, EMISSION):
        sel = [p for p in params if p[0] == kind]
        a = np.array([grad_of(k, m, c, *ga) for k, m, c in sel])
        o = np.array([grad_of(k, m, c, *go) for k, m, c in sel])
        rel = np.linalg.norm(a - o) / max(np.linalg.norm(o), 1e-30)
        big = np.abs(o) > 1e-2 * np.abs(o).max()
        per = np.abs(a - o)[big] <= 5e-2 * np.abs(o)[big]
        out[kind] = (rel, per.mean(), np.linalg.norm(o))
    return out


@pytest.mark.parametrize("n_quads,size,spp,depth", [(12, 24, 16, 4), (60, 40, 16, 6)])
def test_device_adjoint_matches_f64_oracle_adjoint(n_quads, size, spp, depth):
    world, cfg = W.diff_quads(width=size, height=size, spp=spp, max_depth=depth, n_quads=n_quads)
    g = seeded_weights(cfg.out_shape(), 3)
    ga = gpu_grads(world, cfg, g)[:3]
    go = O.OracleScene(world).adjoint(cfg, g, world.light_material_indices(), detach=True)[:3]
    res = compare_kinds(world, ga, go)
    for kind, (rel, frac, norm) in res.items():
        assert norm > 0, kind
        assert rel <= 2e-2, (kind, res)
        assert frac >= 0.9, (kind, res)


def test_forward_is_lum_render_and_backward_is_linear():
    world, cfg = W.diff_quads(width=32, height=32, spp=16, max_depth=6, n_quads=60)
    sc = L.GpuScene(world)
    img, _ = sc.forward(cfg)
    ref, _ = sc.render(cfg)
    assert np.array_equal(img, ref)
    lm = world.light_material_indices()
    g1 = seeded_weights(cfg.out_shape(), 1).astype(np.float32)
    g2 = seeded_weights(cfg.out_shape(), 2).astype(np.float32)
    a1, r1, e1, _ = sc.backward(cfg, g1, lm)
    a2, r2, e2, _ = sc.backward(cfg, g2, lm)
    a3, r3, e3, _ = sc.backward(cfg, g1 + g2, lm)
    for x, y in ((a3, a1 + a2), (r3, r1 + r2), (e3, e1 + e2)):
        np.testing.assert_allclose(x, y, rtol=1e-3, atol=1e-4 * np.abs(y).max())
    z = sc.backward(cfg, np.zeros_like(g1), lm)
    assert all(not np.any(v) for v in z[:3])


def test_backward_rejects_deep_paths():
    world, cfg = W.diff_quads(width=8, height=8, spp=1, max_depth=17, n_quads=4)
    sc = L.GpuScene(world)
    with pytest.raises(L.LuminaraError):
        sc.backward(cfg, np.zeros(cfg.out_shape(), np.float32), world.light_material_indices())


def c5_problem():
    """The differentiable workload and an L2 loss against a render at perturbed parameters."""
    world, cfg = W.diff_quads()
    rng = np.random.default_rng(77)
    undos = []
    for k, m, c in param_list(world):
        d = float(rng.normal(0.0, 0.05))
        if k == EMISSION:
            d *= world.materials[m].intensity      # 5% of the emission scale
        undos.append(perturb(world, k, m, c, d))
    target, _ = L.GpuScene(world).render(cfg)
    for u in reversed(undos):
        u()
    return world, cfg, target.astype(np.float64)


def l2(world, cfg, target):
    img, _ = L.GpuScene(world).render(cfg)
    return float(((img.astype(np.float64) - target) ** 2).sum()), img


def test_c5_emission_central_finite_differences_per_parameter():
    world, cfg, target = c5_problem()
    loss0, img = l2(world, cfg, target)
    assert loss0 > 0
    da, dr, de, st = gpu_grads(world, cfg, (2.0 * (img.astype(np.float64) - target)).astype(np.float32))
    eps = 1e-3
    for k, m, c in [p for p in param_list(world) if p[0] == EMISSION]:
        g = grad_of(k, m, c, da, dr, de)
        undo = perturb(world, k, m, c, eps)
        lp, _ = l2(world, cfg, target)
        undo()
        undo = perturb(world, k, m, c, -eps)
        ln, _ = l2(world, cfg, target)
        undo()
        fd = (lp - ln) / (2 * eps)
        assert abs(fd - g) <= 1e-2 * abs(g), (k, m, c, fd, g)


def test_c5_albedo_roughness_finite_differences_seed_average():
    world, cfg, target = c5_problem()
    params = param_list(world)
    lm = world.light_material_indices()
    # loss weights and directions from reference seeds, disjoint from the test seeds
    cfg.seed = 999
    sc = L.GpuScene(world)
    img0, _ = sc.render(cfg)
    g = (2.0 * (img0.astype(np.float64) - target)).astype(np.float32)
    sels = {k: [p for p in params if p[0] == k] for k in (ALBEDO, ROUGHNESS)}
    acc = {k: 0.0 for k in sels}
    for r in range(16):
        cfg.seed = 900 + r
        da, dr, de, _ = sc.backward(cfg, g, lm)
        for k in sels:
            acc[k] = acc[k] + np.array([grad_of(*p, da, dr, de) for p in sels[k]], dtype=np.float64)
    dirs = {k: acc[k] / np.linalg.norm(acc[k]) for k in sels}
    eps = 5e-2                      # along a unit direction over ~3000 parameters: ~1e-3 each
    rows = {k: [] for k in sels}
    # the perturbed worlds are fixed: one scene each, rendered with every seed
    pert = {}
    for k in sels:
        for sign in (1, -1):
            undo = directional(world, dict(zip(sels[k], dirs[k])), sign * eps)
            pert[(k, sign)] = L.GpuScene(world)
            undo()
    idx = {k: [(m, c) for _, m, c in sels[k]] for k in sels}
    g64 = g.astype(np.float64)
    for s in range(2048):
        cfg.seed = 1000 + s
        da, dr, de, _ = sc.backward(cfg, g, lm)
        for k in sels:
            grads = (np.array([da[m, c] for m, c in idx[k]]) if k == ALBEDO
                     else np.array([dr[m] for m, _ in idx[k]]))
            ad = float(grads.astype(np.float64) @ dirs[k])
            vals = [float((g64 * pert[(k, sign)].render(cfg)[0]).sum()) for sign in (1, -1)]
            rows[k].append(((vals[0] - vals[1]) / (2 * eps), ad))
    for k in (ALBEDO, ROUGHNESS):
        r = np.array(rows[k])
        diff = r[:, 0] - r[:, 1]
        se = diff.std(ddof=1) / np.sqrt(len(diff))
        fd, ad = r[:, 0].mean(), r[:, 1].mean()
        print(f"{k}: mean FD {fd:.2f}, mean adjoint {ad:.2f}, rel diff {(fd - ad) / ad:+.4f}, rel SE {se / abs(ad):.4f}")
        assert abs(fd - ad) <= 1e-2 * abs(ad) + 2.0 * se, (k, fd, ad, se)


def test_c5_adjoint_costs_at_most_three_forward_renders():
    world, cfg, target = c5_problem()
    sc = L.GpuScene(world)
    img, _ = sc.forward(cfg)
    g = (2.0 * (img - target)).astype(np.float32)
    lm = world.light_material_indices()
    fwd, bwd = [], []
    for _ in range(3):
        _, s = sc.forward(cfg)
        fwd.append(s.kernel_ms)
        *_, s = sc.backward(cfg, g, lm)
        bwd.append(s.kernel_ms)
    ratio = min(bwd) / min(fwd)
    print(f"forward {min(fwd):.3f} ms, backward {min(bwd):.3f} ms, ratio {ratio:.2f}")
    assert ratio <= 3.0, ratio
