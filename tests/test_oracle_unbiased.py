"""The adjoint's estimator is unbiased: f64 statistics over many seeds (CPU, oracle).

For a small all-planar scene (10 GGX quads, 4 rect lights, 12x12, 4 spp, depth 4) and the
loss sum(image), the mean over 16000 seeds of a central finite difference with common random
numbers (step 5e-2 along the all-ones unit direction over the albedo or roughness parameters)
estimates the derivative of the expected image.  Three per-sample derivative estimators of the
oracle (orc_adjoint_dir) are compared with it:
  plain       the derivative of the per-sample image with every decision held: biased, since
              Russian roulette, the microfacet lobe and the NEE term move with the parameters;
  held        RR and lobe probabilities held in the weights they divide: still biased, because
              the reference adds the NEE term only on surviving paths without dividing by the
              survival probability (its expectation is surv * term);
  held+score  held plus the survival score term (surv'/surv) * NEE term: unbiased.  This is
              the estimator lum_backward computes (its agreement with the device is tested in
              test_gpu_adjoint.py).
"""
import os

import numpy as np
import torch.multiprocessing as mp

N_SEEDS = 16000
EPS = 5e-2


def _setup():
    from luminara_b200 import workloads as W
    from tests.diffparams import ALBEDO, ROUGHNESS, param_list

    world, cfg = W.diff_quads(width=12, height=12, spp=4, max_depth=4, n_quads=10)
    n = len(world.materials)
    dirs = {}
    for kind in (ALBEDO, ROUGHNESS):
        sel = [p for p in param_list(world) if p[0] == kind]
        v = np.ones(len(sel)) / np.sqrt(len(sel))
        vec = np.zeros(7 * n)
        for (k, m, c), x in zip(sel, v):
            vec[3 * m + c if kind == ALBEDO else 3 * n + m] = x
        dirs[kind] = (dict(zip(sel, v)), vec)
    return world, cfg, dirs


def _work(seeds):
    import oracle as O
    from tests.diffparams import ALBEDO, ROUGHNESS, directional

    world, cfg, dirs = _setup()
    lm = world.light_material_indices()
    g = np.ones(cfg.out_shape())
    out = []
    for s in seeds:
        cfg.seed = 7000 + s
        osc = O.OracleScene(world)
        row = []
        for kind in (ALBEDO, ROUGHNESS):
            d, vec = dirs[kind]
            row += [osc.adjoint_dir(cfg, g, vec, lm, detach=mode, threads=1) for mode in (0, 2, 1)]
            vals = []
            for sign in (1, -1):
                undo = directional(world, d, sign * EPS)
                im, _ = O.OracleScene(world).render(cfg, mode=O.MODE_KEYED, threads=1)
                undo()
                vals.append(float(im.sum()))
            row.append((vals[0] - vals[1]) / (2 * EPS))
        out.append(row)
    return out


def test_held_probabilities_with_survival_score_are_unbiased():
    nproc = max(1, min(8, os.cpu_count() or 1))
    ctx = mp.get_context("spawn")
    with ctx.Pool(nproc) as pool:
        parts = pool.map(_work, [list(range(i, N_SEEDS, nproc)) for i in range(nproc)])
    r = np.array([row for part in parts for row in part])
    z = {}
    for ki, kind in enumerate(("albedo", "roughness")):
        fd = r[:, 4 * ki + 3]
        for mi, name in enumerate(("plain", "held", "held+score")):
            diff = fd - r[:, 4 * ki + mi]
            z[kind, name] = diff.mean() / (diff.std(ddof=1) / np.sqrt(len(diff)))
    print({k: round(v, 2) for k, v in z.items()})
    assert abs(z["albedo", "held+score"]) < 3 and abs(z["roughness", "held+score"]) < 3
    assert abs(z["albedo", "plain"]) > 5 and abs(z["albedo", "held"]) > 5
    assert abs(z["roughness", "held"]) > 4
