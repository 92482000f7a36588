"""Material-parameter perturbation for finite-difference checks of the adjoint.

Parameters follow lum_backward's layout: albedo (material, channel), roughness (material),
emission (material, channel) where emission is the Emissive colour times its intensity.  An
emission change is applied to the material and to every NEE light that carries it, so the
rendered estimator stays consistent (the light list holds its own copy of the emission).
"""
from dataclasses import replace

import numpy as np

from luminara_b200 import abi

ALBEDO, ROUGHNESS, EMISSION = "albedo", "roughness", "emission"


def perturb(world, kind, m, c, delta):
    """Adds delta to one parameter of world (in place); returns a function that undoes it."""
    mat = world.materials[m]
    old_mat = replace(mat)
    old_lights = [replace(l) for l in world.lights]
    if kind == ALBEDO:
        col = list(mat.color)
        col[c] += delta
        mat.color = tuple(col)
    elif kind == ROUGHNESS:
        mat.roughness = mat.roughness + delta
    else:
        assert mat.kind == abi.MAT_EMISSIVE
        col = list(mat.color)
        col[c] += delta / mat.intensity
        mat.color = tuple(col)
        for l, lm in zip(world.lights, world.light_materials):
            if lm is mat:
                e = list(l.emission)
                e[c] += delta
                l.emission = tuple(e)

    def undo():
        for f in ("color", "roughness", "intensity"):
            setattr(mat, f, getattr(old_mat, f))
        for l, o in zip(world.lights, old_lights):
            l.emission = o.emission

    return undo


def grad_of(kind, m, c, da, dr, de):
    return da[m, c] if kind == ALBEDO else (dr[m] if kind == ROUGHNESS else de[m, c])


def param_list(world, kinds=(ALBEDO, ROUGHNESS, EMISSION)):
    out = []
    for m, mat in enumerate(world.materials):
        if mat.kind == abi.MAT_EMISSIVE:
            if EMISSION in kinds:
                out += [(EMISSION, m, c) for c in range(3)]
        elif mat.kind in (abi.MAT_LAMBERTIAN, abi.MAT_METAL, abi.MAT_MICROFACET):
            if ALBEDO in kinds:
                out += [(ALBEDO, m, c) for c in range(3)]
            if mat.kind == abi.MAT_MICROFACET and ROUGHNESS in kinds:
                out.append((ROUGHNESS, m, 0))
    return out


def directional(world, direction, scale):
    """Applies scale * direction (a dict param -> weight) to world; returns the undo."""
    undos = [perturb(world, k, m, c, scale * w) for (k, m, c), w in direction.items()]

    def undo():
        for u in reversed(undos):
            u()

    return undo


def seeded_weights(shape, seed=5):
    return np.random.default_rng(seed).normal(size=shape)
