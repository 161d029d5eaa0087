"""The hex8 element of the voxel grid (loadpath/fem.py:30, :113-224), host-side setup.

`hex8_ke(nu, element)` is the unit-cube stiffness at E = 1 with 2x2x2 Gauss integration;
"im" condenses Wilson's nine incompatible bubble modes, "plain" is the trilinear brick.
For side h and modulus E the element matrix is E * h * hex8_ke. The element in force follows
LOADPATH_HEX8 (im | plain), as in the reference.
"""
from __future__ import annotations

import os

import numpy as np

__all__ = ["CORNERS", "hex8_element", "hex8_ke", "elastic_c", "hex8_b", "corner_stress_ops"]

CORNERS = np.array([[(k >> a) & 1 for a in range(3)] for k in range(8)])
_ELEMENTS = ("im", "plain")
_CACHE: dict = {}


def hex8_element() -> str:
    e = os.environ.get("LOADPATH_HEX8", "im").strip().lower() or "im"
    if e not in _ELEMENTS:
        raise ValueError(f"LOADPATH_HEX8 must be one of {_ELEMENTS}, not {e!r}")
    return e


def elastic_c(nu: float) -> np.ndarray:
    """6x6 isotropic elasticity at unit modulus; Voigt order xx yy zz xy yz zx."""
    lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = 0.5 / (1.0 + nu)
    c = np.zeros((6, 6))
    c[:3, :3] = lam
    c[range(3), range(3)] += 2.0 * mu
    c[range(3, 6), range(3, 6)] = mu
    return c


def _strain_op(grads: np.ndarray) -> np.ndarray:
    """(6, 3n) strain operator of n vector basis functions with gradients grads (n, 3)."""
    n = len(grads)
    b = np.zeros((6, 3 * n))
    for k, (gx, gy, gz) in enumerate(grads):
        col = 3 * k
        b[0, col], b[1, col + 1], b[2, col + 2] = gx, gy, gz
        b[3, col], b[3, col + 1] = gy, gx
        b[4, col + 1], b[4, col + 2] = gz, gy
        b[5, col], b[5, col + 2] = gz, gx
    return b


def _gauss_points():
    g = 1.0 / np.sqrt(3.0)
    return [(a, b, c) for a in (-g, g) for b in (-g, g) for c in (-g, g)]


def _corner_grads(pt) -> np.ndarray:
    s = 2.0 * CORNERS - 1.0
    xi = np.asarray(pt)
    out = np.empty((8, 3))
    for a in range(3):
        o1, o2 = [b for b in range(3) if b != a]
        out[:, a] = 0.25 * s[:, a] * (1 + xi[o1] * s[:, o1]) * (1 + xi[o2] * s[:, o2])
    return out


def _bubble_grads(pt) -> np.ndarray:
    # mode m is (1 - x_m^2) on the cube [-1, 1]^3 mapped to the unit cube: d/dx_m = -4 x_m
    out = np.zeros((3, 3))
    for m in range(3):
        out[m, m] = -4.0 * pt[m]
    return out


def hex8_ke(nu: float, element: str | None = None) -> np.ndarray:
    element = element or hex8_element()
    key = (float(nu), element)
    if key not in _CACHE:
        c = elastic_c(nu)
        kuu = np.zeros((24, 24))
        kua = np.zeros((24, 9))
        kaa = np.zeros((9, 9))
        for pt in _gauss_points():
            b = _strain_op(_corner_grads(pt))
            ba = _strain_op(_bubble_grads(pt))
            kuu += 0.125 * b.T @ c @ b
            kua += 0.125 * b.T @ c @ ba
            kaa += 0.125 * ba.T @ c @ ba
        if element == "plain":
            k = kuu
        elif element == "im":
            k = kuu - kua @ np.linalg.solve(kaa, kua.T)
        else:
            raise ValueError(element)
        _CACHE[key] = 0.5 * (k + k.T)
    return _CACHE[key].copy()


def hex8_b(pt, nu: float, element: str | None = None) -> np.ndarray:
    """Strain-displacement matrix (6x24) of the unit cube at the natural point pt: the trilinear
    field plus, for the incompatible-mode element, the condensed bubbles' strain (zero at the
    centre) (loadpath/fem.py:227-237). For side h, divide by h."""
    element = element or hex8_element()
    b = _strain_op(_corner_grads(pt))
    if element == "plain":
        return b
    c = elastic_c(nu)
    kua = np.zeros((24, 9))
    kaa = np.zeros((9, 9))
    for g in _gauss_points():
        bg = _strain_op(_corner_grads(g))
        ba = _strain_op(_bubble_grads(g))
        kua += 0.125 * bg.T @ c @ ba
        kaa += 0.125 * ba.T @ c @ ba
    return b + _strain_op(_bubble_grads(pt)) @ (-np.linalg.solve(kaa, kua.T))


def corner_stress_ops(nu: float, pitch: float = 1.0, element: str | None = None) -> np.ndarray:
    """(8, 6, 24): the stress C B at the cube's eight corners per unit modulus, corners taken with
    x outermost (loadpath/constrained.py:443-446, its STRESS_POINTS = "corners")."""
    c = elastic_c(nu)
    return np.array([c @ hex8_b((a, b, cz), nu, element) / pitch
                     for a in (-1.0, 1.0) for b in (-1.0, 1.0) for cz in (-1.0, 1.0)])
