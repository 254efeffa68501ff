"""Quadrature rules for boundary-element integration (host side, float64).

These are the integration rules the BEM path uses on every face:

* ``lobatto_nodes(n)`` -- Legendre-Gauss-Lobatto nodes and weights on [-1, 1]
  by Newton iteration from Chebyshev-Gauss-Lobatto starting points (the
  published von Winckel algorithm).  Mirrors ``mnpbem/utils/quadrature.py:15``.
* ``triangle_rule(18)`` -- the 28-point, degree-11 rule on the unit triangle
  from Burkardt's ``triangle_unit_set`` collection, weights normalised to sum 1.
  Mirrors ``mnpbem/utils/quadrature.py:92`` (rule 18 branch).  The table has to
  be the published one so the refined near-field integrals agree with the
  reference to rounding.
* ``polar_triangle_rule`` / ``polar_quad_rule`` -- polar integration around the
  centroid used for the singular self term: a Lobatto grid in (rho, phi) over
  one 60 degree (triangle) or 45 degree (quad) sector, rotated 3 or 4 times.
  Mirrors ``mnpbem/utils/quadface.py:106`` and ``:179``.

Operation order follows the reference so that points and weights agree to the
last bit (they feed the bit-exact near-pair classification only through the
face geometry, but bit-equality makes the parity tests sharp).
"""

import numpy as np

__all__ = ["lobatto_nodes", "triangle_rule", "polar_triangle_rule",
           "polar_quad_rule", "QuadRules"]


def lobatto_nodes(n):
    """Legendre-Gauss-Lobatto nodes/weights, n+1 points on [-1, 1].

    Newton iteration on x*P_n(x) - P_{n-1}(x) with the three-term Legendre
    recursion; mirrors ``mnpbem/utils/quadrature.py:15-89``.
    """
    if n < 2:
        raise ValueError("lobatto_nodes: n must be >= 2")
    n1 = n + 1
    x = np.cos(np.pi * np.arange(n1) / n)
    p = np.zeros((n1, n1))
    xold = 2.0 * np.ones(n1)
    while np.max(np.abs(x - xold)) > np.finfo(float).eps:
        xold = x.copy()
        p[:, 0] = 1.0
        p[:, 1] = x
        for k in range(2, n + 1):
            p[:, k] = ((2 * k - 1) * x * p[:, k - 1] - (k - 1) * p[:, k - 2]) / k
        x = xold - (x * p[:, n] - p[:, n - 1]) / (n1 * p[:, n])
    w = 2.0 / (n * n1 * p[:, n] ** 2)
    return x, w


# Burkardt triangle_unit_set rule 18: 28 points, precision 11.  Orbit
# generators (x, y) and the weight of each orbit; the point list below is the
# published ordering.
_R18_A = 1.0 / 3.0
_R18 = dict(b=0.9480217181434233, c=0.02598914092828833,
            d=0.8114249947041546, e=0.09428750264792270,
            f=0.01072644996557060, g=0.4946367750172147,
            p=0.5853132347709715, q=0.2073433826145142,
            r=0.1221843885990187, s=0.4389078057004907,
            t=0.6779376548825902, u=0.04484167758913055,
            v=0.27722066752827925, w=0.8588702812826364,
            x=0.0, y=0.1411297187173636)
_R18_W = (0.08797730116222190, 0.008744311553736190, 0.03808157199393533,
          0.01885544805613125, 0.07215969754474100, 0.06932913870553720,
          0.04105631542928860, 0.007362383783300573)


def triangle_rule(rule=18):
    """Points (x, y) and weights (sum 1) on the unit triangle (0,0),(1,0),(0,1).

    Only the rule the BEM path uses by default (18, 28 points) and the
    1-point centroid rule are provided.  Mirrors
    ``mnpbem/utils/quadrature.py:92-287``.
    """
    if rule == 1:
        return np.array([1 / 3]), np.array([1 / 3]), np.array([1.0])
    if rule != 18:
        raise ValueError("triangle_rule: only rules 1 and 18 are provided")
    a = _R18_A
    c = _R18
    xs = [a, c['b'], c['c'], c['c'], c['d'], c['e'], c['e'], c['f'], c['g'], c['g'],
          c['p'], c['q'], c['q'], c['r'], c['s'], c['s'], c['t'], c['t'], c['u'], c['u'],
          c['v'], c['v'], c['w'], c['w'], c['x'], c['x'], c['y'], c['y']]
    ys = [a, c['c'], c['b'], c['c'], c['e'], c['d'], c['e'], c['g'], c['f'], c['g'],
          c['q'], c['p'], c['q'], c['s'], c['r'], c['s'], c['u'], c['v'], c['t'], c['v'],
          c['t'], c['u'], c['x'], c['y'], c['w'], c['y'], c['w'], c['x']]
    w1, w2, w3, w4, w5, w6, w7, w8 = _R18_W
    ws = [w1, w2, w2, w2, w3, w3, w3, w4, w4, w4,
          w5, w5, w5, w6, w6, w6, w7, w7, w7, w7,
          w7, w7, w8, w8, w8, w8, w8, w8]
    x = np.array(xs)
    y = np.array(ys)
    w = np.array(ws)
    w = w / np.sum(w)
    return x, y, w


def _polar_grid(npol, phi_lo_deg, phi_span_deg):
    n_rad, n_ang = npol
    x1, w1 = lobatto_nodes(n_rad)
    rho_1d = 0.5 * (x1 + 1 + 1e-6)
    x2, w2 = lobatto_nodes(n_ang)
    phi_1d = np.deg2rad(phi_lo_deg + phi_span_deg * x2)
    rho_grid, phi_grid = np.meshgrid(rho_1d, phi_1d, indexing='ij')
    return rho_grid.ravel(), phi_grid.ravel(), np.outer(w1, w2).ravel()


def polar_triangle_rule(npol=(7, 5)):
    """Polar rule for the self term of a triangle (unit-triangle coords).

    3 sectors of 60 degrees around the centroid; weights sum to 1.  Mirrors
    ``mnpbem/utils/quadface.py:106-177``.
    """
    if np.isscalar(npol):
        npol = (int(npol), int(npol))
    rho, phi, w2d = _polar_grid(npol, 270, 60)
    rad = 1.0 / np.abs(2 * np.sin(phi))
    phi0 = np.deg2rad(120)
    phis = np.hstack([phi, phi + phi0, phi + 2 * phi0])
    rho_rep = np.tile(rho, 3)
    rad_rep = np.tile(rad, 3)
    xp = np.cos(phis) * rho_rep * rad_rep
    yp = np.sin(phis) * rho_rep * rad_rep
    x = (1 - np.sqrt(3) * xp - yp) / 3
    y = (1 + np.sqrt(3) * xp - yp) / 3
    w = np.tile(w2d * rho * rad ** 2, 3)
    w = w / np.sum(w)
    return x, y, w


def polar_quad_rule(npol=(7, 5)):
    """Polar rule for the self term of a quadrilateral on [-1,1]^2.

    4 sectors of 45 degrees; weights sum to 4.  Mirrors
    ``mnpbem/utils/quadface.py:179-240``.
    """
    if np.isscalar(npol):
        npol = (int(npol), int(npol))
    rho, phi, w2d = _polar_grid(npol, 90, 45)
    rad = 1.0 / np.abs(np.sin(phi))
    phi0 = np.deg2rad(90)
    phis = np.hstack([phi, phi + phi0, phi + 2 * phi0, phi + 3 * phi0])
    rho_rep = np.tile(rho, 4)
    rad_rep = np.tile(rad, 4)
    x = np.cos(phis) * rho_rep * rad_rep
    y = np.sin(phis) * rho_rep * rad_rep
    w = np.tile(w2d * rho * rad ** 2, 4)
    w = 4 * w / np.sum(w)
    return x, y, w


class QuadRules(object):
    """Bundle of the three rules a particle carries (``rule``, ``npol``).

    Mirrors the data members of ``mnpbem/utils/quadface.py:47`` (QuadFace):
    ``x, y, w`` (standard), ``x3, y3, w3`` (polar triangle),
    ``x4, y4, w4`` (polar quad).
    """

    def __init__(self, rule=18, npol=(7, 5)):
        if np.isscalar(npol):
            npol = (int(npol), int(npol))
        self.rule = rule
        self.npol = tuple(npol)
        self.x, self.y, self.w = triangle_rule(rule)
        self.x3, self.y3, self.w3 = polar_triangle_rule(npol)
        self.x4, self.y4, self.w4 = polar_quad_rule(npol)
