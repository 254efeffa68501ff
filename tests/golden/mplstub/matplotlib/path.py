"""Minimal stand-in for matplotlib.path used while generating fixtures.

The reference imports ``matplotlib.path.Path`` for its electron-beam
crossing test (point in projected face polygon); matplotlib is not installed
here.  ``contains_points`` answers by even-odd ray casting; a positive
``radius`` also accepts points within that distance of an edge (how the
reference uses it: ``radius=1e-10`` marks points on the boundary).  Fixtures
made with it avoid impact parameters on face edges, where the two answers
could differ.
"""

import numpy as np


class Path(object):
    def __init__(self, vertices, codes=None, *args, **kwargs):
        self.vertices = np.asarray(vertices, dtype=float)

    def contains_points(self, points, transform=None, radius=0.0):
        pts = np.atleast_2d(np.asarray(points, dtype=float))
        v = self.vertices
        if len(v) > 1 and np.allclose(v[0], v[-1]):
            v = v[:-1]
        x, y = pts[:, 0], pts[:, 1]
        inside = np.zeros(len(pts), dtype=bool)
        m = len(v)
        for a in range(m):
            x1, y1 = v[a]
            x2, y2 = v[(a + 1) % m]
            cross = (y1 > y) != (y2 > y)
            with np.errstate(divide='ignore', invalid='ignore'):
                xc = x1 + (y - y1) * (x2 - x1) / (y2 - y1)
            inside ^= cross & (x < xc)
        if radius and radius > 0:
            for a in range(m):
                p1, p2 = v[a], v[(a + 1) % m]
                d = p2 - p1
                t = np.clip(((x - p1[0]) * d[0] + (y - p1[1]) * d[1]) / max(d @ d, 1e-300), 0, 1)
                dist = np.hypot(x - p1[0] - t * d[0], y - p1[1] - t * d[1])
                inside |= dist <= radius
        return inside
