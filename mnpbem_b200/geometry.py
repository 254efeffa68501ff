"""Discretised particle surfaces (host side, float64).

``Particle`` and ``ComParticle`` reproduce the face data the BEM path reads
from the reference's geometry objects: centroids ``pos``, unit normal
``nvec``, tangents ``tvec1/tvec2``, ``area``, the boundary-element radius
``bradius()``, the standard face quadrature ``quad()`` (28 points per
triangle, quads split in two triangles) and the polar self-term quadrature
``quadpol()`` (144 points per triangle, 192 per quad).

Reference behaviour mirrored (file:line in the reference project):

* ``Particle.__init__``           mnpbem/geometry/particle.py:310-398
* flat normals / areas            mnpbem/geometry/particle.py:464-549
* curved normals / areas          mnpbem/geometry/particle.py:551-615
* ``totriangles`` (flat / curv)   mnpbem/geometry/particle.py:647-725
* ``quad`` (flat / curv)          mnpbem/geometry/particle.py:1431-1575
* ``quadpol`` (flat / curv)       mnpbem/geometry/particle.py:1276-1429
* shape functions                 mnpbem/geometry/particle.py:1607-1743
* ``bradius``                     mnpbem/geometry/particle.py:2848-2880
* ``ComParticle``                 mnpbem/geometry/comparticle.py:55-127, 596-800

The array arithmetic uses the same operation order as the reference
(``einsum`` subscripts, ``cross``, ``linalg.norm``) so that centroids,
normals and radii agree bit for bit: the near-pair classification that
consumes them is integer-exact only if its inputs are.

A particle given to the BEM classes may be one of these objects or any
object with the same attributes (for example the reference's own
``ComParticle``); the BEM classes only read the attributes listed above.
"""

import numpy as np

from .quadrature import QuadRules

__all__ = ["Particle", "ComParticle", "load_mesh", "trisphere"]


# --------------------------------------------------------------------------
# shape functions (unit triangle / [-1,1]^2 quad)
# --------------------------------------------------------------------------

def _tri6_shape(x, y):
    x, y = np.atleast_1d(x), np.atleast_1d(y)
    l1, l2, l3 = x, y, 1 - x - y
    n = np.zeros((len(x), 6))
    n[:, 0] = l1 * (2 * l1 - 1)
    n[:, 1] = l2 * (2 * l2 - 1)
    n[:, 2] = l3 * (2 * l3 - 1)
    n[:, 3] = 4 * l1 * l2
    n[:, 4] = 4 * l2 * l3
    n[:, 5] = 4 * l3 * l1
    return n


def _tri6_deriv(x, y):
    x, y = np.atleast_1d(x), np.atleast_1d(y)
    l1, l2, l3 = x, y, 1 - x - y
    dx = np.zeros((len(x), 6))
    dy = np.zeros((len(x), 6))
    dx[:, 0] = 4 * l1 - 1
    dx[:, 1] = 0
    dx[:, 2] = -4 * l3 + 1
    dx[:, 3] = 4 * l2
    dx[:, 4] = -4 * l2
    dx[:, 5] = 4 * (l3 - l1)
    dy[:, 0] = 0
    dy[:, 1] = 4 * l2 - 1
    dy[:, 2] = -4 * l3 + 1
    dy[:, 3] = 4 * l1
    dy[:, 4] = 4 * (l3 - l2)
    dy[:, 5] = -4 * l1
    return dx, dy


def _quad4_shape(x, y):
    x, y = np.atleast_1d(x), np.atleast_1d(y)
    n = np.zeros((len(x), 4))
    n[:, 0] = 0.25 * (1 - x) * (1 - y)
    n[:, 1] = 0.25 * (1 + x) * (1 - y)
    n[:, 2] = 0.25 * (1 + x) * (1 + y)
    n[:, 3] = 0.25 * (1 - x) * (1 + y)
    return n


def _quad4_deriv(x, y):
    x, y = np.atleast_1d(x), np.atleast_1d(y)
    dx = np.zeros((len(x), 4))
    dx[:, 0] = -0.25 * (1 - y)
    dx[:, 1] = 0.25 * (1 - y)
    dx[:, 2] = 0.25 * (1 + y)
    dx[:, 3] = -0.25 * (1 + y)
    dy = np.zeros((len(x), 4))
    dy[:, 0] = -0.25 * (1 - x)
    dy[:, 1] = -0.25 * (1 + x)
    dy[:, 2] = 0.25 * (1 + x)
    dy[:, 3] = 0.25 * (1 - x)
    return dx, dy


def _quad9_shape(x, y):
    x, y = np.atleast_1d(x), np.atleast_1d(y)
    n = np.zeros((len(x), 9))
    n[:, 0] = 0.25 * x * (x - 1) * y * (y - 1)
    n[:, 1] = 0.25 * x * (x + 1) * y * (y - 1)
    n[:, 2] = 0.25 * x * (x + 1) * y * (y + 1)
    n[:, 3] = 0.25 * x * (x - 1) * y * (y + 1)
    n[:, 4] = 0.5 * (1 - x ** 2) * y * (y - 1)
    n[:, 5] = 0.5 * x * (x + 1) * (1 - y ** 2)
    n[:, 6] = 0.5 * (1 - x ** 2) * y * (y + 1)
    n[:, 7] = 0.5 * x * (x - 1) * (1 - y ** 2)
    n[:, 8] = (1 - x ** 2) * (1 - y ** 2)
    return n


def _quad9_deriv(x, y):
    x, y = np.atleast_1d(x), np.atleast_1d(y)
    dx = np.zeros((len(x), 9))
    dy = np.zeros((len(x), 9))
    dx[:, 0] = 0.25 * (2 * x - 1) * y * (y - 1)
    dx[:, 1] = 0.25 * (2 * x + 1) * y * (y - 1)
    dx[:, 2] = 0.25 * (2 * x + 1) * y * (y + 1)
    dx[:, 3] = 0.25 * (2 * x - 1) * y * (y + 1)
    dy[:, 0] = 0.25 * x * (x - 1) * (2 * y - 1)
    dy[:, 1] = 0.25 * x * (x + 1) * (2 * y - 1)
    dy[:, 2] = 0.25 * x * (x + 1) * (2 * y + 1)
    dy[:, 3] = 0.25 * x * (x - 1) * (2 * y + 1)
    dx[:, 4] = -x * y * (y - 1)
    dx[:, 5] = 0.5 * (2 * x + 1) * (1 - y ** 2)
    dx[:, 6] = -x * y * (y + 1)
    dx[:, 7] = 0.5 * (2 * x - 1) * (1 - y ** 2)
    dy[:, 4] = 0.5 * (1 - x ** 2) * (2 * y - 1)
    dy[:, 5] = -x * (x + 1) * y
    dy[:, 6] = 0.5 * (1 - x ** 2) * (2 * y + 1)
    dy[:, 7] = -x * (x - 1) * y
    dx[:, 8] = -2 * x * (1 - y ** 2)
    dy[:, 8] = -2 * (1 - x ** 2) * y
    return dx, dy


# --------------------------------------------------------------------------
# Particle
# --------------------------------------------------------------------------

class Particle(object):
    """Triangle / quadrilateral surface mesh, flat or curved (6/9-node) faces.

    ``faces`` has 3, 4 or 9 columns.  With 9 columns (``verts`` then holds the
    extra midpoint vertices) the particle is curved: columns 0-3 are corners
    (column 3 NaN for triangles), 4-7 edge midpoints, 8 the quad centre.
    """

    def __init__(self, verts, faces, interp='flat', rule=18, npol=(7, 5)):
        verts = np.asarray(verts, dtype=float)
        faces = np.asarray(faces, dtype=float)
        if verts.ndim != 2 or verts.shape[1] != 3:
            raise ValueError("Particle: verts must have shape (n, 3)")
        if faces.ndim != 2 or faces.shape[1] not in (3, 4, 9):
            raise ValueError("Particle: faces must have 3, 4 or 9 columns")
        self.verts2 = None
        self.faces2 = None
        if faces.shape[1] == 3:
            self.verts = verts
            self.faces = np.hstack([faces, np.full((faces.shape[0], 1), np.nan)])
        elif faces.shape[1] == 4:
            self.verts = verts
            self.faces = faces
        else:
            self.verts2 = verts
            self.faces2 = faces
            corner = faces[:, :4].reshape(-1)
            valid = ~np.isnan(corner)
            uniq, inv = np.unique(corner[valid].astype(int), return_inverse=True)
            self.verts = verts[uniq]
            nf = np.full_like(faces[:, :4], np.nan)
            nf.flat[valid] = inv
            self.faces = nf
        self.quad_rules = QuadRules(rule=rule, npol=npol)
        self.interp = interp
        self._norm()

    # ---- basic properties ------------------------------------------------
    @property
    def nfaces(self):
        return self.faces.shape[0]

    n = nfaces

    @property
    def nverts(self):
        return self.verts.shape[0]

    @property
    def nvec(self):
        return self.vec[2]

    @property
    def tvec1(self):
        return self.vec[0]

    @property
    def tvec2(self):
        return self.vec[1]

    def index34(self, ind=None):
        f = self.faces if ind is None else self.faces[np.asarray(ind)]
        is_tri = np.isnan(f[:, 3])
        return np.where(is_tri)[0], np.where(~is_tri)[0]

    # ---- interpolation mode ------------------------------------------------
    def flat(self):
        """Flat boundary elements (mnpbem/geometry/particle.py:1745)."""
        self.interp = 'flat'
        self._norm()
        return self

    def curved(self):
        """Curved boundary elements (particle.py:1755).  A particle without
        midpoint vertices gets the straight-edge midpoints and, for
        quadrilaterals, the corner mean as centre node (the reference's
        ``midpoints('flat')``)."""
        if self.verts2 is None:
            self._flat_midpoints()
        self.interp = 'curv'
        self._norm()
        return self

    def _flat_midpoints(self):
        n = self.nverts
        ind3, ind4 = self.index34()
        f = self.faces
        # edges (k, k+1) of every face, triangles (0,1), (1,2), (2,0) and
        # quadrilaterals (0,1), (1,2), (2,3), (3,0): one midpoint per distinct edge
        ends = []
        for k in range(4):
            a = f[:, k]
            b = np.where(np.isnan(f[:, 3]) & (k == 2), f[:, 0], f[:, (k + 1) % 4])
            ends.append(np.column_stack([a, b]))
        e = np.stack(ends, axis=1)                        # (nfaces, 4, 2)
        valid = ~np.isnan(e[..., 0]) & ~np.isnan(e[..., 1])
        valid[ind3, 3] = False
        key = np.sort(e[valid].astype(np.int64), axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        mid = 0.5 * (self.verts[uniq[:, 0]] + self.verts[uniq[:, 1]])
        faces2 = np.full((self.nfaces, 9), np.nan)
        faces2[:, :4] = f
        cols = np.full(e.shape[:2], np.nan)
        cols[valid] = n + inv.reshape(-1)
        faces2[:, 4:8] = cols
        verts2 = np.vstack([self.verts, mid])
        if len(ind4) > 0:
            f4 = f[ind4].astype(int)
            cen = 0.25 * (self.verts[f4[:, 0]] + self.verts[f4[:, 1]] + self.verts[f4[:, 2]] +
                          self.verts[f4[:, 3]])
            faces2[ind4, 8] = verts2.shape[0] + np.arange(len(ind4))
            verts2 = np.vstack([verts2, cen])
        self.verts2, self.faces2 = verts2, faces2

    # ---- normals, centroids, areas ----------------------------------------
    def _norm(self):
        if self.interp == 'flat':
            self._norm_flat()
        else:
            if self.verts2 is None:
                raise ValueError("Particle: curved interpolation needs midpoint vertices")
            self._norm_curv()

    def _totriangles_flat(self, ind=None):
        ind = np.arange(self.nfaces) if ind is None else np.asarray(ind)
        _, ind4 = self.index34(ind)
        faces = self.faces[ind, :3].copy()
        if len(ind4) > 0:
            second = np.column_stack([self.faces[ind[ind4], 2], self.faces[ind[ind4], 3],
                                      self.faces[ind[ind4], 0]])
            faces = np.vstack([faces, second])
            ind4_out = np.column_stack([ind4, len(ind) + np.arange(len(ind4))])
        else:
            ind4_out = np.zeros((0, 2), dtype=int)
        return faces, ind4_out

    def _totriangles_curv(self, ind=None):
        ind = np.arange(self.nfaces) if ind is None else np.asarray(ind)
        ind3, ind4 = self.index34(ind)
        faces = np.zeros((len(ind), 6))
        if len(ind3) > 0:
            faces[ind3] = self.faces2[ind[ind3]][:, [0, 1, 2, 4, 5, 6]]
        if len(ind4) > 0:
            faces[ind4] = self.faces2[ind[ind4]][:, [0, 1, 2, 4, 5, 8]]
            second = self.faces2[ind[ind4]][:, [2, 3, 0, 6, 7, 8]]
            faces = np.vstack([faces, second])
            ind4_out = np.column_stack([ind4, len(ind) + np.arange(len(ind4))])
        else:
            ind4_out = np.zeros((0, 2), dtype=int)
        return faces, ind4_out

    def totriangles(self, ind=None):
        if self.interp == 'flat':
            return self._totriangles_flat(ind)
        return self._totriangles_curv(ind)

    def _norm_flat(self):
        n = self.nfaces
        ind3, ind4 = self.index34()
        self.pos = np.zeros((n, 3))
        if len(ind3) > 0:
            f3 = self.faces[ind3, :3].astype(int)
            self.pos[ind3] = (self.verts[f3[:, 0]] + self.verts[f3[:, 1]] +
                              self.verts[f3[:, 2]]) / 3.0
        if len(ind4) > 0:
            f4 = self.faces[ind4].astype(int)
            self.pos[ind4] = (self.verts[f4[:, 0]] + self.verts[f4[:, 1]] +
                              self.verts[f4[:, 2]] + self.verts[f4[:, 3]]) / 4.0
        tri, ind4s = self._totriangles_flat()
        v1 = self.verts[tri[:, 0].astype(int)]
        v2 = self.verts[tri[:, 1].astype(int)]
        v3 = self.verts[tri[:, 2].astype(int)]
        vec1 = v1 - v2
        vec2 = v3 - v2
        nvec = np.cross(vec1, vec2)
        area = 0.5 * np.sqrt(np.sum(nvec * nvec, axis=1))
        vec1_norm = np.sqrt(np.sum(vec1 * vec1, axis=1, keepdims=True))
        nvec_norm = np.sqrt(np.sum(nvec * nvec, axis=1, keepdims=True))
        vec1 = vec1 / np.maximum(vec1_norm, 1e-14)
        nvec = nvec / np.maximum(nvec_norm, 1e-14)
        vec2 = np.cross(nvec, vec1)
        if len(ind4s) == 0:
            self.area = area
            self.vec = [vec1, vec2, nvec]
            return
        self.area = area[:n].copy()
        # the second triangle of each quad adds its area to the quad
        np.add.at(self.area, ind4s[:, 0], area[ind4s[:, 1]])
        v1o, v2o, nvo = vec1[:n].copy(), vec2[:n].copy(), nvec[:n].copy()
        larger = area[ind4s[:, 1]] > area[ind4s[:, 0]]
        sel = ind4s[larger]
        v1o[sel[:, 0]] = vec1[sel[:, 1]]
        v2o[sel[:, 0]] = vec2[sel[:, 1]]
        nvo[sel[:, 0]] = nvec[sel[:, 1]]
        self.vec = [v1o, v2o, nvo]

    def _norm_curv(self):
        n = self.nfaces
        self.area = _row_sums(self)
        ind3, ind4 = self.index34()
        faces = self._totriangles_curv()[0]
        pos = np.zeros((n, 3))
        vec1 = np.zeros((n, 3))
        vec2 = np.zeros((n, 3))
        if len(ind3) > 0:
            tri = np.array([-1, -1, -1, 4, 4, 4]) / 9
            trix = np.array([1, 0, -1, 4, -4, 0]) / 3
            triy = np.array([0, 1, -1, 4, 0, -4]) / 3
            blk = self.verts2[faces[ind3, :6].astype(int)]
            pos[ind3] = np.einsum('c,icd->id', tri, blk)
            vec1[ind3] = np.einsum('c,icd->id', triy, blk)
            vec2[ind3] = np.einsum('c,icd->id', trix, blk)
        if len(ind4) > 0:
            fi = faces[ind4, :6].astype(int)
            pos[ind4] = self.verts2[fi[:, 5]]
            trix4 = np.array([1, 0, -1, 0, 0, 0])
            triy4 = np.array([0, -1, -1, 2, 2, -2])
            blk = self.verts2[fi]
            vec1[ind4] = np.einsum('c,icd->id', triy4, blk)
            vec2[ind4] = np.einsum('c,icd->id', trix4, blk)
        nvec = np.cross(vec1, vec2)
        nvec = nvec / np.maximum(np.linalg.norm(nvec, axis=1, keepdims=True), 1e-14)
        vec1 = vec1 / np.maximum(np.linalg.norm(vec1, axis=1, keepdims=True), 1e-14)
        vec2 = np.cross(nvec, vec1)
        self.pos = pos
        self.vec = [vec1, vec2, nvec]

    # ---- quadrature ----------------------------------------------------------
    def quad(self, ind=None):
        """Face quadrature: (pos (P,3), w (P,), row (P,)).

        ``row[p]`` is the position of the owning face inside ``ind``.  Points
        are ordered triangle by triangle: first one triangle per selected
        face, then the second triangles of the selected quads.  Weights
        include the surface Jacobian.
        """
        ind = np.arange(self.nfaces) if ind is None else np.asarray(ind)
        q = self.quad_rules
        x, y, w = q.x, q.y, q.w
        m = len(w)
        if self.interp == 'flat':
            # the face quadrature splits a quad (v0,v1,v2,v3) into (v0,v1,v2)
            # and (v0,v2,v3) (mnpbem/geometry/particle.py:1577-1604), unlike
            # the normal computation above
            faces = self.faces[ind]
            is_quad = ~np.isnan(faces[:, 3])
            qidx = np.where(is_quad)[0]
            tri = faces[:, :3]
            if len(qidx) > 0:
                tri = np.vstack([tri, faces[qidx][:, [0, 2, 3]]])
            ind3 = np.hstack([np.arange(len(ind)), qidx])
            v1 = self.verts[tri[:, 1].astype(int)] - self.verts[tri[:, 0].astype(int)]
            v2 = self.verts[tri[:, 2].astype(int)] - self.verts[tri[:, 0].astype(int)]
            area = 0.5 * np.linalg.norm(np.cross(v1, v2), axis=1)
            shape = np.column_stack([x, y, 1 - x - y])
            blk = self.verts[tri[:, :3].astype(int)]
            pos = np.einsum('tc,icd->itd', shape, blk).reshape(-1, 3)
            weight = (w[np.newaxis, :] * area[:, np.newaxis]).ravel()
        else:
            tri, ind4 = self._totriangles_curv(ind)
            ind3 = np.arange(len(ind))
            if len(ind4) > 0:
                ind3 = np.hstack([ind3, ind4[:, 0]])
            shape = _tri6_shape(x, y)
            dx, dy = _tri6_deriv(x, y)
            blk = self.verts2[tri[:, :6].astype(int)]
            pos = np.einsum('tc,icd->itd', shape, blk)
            px = np.einsum('tc,icd->itd', dx, blk)
            py = np.einsum('tc,icd->itd', dy, blk)
            jac = np.linalg.norm(np.cross(px, py, axis=2), axis=2)
            pos = pos.reshape(-1, 3)
            weight = (0.5 * w[np.newaxis, :] * jac).ravel()
        row = np.repeat(np.asarray(ind3), m)
        return pos, weight, row

    quad_integration = quad

    def quadpol(self, ind=None):
        """Polar self-term quadrature: (pos (P,3), w (P,), row (P,)).

        Triangles of ``ind`` come first (144 points each with the default
        rule), then quads (192 points each); ``row`` indexes into ``ind``.
        """
        ind = np.arange(self.nfaces) if ind is None else np.asarray(ind)
        ind3, ind4 = self.index34(ind)
        q = self.quad_rules
        m3, m4 = len(q.x3), len(q.x4)
        parts_pos, parts_w, parts_row = [], [], []
        if self.interp == 'flat':
            if len(ind3) > 0:
                shape = np.column_stack([q.x3, q.y3, 1 - q.x3 - q.y3])
                blk = self.verts[self.faces[ind[ind3], :3].astype(int)]
                parts_pos.append(np.einsum('tc,icd->itd', shape, blk).reshape(-1, 3))
                parts_w.append((q.w3[np.newaxis, :] * self.area[ind[ind3]][:, np.newaxis]).ravel())
                parts_row.append(np.repeat(ind3, m3))
            if len(ind4) > 0:
                shape = _quad4_shape(q.x4, q.y4)
                dx, dy = _quad4_deriv(q.x4, q.y4)
                blk = self.verts[self.faces[ind[ind4], :4].astype(int)]
                pos = np.einsum('tc,icd->itd', shape, blk)
                px = np.einsum('tc,icd->itd', dx, blk)
                py = np.einsum('tc,icd->itd', dy, blk)
                jac = np.linalg.norm(np.cross(px, py, axis=2), axis=2)
                parts_pos.append(pos.reshape(-1, 3))
                parts_w.append((q.w4[np.newaxis, :] * jac).ravel())
                parts_row.append(np.repeat(ind4, m4))
        else:
            faces = self.faces2[ind]
            if len(ind3) > 0:
                shape = _tri6_shape(q.x3, q.y3)
                dx, dy = _tri6_deriv(q.x3, q.y3)
                blk = self.verts2[faces[ind3][:, [0, 1, 2, 4, 5, 6]].astype(int)]
                pos = np.einsum('tc,icd->itd', shape, blk)
                px = np.einsum('tc,icd->itd', dx, blk)
                py = np.einsum('tc,icd->itd', dy, blk)
                jac = 0.5 * np.linalg.norm(np.cross(px, py, axis=2), axis=2)
                parts_pos.append(pos.reshape(-1, 3))
                parts_w.append((q.w3[np.newaxis, :] * jac).ravel())
                parts_row.append(np.repeat(ind3, m3))
            if len(ind4) > 0:
                shape = _quad9_shape(q.x4, q.y4)
                dx, dy = _quad9_deriv(q.x4, q.y4)
                blk = self.verts2[faces[ind4][:, :9].astype(int)]
                pos = np.einsum('tc,icd->itd', shape, blk)
                px = np.einsum('tc,icd->itd', dx, blk)
                py = np.einsum('tc,icd->itd', dy, blk)
                jac = np.linalg.norm(np.cross(px, py, axis=2), axis=2)
                parts_pos.append(pos.reshape(-1, 3))
                parts_w.append((q.w4[np.newaxis, :] * jac).ravel())
                parts_row.append(np.repeat(ind4, m4))
        if not parts_pos:
            return np.zeros((0, 3)), np.zeros(0), np.zeros(0, dtype=int)
        return np.vstack(parts_pos), np.concatenate(parts_w), np.concatenate(parts_row)

    # ---- element radius ------------------------------------------------------
    def bradius(self):
        """Radius of the smallest centroid-centred sphere holding each face."""
        r = np.zeros(self.nfaces)
        ind3, ind4 = self.index34()
        for ind, nc in ((ind3, 3), (ind4, 4)):
            if len(ind) == 0:
                continue
            for i in range(nc):
                vc = self.verts[self.faces[ind, i].astype(int)]
                r[ind] = np.maximum(r[ind], np.linalg.norm(self.pos[ind] - vc, axis=1))
        return r

    def flipfaces(self):
        """Reverse the face orientation (normals point the other way)."""
        f = self.faces.copy()
        ind3, ind4 = self.index34()
        f[ind3, :3] = f[ind3][:, [2, 1, 0]]
        f[ind4, :4] = f[ind4][:, [3, 2, 1, 0]]
        if self.faces2 is not None:
            raise NotImplementedError("flipfaces of curved particles is not needed on this path")
        return Particle(self.verts, f, interp=self.interp, rule=self.quad_rules.rule,
                        npol=self.quad_rules.npol)


def _row_sums(p):
    """Per-face sum of the face-quadrature weights (the curved face area)."""
    _, w, row = p.quad()
    # the reference sums the rows of a sparse (nfaces, npoints) weight matrix,
    # i.e. a segmented add.reduceat over each face's weights in point order
    order = np.argsort(row, kind='stable')
    ws, rs = w[order], row[order]
    counts = np.bincount(rs, minlength=p.nfaces)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.intp)
    return np.add.reduceat(ws, starts)


def _vertcat(particles):
    """Concatenate particles into one surface (same interpolation)."""
    if len(particles) == 1:
        return particles[0]
    interp = particles[0].interp
    if interp == 'flat':
        verts, faces, off = [], [], 0
        for q in particles:
            verts.append(q.verts)
            faces.append(q.faces + off)
            off += q.nverts
        return Particle(np.vstack(verts), np.vstack(faces), interp='flat',
                        rule=particles[0].quad_rules.rule, npol=particles[0].quad_rules.npol)
    verts, faces, off = [], [], 0
    for q in particles:
        verts.append(q.verts2)
        faces.append(q.faces2 + off)
        off += q.verts2.shape[0]
    return Particle(np.vstack(verts), np.vstack(faces), interp=interp,
                    rule=particles[0].quad_rules.rule, npol=particles[0].quad_rules.npol)


# --------------------------------------------------------------------------
# ComParticle
# --------------------------------------------------------------------------

class ComParticle(object):
    """Particles with the dielectric functions inside / outside each surface.

    ``eps`` is a list of dielectric functions (callables returning
    ``(eps, k)``), ``inout[i] = [inside, outside]`` holds 1-based indices into
    ``eps``.  Every particle is treated as its own closed surface unless
    ``closed`` lists are given (the reference defaults to that as well,
    mnpbem/greenfun/compgreen_ret.py:224-229).
    Mirrors mnpbem/geometry/comparticle.py:55-127.
    """

    def __init__(self, eps, particles, inout, *closed, **options):
        if eps is None or particles is None or inout is None:
            raise ValueError("ComParticle: eps, particles and inout are required")
        self.eps = list(eps)
        self.p = list(particles) if isinstance(particles, (list, tuple)) else [particles]
        # particle options, applied to the given particles as the reference
        # does (comparticle.py:129-163): interp 'curv' / 'flat', quadrature
        # rule and npol
        unknown = set(options) - {'interp', 'rule', 'npol'}
        if unknown:
            raise TypeError("ComParticle: unsupported options {}".format(sorted(unknown)))
        if 'rule' in options or 'npol' in options:
            for q in self.p:
                q.quad_rules = QuadRules(rule=options.get('rule', 18),
                                         npol=options.get('npol', (7, 5)))
        if 'interp' in options:
            for q in self.p:
                q.curved() if options['interp'] == 'curv' else q.flat()
        inout = np.atleast_2d(np.asarray(inout, dtype=int))
        if inout.shape != (len(self.p), 2):
            raise ValueError("ComParticle: inout must have one [in, out] row per particle")
        if inout.min() < 1 or inout.max() > len(self.eps):
            raise ValueError("ComParticle: inout indices are 1-based into eps")
        self.inout = inout
        self.closed = [None] * len(self.p)
        for i, c in enumerate(closed):
            if i < len(self.p):
                self.closed[i] = None if c is None else list(np.atleast_1d(c))
        if all(c is None for c in self.closed):
            self.closed = [[k + 1] for k in range(len(self.p))]
        self.pc = _vertcat(self.p)

    @property
    def nfaces(self):
        return int(sum(q.nfaces for q in self.p))

    n = nfaces

    @property
    def np(self):
        return len(self.p)

    @property
    def pos(self):
        return self.pc.pos

    @property
    def nvec(self):
        return self.pc.nvec

    @property
    def tvec1(self):
        return self.pc.tvec1

    @property
    def tvec2(self):
        return self.pc.tvec2

    @property
    def area(self):
        return self.pc.area

    def bradius(self):
        return np.hstack([q.bradius() for q in self.p])

    def quad(self, ind=None):
        return self.pc.quad(ind)

    quad_integration = quad

    def quadpol(self, ind=None):
        return self.pc.quadpol(ind)

    def index_func(self, i):
        """Face indices of particle ``i`` (1-based)."""
        off = np.cumsum([0] + [q.nfaces for q in self.p])
        return np.arange(off[i - 1], off[i])

    def offsets(self):
        return np.cumsum([0] + [q.nfaces for q in self.p]).astype(np.int64)

    @property
    def inout_faces(self):
        out = np.zeros((self.nfaces, 2), dtype=int)
        off = self.offsets()
        for i in range(len(self.p)):
            out[off[i]:off[i + 1]] = self.inout[i]
        return out

    def _eps_side(self, enei, col):
        vals = np.zeros(self.nfaces, dtype=complex)
        off = self.offsets()
        for i in range(len(self.p)):
            e, _ = self.eps[int(self.inout[i, col]) - 1](enei)
            vals[off[i]:off[i + 1]] = complex(np.asarray(e).flat[0])
        return vals

    def eps1(self, enei):
        return self._eps_side(enei, 0)

    def eps2(self, enei):
        return self._eps_side(enei, 1)

    def closed_groups(self):
        """Per particle: (direction, face indices of its closed surface) or None.

        Only closed surfaces made of this object's own particles (all
        entries positive) are supported, which is the default.  Mirrors
        ``ComParticle.closedparticle`` (mnpbem/geometry/comparticle.py:267-346)
        for that case.
        """
        out = []
        for i, c in enumerate(self.closed):
            if c is None:
                out.append(None)
                continue
            if any(int(v) <= 0 for v in c):
                raise NotImplementedError("closed surfaces with flipped parts are not supported")
            loc = np.hstack([self.index_func(int(v)) for v in c])
            out.append((1.0, loc))
        return out


# --------------------------------------------------------------------------
# packaged meshes
# --------------------------------------------------------------------------

_MESH_CACHE = {}


def load_mesh(name, second=False):
    """Load a packaged mesh ``(verts, faces)`` by name from ``data/meshes.npz``
    (``second``: the separately stored midpoint mesh ``(verts2, faces2)`` of a
    flat particle).

    The packaged meshes are the reference's own mesh-generator outputs
    (curved meshes are stored with their midpoint vertices), written by
    ``tests/golden/make_meshes.py``.
    """
    import os
    if not _MESH_CACHE:
        path = os.path.join(os.path.dirname(__file__), 'data', 'meshes.npz')
        with np.load(path) as z:
            for k in z.files:
                _MESH_CACHE[k] = z[k]
    suf = '2' if second else ''
    if name + '_verts' + suf not in _MESH_CACHE:
        raise KeyError("no packaged mesh named {!r}".format(name))
    return _MESH_CACHE[name + '_verts' + suf], _MESH_CACHE[name + '_faces' + suf]


def trisphere(n, diameter, interp='curv'):
    """Curved sphere mesh of ``n`` vertices and the given diameter (nm), the
    reference's ``trisphere(n, diameter)`` (mnpbem/geometry/mesh_generators.py:13).

    Packaged (n, diameter) pairs are the reference's output itself; other
    diameters scale the packaged unit-diameter mesh of the same ``n`` (equal to
    the reference's to rounding).
    """
    try:
        v, f = load_mesh('trisphere_{}_{:g}'.format(int(n), float(diameter)))
    except KeyError:
        v, f = load_mesh('trisphere_{}_1'.format(int(n)))
        v = v * float(diameter)
    if interp == 'curv':
        return Particle(v, f, interp='curv')
    return Particle(v, f, interp='curv')._as_flat()


def trirod(diameter, height, n):
    """Flat rod mesh (cylinder with hemispherical caps), quads + triangles,
    the reference's ``trirod(diameter, height, n)`` (mnpbem/geometry/
    mesh_generators.py:592).  Packaged parameter sets are the reference's
    output itself; others are built by ``rod_mesh``."""
    key = 'trirod_{:g}_{:g}_{}_{}_{}'.format(float(diameter), float(height), *n)
    try:
        v, f = load_mesh(key)
    except KeyError:
        return Particle(*rod_mesh(diameter, height, n), interp='flat')
    p = Particle(v, f, interp='flat')
    try:
        # the reference's midpoint mesh on the rod surface, for curved()
        p.verts2, p.faces2 = load_mesh(key, second=True)
    except KeyError:
        pass
    return p


def rod_mesh(diameter, height, n=(15, 20, 20)):
    """Vertices and faces of a rod along z: a cylinder of the given diameter
    with hemispherical caps, total length ``height`` (nm), centred at the
    origin -- the surface of the reference's ``trirod`` (mnpbem/geometry/
    mesh_generators.py:549-636): ``n = (nphi, ntheta, nz)`` grid points in
    azimuth (0..2 pi, the last equal to the first), in polar angle per cap
    (pole to equator) and along the cylinder.  Faces are quadrilaterals
    ordered outward, with triangles around the two poles; face count
    (nphi - 1) (2 (ntheta - 1) + nz - 1).

    Returns (verts (nv, 3), faces (nf, 4) 0-based, NaN in column 3 of the
    triangles).
    """
    nphi, ntheta, nz = (int(v) for v in n)
    if nphi < 4 or ntheta < 2 or nz < 2:
        raise ValueError("rod_mesh: n = (nphi >= 4, ntheta >= 2, nz >= 2)")
    if not height > diameter > 0:
        raise ValueError("rod_mesh: needs height > diameter > 0")
    r, h = 0.5 * diameter, 0.5 * (height - diameter)
    na = nphi - 1
    phi = np.linspace(0.0, 2.0 * np.pi, nphi)[:na]
    theta = np.linspace(0.0, 0.5 * np.pi, ntheta)
    zc = h * np.linspace(1.0, -1.0, nz)
    # rings from the top pole down: cap rings theta_1 .. theta_{ntheta-2}, the
    # cylinder rings (top one = upper cap equator, bottom one = lower cap
    # equator), then the lower cap rings mirrored
    rings = []
    for t in theta[1:-1]:
        rings.append((r * np.sin(t), h + r * np.cos(t)))
    for z in zc:
        rings.append((r, z))
    for t in theta[-2:0:-1]:
        rings.append((r * np.sin(t), -h - r * np.cos(t)))
    nr = len(rings)
    verts = [np.array([[0.0, 0.0, h + r]])]
    for rad, z in rings:
        verts.append(np.column_stack([rad * np.cos(phi), rad * np.sin(phi), np.full(na, z)]))
    verts.append(np.array([[0.0, 0.0, -h - r]]))
    verts = np.vstack(verts)
    top, bot = 0, 1 + nr * na
    ring = lambda k, a: 1 + k * na + (a % na)
    faces = []
    for a in range(na):
        faces.append([top, ring(0, a), ring(0, a + 1), np.nan])
    for k in range(nr - 1):
        for a in range(na):
            faces.append([ring(k, a), ring(k + 1, a), ring(k + 1, a + 1), ring(k, a + 1)])
    for a in range(na):
        faces.append([ring(nr - 1, a), bot, ring(nr - 1, a + 1), np.nan])
    faces = np.array(faces, dtype=float)
    # vertex order as the reference meshes: (v1 - v0) x (v2 - v0) points
    # into the body (Particle turns that into an outward normal)
    for f in faces:
        idx = f[~np.isnan(f)].astype(int)
        p = verts[idx]
        nrm = np.cross(p[1] - p[0], p[2] - p[0])
        c = p.mean(axis=0)
        out = np.array([c[0], c[1], 0.0 if abs(c[2]) <= h else c[2] - np.sign(c[2]) * h])
        if np.dot(nrm, out) > 0:
            f[:len(idx)] = idx[::-1]
    return verts, faces


def _as_flat(self):
    return Particle(self.verts, self.faces, interp='flat', rule=self.quad_rules.rule,
                    npol=self.quad_rules.npol)


def _transformed(self, fn):
    if self.verts2 is not None:
        v, f = fn(self.verts2), self.faces2
    else:
        v, f = fn(self.verts), self.faces
    return Particle(v, f, interp=self.interp, rule=self.quad_rules.rule,
                    npol=self.quad_rules.npol)


def _shift(self, vec):
    """Translated copy (vertices + vec), as mnpbem/geometry/particle.py:755."""
    vec = np.asarray(vec, dtype=float)
    return _transformed(self, lambda v: v + vec)


def _scale(self, factor):
    """Scaled copy (vertices * factor, scalar or per axis), as
    mnpbem/geometry/particle.py:820."""
    factor = np.asarray(factor, dtype=float)
    return _transformed(self, lambda v: v * factor)


Particle._as_flat = _as_flat
Particle.shift = _shift
Particle.scale = _scale
