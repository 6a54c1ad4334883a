"""Fixed-topology family of window-frame yokes for the learned warm start.

A base mesh is morphed by a smooth radial-basis displacement of its nodes driven by 8 shape
parameters; the coil current density is the 9th input.  Every member has the base mesh's
cells, edges, orientations and material tags, so one solver (CSR pattern, element topology)
serves the whole family: only the node coordinates and the coil source field change.

Shape parameters p[0..7] in [-1, 1] (amplitude ``amp``, metres):
  0 outer half-width (x)      outer corners move by sign(x) * amp * p0
  1 outer half-height (y)     outer corners move by sign(y) * amp * p1
  2 aperture half-width       aperture corners move by sign(x) * amp * p2
  3 aperture half-height      aperture corners move by sign(y) * amp/2 * p3
  4 half-length (z)           all yoke corners move by sign(z) * 2 amp * p4
  5 x taper along z           all yoke corners move in x by sign(x) sign(z) * amp/2 * p5
  6 y taper along z           all yoke corners move in y by sign(y) sign(z) * amp/2 * p6
  7 aperture shift (x)        aperture corners move in x by amp/2 * p7
p[8] in [-1, 1] sets the coil current density J = J0 + dJ * p8 (default 3 +- 2 A/mm^2).

The displacement interpolates these corner moves with a Wendland C2 radial basis
(phi(r) = (1 - r/R)^4 (4 r/R + 1) for r < R) over the 16 yoke corners and 26 fixed points on
the air box (corners, edge midpoints, face centres) where it is zero; nodes on the box faces
are held fixed exactly.  The coil filaments are moved by the same displacement.
"""

import numpy as np

from . import mesh as M

N_PARAMS = 9


def wendland_c2(r, R):
    q = np.clip(r / R, 0.0, 1.0)
    return (1.0 - q) ** 4 * (4.0 * q + 1.0)


class YokeMorphFamily:
    def __init__(self, base_tets=300_000, seed=7, amp=0.02, support=0.45, J0=3e6, dJ=2e6, jitter=0.15):
        self.geometry = M.WindowFrameGeometry()
        self.mesh = M.window_frame_mesh(base_tets, jitter=jitter, seed=seed, geometry=self.geometry)
        self.base_nodes = self.mesh.nodes.copy()
        self.amp, self.support, self.J0, self.dJ = float(amp), float(support), float(J0), float(dJ)
        g = self.geometry
        ox, oy, l2 = 0.5 * g.outer_w, 0.5 * g.outer_h, 0.5 * g.length
        ax, ay = 0.5 * g.ap_w, 0.5 * g.ap_h
        sx, sy, sz = np.meshgrid([-1.0, 1.0], [-1.0, 1.0], [-1.0, 1.0], indexing="ij")
        sgn = np.stack([sx.ravel(), sy.ravel(), sz.ravel()], axis=1)  # 8 sign triples
        self._sgn = sgn
        outer = sgn * np.array([ox, oy, l2])
        aper = sgn * np.array([ax, ay, l2])
        bx, by, bz = (0.5 * b for b in g.box)
        grid = np.array([[i, j, k] for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)
                         if (i, j, k) != (0, 0, 0)], dtype=np.float64)
        fixed = grid * np.array([bx, by, bz])  # 26 points on the box surface
        self.ctrl = np.concatenate([outer, aper, fixed])
        self.n_moving = 16
        d = np.linalg.norm(self.ctrl[:, None, :] - self.ctrl[None, :, :], axis=2)
        self._Phi = wendland_c2(d, self.support)
        self._Phi_inv = np.linalg.inv(self._Phi)
        self._box = np.array([bx, by, bz])
        self._base_coils = g.coils()
        self._base_segments = [c.get_segments() for c in self._base_coils]
        self._weights_cache = {}
        # basis of the node displacement: one field per control point, evaluated once
        self._node_basis = self._basis(self.base_nodes)

    # -- parameters --------------------------------------------------------------------
    @staticmethod
    def sample(n, seed=0):
        """n seeded parameter vectors, uniform in [-1, 1]^9."""
        return np.random.default_rng(seed).uniform(-1.0, 1.0, size=(n, N_PARAMS))

    def corner_moves(self, p):
        """Displacements [16, 3] of the outer then aperture corners for shape parameters p[:8]."""
        a = self.amp
        s = self._sgn
        out = np.zeros((8, 3))
        ap = np.zeros((8, 3))
        out[:, 0] = s[:, 0] * a * p[0]
        out[:, 1] = s[:, 1] * a * p[1]
        ap[:, 0] = s[:, 0] * a * p[2]
        ap[:, 1] = s[:, 1] * 0.5 * a * p[3]
        for blk in (out, ap):
            blk[:, 2] += s[:, 2] * 2.0 * a * p[4]
            blk[:, 0] += s[:, 0] * s[:, 2] * 0.5 * a * p[5]
            blk[:, 1] += s[:, 1] * s[:, 2] * 0.5 * a * p[6]
        ap[:, 0] += 0.5 * a * p[7]
        return np.concatenate([out, ap])

    def _basis(self, pts):
        """[P, n_ctrl] matrix mapping control-point displacements to displacements at pts."""
        d = np.linalg.norm(pts[:, None, :] - self.ctrl[None, :, :], axis=2)
        return wendland_c2(d, self.support) @ self._Phi_inv

    def displacement(self, p, pts=None, basis=None):
        """Displacement [P, 3] at pts (the mesh nodes by default) for parameters p."""
        vals = np.zeros((len(self.ctrl), 3))
        vals[: self.n_moving] = self.corner_moves(np.asarray(p, dtype=np.float64))
        B = self._node_basis if (pts is None and basis is None) else (basis if basis is not None else self._basis(pts))
        u = B @ vals
        if pts is None and basis is None:
            on_box = np.any(np.isclose(np.abs(self.base_nodes), self._box, rtol=0.0, atol=1e-9), axis=1)
            u[on_box] = 0.0
        return u

    # -- members -----------------------------------------------------------------------
    def nodes(self, p):
        return self.base_nodes + self.displacement(p)

    def current_density(self, p):
        return self.J0 + self.dJ * float(p[8])

    def coil_segments(self, p):
        """Per coil: (segments [S, 6] moved with the nodes, current per filament)."""
        scale = self.current_density(p) / self.geometry.current_density
        out = []
        for coil, segs in zip(self._base_coils, self._base_segments):
            pts = segs.reshape(-1, 3)
            moved = (pts + self.displacement(p, pts=pts)).reshape(-1, 6)
            out.append((moved, coil.current * scale, coil.rad))
        return out

    def check(self, p):
        """Smallest signed tet volume (x6) of the morphed mesh: positive for a valid member."""
        X = self.nodes(p)[self.mesh.cells]
        a, b, c = X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]
        return float(np.einsum("ij,ij->i", a, np.cross(b, c)).min())
