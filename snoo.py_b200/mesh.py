"""Tetrahedral meshes, edge numbering and boundary data.

The reference takes all of this from gmsh: nodes (``curl_curl_assembler.py:56-64``),
per-domain cells (``:88-129``), global edge ids from ``getKeysForElement``
(``mesh_tools.py:177-312``), per-element orientations (``mesh_tools.py:106-135``) and
the Dirichlet edge set (``mesh_tools.py:350-427``).  gmsh is not available, so
this module builds its own meshes and states the same data:

* ``nodes``        float64[N, 3]
* ``cells``        int32[E, 4], 0-based, every element positively oriented (det J > 0)
* ``elem_domain``  int32[E], the volume tag of each element
* ``edges``        int64[n, 2], (lower node, higher node), sorted; the row is the DoF id
* ``elem_edges``   int32[E, 6], 0-based DoF ids of the local edges (0,1),(0,2),(0,3),(1,2),(1,3),(2,3)
* ``orientations`` int32[E], 6-bit mask, bit j set when local edge j runs from the higher to the
  lower global node (see ``finite_element``)

The reference's 1-based conventions are kept where its Python code exposes them
(``global_ids`` and ``cells`` attributes of the assemblers, Dirichlet DoFs).

Mesh generators: a tensor-product grid whose hexahedra are split into 6 tetrahedra
around the main diagonal (Kuhn/Freudenthal split; conforming across cells), with
optional seeded jitter of the interior nodes.
"""

import numpy as np

from .finite_element import TET_EDGES

# volume tags used by the generators
TAG_IRON = 1
TAG_AIR = 2
TAG_COIL_1 = 3
TAG_COIL_2 = 4

# Kuhn split: the 6 axis permutations, each giving the path 0 -> e_a -> e_a+e_b -> 111
_PERMS = [(0, 1, 2), (1, 2, 0), (2, 0, 1), (0, 2, 1), (2, 1, 0), (1, 0, 2)]
_PERM_EVEN = [True, True, True, False, False, False]


def _kuhn_local_tets():
    """Local corner indices (bit 0 = x, bit 1 = y, bit 2 = z) of the 6 tets, positively ordered."""
    tets = []
    for perm, even in zip(_PERMS, _PERM_EVEN):
        a, b, _ = perm
        v0 = 0
        v1 = 1 << a
        v2 = v1 | (1 << b)
        v3 = 7
        tets.append([v0, v1, v2, v3] if even else [v0, v1, v3, v2])
    return np.array(tets, dtype=np.int64)


def tet_volumes6(nodes, cells):
    """Six times the signed volume of every tetrahedron (det of the affine map)."""
    p = nodes[cells]
    d1 = p[:, 1] - p[:, 0]
    d2 = p[:, 2] - p[:, 0]
    d3 = p[:, 3] - p[:, 0]
    return np.einsum("ij,ij->i", d1, np.cross(d2, d3))


class TetMesh:
    """A first-order tetrahedral mesh with edge DoFs and named boundaries.

    It also answers the few gmsh-model queries the solvers make (``mesh`` attribute,
    ``get_edge_boundary_dofs``), so the reference's solver constructors accept it in
    place of ``gmsh.model``.
    """

    def __init__(self, nodes, cells, elem_domain, grid=None, boundary_node_mask=None):
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        vol = tet_volumes6(self.nodes, cells)
        if np.any(vol <= 0):
            raise ValueError(f"{int(np.sum(vol <= 0))} tetrahedra are not positively oriented")
        self.cells = cells.astype(np.int32)
        self.elem_domain = np.ascontiguousarray(elem_domain, dtype=np.int32)
        self.grid = grid
        self._boundary_node_mask = boundary_node_mask
        self._number_edges()
        self.physical_groups = {}
        # (axis, value): outer-boundary planes that carry the natural condition (a symmetry
        # plane of a model cut in half); every other outer face is "Dirichlet Boundary"
        self.natural_planes = []

    # gmsh-model look-alike: solvers call gmsh_model.mesh
    @property
    def mesh(self):
        return self

    @property
    def num_nodes(self):
        return self.nodes.shape[0]

    @property
    def num_elements(self):
        return self.cells.shape[0]

    @property
    def num_dofs(self):
        return self.edges.shape[0]

    def _number_edges(self):
        c = self.cells.astype(np.int64)
        a = c[:, TET_EDGES[:, 0]]
        b = c[:, TET_EDGES[:, 1]]
        lo = np.minimum(a, b)
        hi = np.maximum(a, b)
        n_nodes = self.nodes.shape[0]
        keys = (lo * n_nodes + hi).reshape(-1)
        uniq, inv = np.unique(keys, return_inverse=True)
        self.edges = np.stack([uniq // n_nodes, uniq % n_nodes], axis=1)
        self.elem_edges = inv.reshape(-1, 6).astype(np.int32)
        bits = (a > b).astype(np.int32)
        self.orientations = (bits << np.arange(6, dtype=np.int32)).sum(axis=1).astype(np.int32)

    def domain_tags(self):
        return sorted(int(t) for t in np.unique(self.elem_domain))

    def domain_elements(self, tag):
        """Element indices of a volume tag (all elements when ``tag`` is -1)."""
        if tag == -1:
            return np.arange(self.num_elements)
        return np.flatnonzero(self.elem_domain == tag)

    def domain_nodes_mask(self, tag):
        m = np.zeros(self.num_nodes, dtype=bool)
        m[self.cells[self.domain_elements(tag)].reshape(-1)] = True
        return m

    def boundary_faces(self):
        """Faces (sorted node triples) that belong to exactly one tetrahedron."""
        c = np.sort(self.cells.astype(np.int64), axis=1)
        faces = np.concatenate([c[:, [0, 1, 2]], c[:, [0, 1, 3]], c[:, [0, 2, 3]], c[:, [1, 2, 3]]])
        n = self.num_nodes
        keys = (faces[:, 0] * n + faces[:, 1]) * n + faces[:, 2]
        uniq, counts = np.unique(keys, return_counts=True)
        b = uniq[counts == 1]
        return np.stack([b // (n * n), (b // n) % n, b % n], axis=1)

    def dirichlet_faces(self):
        """Outer boundary faces without those lying in a natural plane."""
        f = self.boundary_faces()
        if not self.natural_planes:
            return f
        scale = float(np.abs(self.nodes).max()) or 1.0
        keep = np.ones(len(f), dtype=bool)
        for axis, value in self.natural_planes:
            keep &= ~np.all(np.abs(self.nodes[f, axis] - value) <= 1e-12 * scale, axis=1)
        return f[keep]

    def dirichlet_edge_ids(self):
        """0-based ids of the edges on the Dirichlet part of the outer boundary."""
        return self._edge_ids_of_faces(self.dirichlet_faces())

    def boundary_edge_ids(self):
        """0-based ids of the edges on the outer boundary surface."""
        return self._edge_ids_of_faces(self.boundary_faces())

    def _edge_ids_of_faces(self, f):
        pairs = np.concatenate([f[:, [0, 1]], f[:, [0, 2]], f[:, [1, 2]]])
        n = self.num_nodes
        keys = np.unique(pairs[:, 0] * n + pairs[:, 1])
        ekeys = self.edges[:, 0] * n + self.edges[:, 1]
        idx = np.searchsorted(ekeys, keys)
        assert np.all(ekeys[idx] == keys)
        return idx

    def get_edge_boundary_dofs(self, names=("Dirichlet Boundary",), element_order=1):
        """1-based Dirichlet edge DoFs, like ``mesh_tools.get_edge_boundary_dofs`` (``mesh_tools.py:350-427``).

        The outer boundary of the mesh, without its natural planes, carries the name
        "Dirichlet Boundary".
        """
        out = []
        for name in names:
            if name != "Dirichlet Boundary":
                raise KeyError(f"unknown boundary {name!r}")
            out.append(self.dirichlet_edge_ids() + 1)
        return np.unique(np.concatenate(out)) if out else np.zeros(0, dtype=np.int64)

    def element_centroids(self, elems=None):
        c = self.cells if elems is None else self.cells[elems]
        return self.nodes[c].mean(axis=1)

    def get_cotree_dofs(self):
        """Tree-cotree split of the edges (``mesh_tools.py:468-566``): 0-based edge ids of a
        spanning tree of the node graph and of the remaining (cotree) edges.

        The reference takes networkx's minimum spanning tree of the unit-weight edge graph,
        i.e. any spanning tree.  Here the tree spans the Dirichlet boundary's nodes first (its
        edges are preferred), so that fixing the tree edges on top of the Dirichlet edges
        removes exactly the gradient null space of the other nodes.
        """
        from scipy.sparse import coo_matrix
        from scipy.sparse.csgraph import connected_components, minimum_spanning_tree

        n = self.num_nodes
        m = self.num_dofs
        w = np.full(m, 2.0)
        w[self.dirichlet_edge_ids()] = 1.0
        # edge id + 1 rides along in the weight's fraction so that the tree's edges come back
        # by id (weights stay ordered: boundary < interior)
        ids = np.arange(m, dtype=np.float64)
        G = coo_matrix((w + (ids + 1.0) / (2.0 * (m + 1)), (self.edges[:, 0], self.edges[:, 1])), shape=(n, n)).tocsr()
        ncomp, _ = connected_components(G, directed=False)
        if ncomp != 1:
            raise ValueError("The input graph must be connected.")
        T = minimum_spanning_tree(G).tocoo()
        frac = T.data - np.floor(T.data)
        tree = np.rint(frac * 2.0 * (m + 1) - 1.0).astype(np.int64)
        tree = np.sort(tree)
        mask = np.ones(m, dtype=bool)
        mask[tree] = False
        return tree, np.flatnonzero(mask)

    def index(self):
        """Device ``MeshIndex`` (bucket grid + node incidence) of this mesh, rebuilt when the
        node coordinates change."""
        from .mesh_index import MeshIndex

        key = (self.nodes.shape, self.cells.shape, float(np.add.reduce(self.nodes, axis=None)),
               int(self.cells[:: max(1, len(self.cells) // 64)].sum()))
        if getattr(self, "_index_key", None) != key:
            self._index = MeshIndex(self.nodes, self.cells)
            self._index_key = key
        return self._index

    def locate(self, points, tol=1e-12):
        """Element index (-1 outside) and barycentric coordinates of each point, on the device.

        Elements are bucketed by centroid on a uniform grid whose cell is at least the
        largest element extent, so a point's element lies in the 27 buckets around it.
        Replaces gmsh's point location used by ``evaluators.py:155-295``.
        """
        return self.index().locate(points, tol)


def tensor_grid_mesh(xs, ys, zs, cell_domain, jitter=0.0, seed=0, fixed_planes=None):
    """Split a tensor-product grid into positively oriented tetrahedra.

    :param xs, ys, zs: grid lines (strictly increasing).
    :param cell_domain: int array [nx, ny, nz] of volume tags per hexahedral cell.
    :param jitter: interior nodes move by U[-jitter, jitter] times the local spacing.
    :param fixed_planes: optional (x, y, z) lists of grid-line indices whose nodes do
        not move in that coordinate (material interfaces stay planar).
    """
    xs, ys, zs = (np.asarray(a, dtype=np.float64) for a in (xs, ys, zs))
    nx, ny, nz = len(xs) - 1, len(ys) - 1, len(zs) - 1
    n1x, n1y, n1z = nx + 1, ny + 1, nz + 1
    I, J, K = np.meshgrid(np.arange(n1x), np.arange(n1y), np.arange(n1z), indexing="ij")
    # node id: i fastest, then j, then k
    nid = lambda i, j, k: i + n1x * (j + n1y * k)
    nodes = np.zeros((n1x * n1y * n1z, 3))
    ids = nid(I, J, K).reshape(-1)
    nodes[ids, 0] = xs[I.reshape(-1)]
    nodes[ids, 1] = ys[J.reshape(-1)]
    nodes[ids, 2] = zs[K.reshape(-1)]
    if jitter > 0:
        rng = np.random.default_rng(seed)
        spacing = []
        for a in (xs, ys, zs):
            d = np.diff(a)
            s = np.empty(len(a))
            s[0] = d[0]
            s[-1] = d[-1]
            s[1:-1] = np.minimum(d[:-1], d[1:])
            spacing.append(s)
        idx = (I.reshape(-1), J.reshape(-1), K.reshape(-1))
        lim = (n1x - 1, n1y - 1, n1z - 1)
        for d in range(3):
            move = (idx[d] > 0) & (idx[d] < lim[d])
            if fixed_planes is not None and len(fixed_planes[d]) > 0:
                move &= ~np.isin(idx[d], np.asarray(fixed_planes[d]))
            # boundary nodes of the other directions stay on the outer surface
            for d2 in range(3):
                if d2 != d:
                    move &= (idx[d2] > 0) & (idx[d2] < lim[d2])
            delta = rng.uniform(-jitter, jitter, size=ids.size) * spacing[d][idx[d]]
            nodes[ids, d] += np.where(move, delta, 0.0)
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci, cj, ck = (a.reshape(-1) for a in (ci, cj, ck))
    # hex cells ordered with i fastest
    order = np.lexsort((ci, cj, ck))
    ci, cj, ck = ci[order], cj[order], ck[order]
    corners = np.stack([nid(ci + (b & 1), cj + ((b >> 1) & 1), ck + ((b >> 2) & 1)) for b in range(8)], axis=1)
    local = _kuhn_local_tets()  # [6, 4]
    cells = corners[:, local].reshape(-1, 4)
    dom = np.asarray(cell_domain)[ci, cj, ck]
    elem_domain = np.repeat(dom, 6)
    bmask = np.zeros(nodes.shape[0], dtype=bool)
    bmask[ids] = ((I == 0) | (I == nx) | (J == 0) | (J == ny) | (K == 0) | (K == nz)).reshape(-1)
    return TetMesh(nodes, cells, elem_domain, grid=(xs, ys, zs), boundary_node_mask=bmask)


def _graded_lines(breaks, h_in, h_out, inner_box):
    """Grid lines through all breakpoints; spacing h_in inside ``inner_box`` and h_out outside."""
    lines = [breaks[0]]
    for a, b in zip(breaks[:-1], breaks[1:]):
        mid = 0.5 * (a + b)
        h = h_in if inner_box[0] - 1e-12 <= mid <= inner_box[1] + 1e-12 else h_out
        n = max(1, int(np.ceil((b - a) / h - 1e-9)))
        lines.extend(list(a + (b - a) * np.arange(1, n + 1) / n))
    return np.array(lines)


class WindowFrameGeometry:
    """Window-frame yoke in an air box (dimensions in m).

    Air box 1.0 x 1.0 x 1.2; yoke 0.6 (x) by 0.6 (y), 0.5 long in z, aperture 0.3 x 0.2;
    the vertical legs are x in [-0.3,-0.15] and [0.15,0.3].  Two coils wind around the
    vertical legs inside the window height |y| <= 0.1 with a 0.05 m thick winding pack
    touching the leg.
    """

    def __init__(self, outer_w=0.6, outer_h=0.6, ap_w=0.3, ap_h=0.2, length=0.5,
                 box=(1.0, 1.0, 1.2), coil_t=0.05, current_density=3e6):
        self.outer_w, self.outer_h = outer_w, outer_h
        self.ap_w, self.ap_h = ap_w, ap_h
        self.length = length
        self.box = box
        self.coil_t = coil_t
        self.current_density = current_density

    def breaks(self, coils=False):
        bx, by, bz = (0.5 * b for b in self.box)
        ox, oy, l2 = 0.5 * self.outer_w, 0.5 * self.outer_h, 0.5 * self.length
        ax, ay = 0.5 * self.ap_w, 0.5 * self.ap_h
        xb = [-bx, -ox, -ax, ax, ox, bx]
        yb = [-by, -oy, -ay, ay, oy, by]
        zb = [-bz, -l2, l2, bz]
        if coils:
            t = self.coil_t
            xb += [-ox - t, -ax + t, ax - t, ox + t]
            zb += [-l2 - t, l2 + t]
        return sorted(set(np.round(xb, 12))), sorted(set(np.round(yb, 12))), sorted(set(np.round(zb, 12)))

    def classify(self, c, coils=False):
        """Volume tag of points c[..., 3]."""
        x, y, z = c[..., 0], c[..., 1], c[..., 2]
        ox, oy, l2 = 0.5 * self.outer_w, 0.5 * self.outer_h, 0.5 * self.length
        ax, ay = 0.5 * self.ap_w, 0.5 * self.ap_h
        iron = (np.abs(x) < ox) & (np.abs(y) < oy) & (np.abs(z) < l2) & ~((np.abs(x) < ax) & (np.abs(y) < ay))
        tag = np.where(iron, TAG_IRON, TAG_AIR)
        if coils:
            t = self.coil_t
            for side, ctag in ((-1.0, TAG_COIL_1), (1.0, TAG_COIL_2)):
                xc = side * x  # leg at xc in [ax, ox]
                in_outer = (xc > ax - t) & (xc < ox + t) & (np.abs(z) < l2 + t)
                in_inner = (xc > ax) & (xc < ox) & (np.abs(z) < l2)
                ring = in_outer & ~in_inner & (np.abs(y) < ay)
                tag = np.where(ring, ctag, tag)
        return tag

    def coil_keypoints(self, side):
        """The 8 racetrack keypoints (x, z) of the winding-pack centreline around one leg."""
        ox, ax, l2, t = 0.5 * self.outer_w, 0.5 * self.ap_w, 0.5 * self.length, self.coil_t
        x0, x1 = ax - 0.5 * t, ox + 0.5 * t  # in side-local coordinates
        z0 = l2 + 0.5 * t
        r = 0.5 * t
        # counter-clockwise rounded rectangle in (x, z), kp7->kp0 is the first straight segment
        kp = np.array([[x1, -z0 + r], [x1, z0 - r], [x1 - r, z0], [x0 + r, z0],
                       [x0, z0 - r], [x0, -z0 + r], [x0 + r, -z0], [x1 - r, -z0]])
        kp[:, 0] *= side
        if side < 0:
            kp = kp[::-1].copy()
        return kp

    def coils(self, n_turns=8, senses=(1.0, -1.0)):
        """Two racetrack filament coils carrying the winding pack's ampere-turns.

        J * t * (aperture height) ampere-turns per coil, split over ``n_turns``
        filaments stacked in y.  ``senses`` (+1/-1) set the winding direction per leg;
        opposite senses drive flux around the frame.
        """
        from .racetrack_coil import RacetrackCoil

        ay = 0.5 * self.ap_h
        y = -ay + self.ap_h * (np.arange(n_turns) + 0.5) / n_turns
        amp_turns = self.current_density * self.coil_t * self.ap_h
        out = []
        for side, s in zip((-1.0, 1.0), senses):
            kp = self.coil_keypoints(side)
            if s < 0:
                kp = kp[::-1].copy()
            out.append(RacetrackCoil(kp, y, rad=0.5 * self.ap_h / n_turns, current=amp_turns / n_turns))
        return out

    def aperture_probes(self, n=1000, seed=1234, margin=0.01):
        """Seeded uniform-random points inside the aperture (inside the yoke length)."""
        rng = np.random.default_rng(seed)
        ax, ay, l2 = 0.5 * self.ap_w - margin, 0.5 * self.ap_h - margin, 0.5 * self.length - margin
        return np.stack([rng.uniform(-ax, ax, n), rng.uniform(-ay, ay, n), rng.uniform(-l2, l2, n)], axis=1)


def window_frame_mesh(target_tets=40000, jitter=0.15, seed=7, coils=False, geometry=None, grading=1.6):
    """Window-frame yoke mesh with about ``target_tets`` tetrahedra.

    Cells inside the yoke's bounding region have spacing h, the air around it h*grading;
    h is chosen by bisection to approach ``target_tets``.  Material interfaces stay planar
    (interface nodes do not move across them).
    """
    g = geometry or WindowFrameGeometry()
    xb, yb, zb = g.breaks(coils)
    ext = 0.5 * max(g.outer_w, g.outer_h) + (g.coil_t if coils else 0.0)
    inner = (-ext - 1e-9, ext + 1e-9)
    zin = (-(0.5 * g.length + (g.coil_t if coils else 0.0)) - 1e-9, 0.5 * g.length + (g.coil_t if coils else 0.0) + 1e-9)

    def lines(h):
        return (_graded_lines(xb, h, h * grading, inner), _graded_lines(yb, h, h * grading, inner),
                _graded_lines(zb, h, h * grading, zin))

    lo, hi = 0.002, 0.5
    for _ in range(60):
        mid = np.sqrt(lo * hi)
        xs, ys, zs = lines(mid)
        ntet = 6 * (len(xs) - 1) * (len(ys) - 1) * (len(zs) - 1)
        if ntet > target_tets:
            lo = mid
        else:
            hi = mid
    xs, ys, zs = lines(hi)
    cx, cy, cz = 0.5 * (xs[1:] + xs[:-1]), 0.5 * (ys[1:] + ys[:-1]), 0.5 * (zs[1:] + zs[:-1])
    C = np.stack(np.meshgrid(cx, cy, cz, indexing="ij"), axis=-1)
    dom = g.classify(C, coils)
    fixed = [np.flatnonzero(np.isin(np.round(a, 12), np.round(b, 12))) for a, b in ((xs, xb), (ys, yb), (zs, zb))]
    mesh = tensor_grid_mesh(xs, ys, zs, dom, jitter=jitter, seed=seed, fixed_planes=fixed)
    mesh.geometry = g
    if coils:
        mesh.coil_terminals = {}
        for ctag in (TAG_COIL_1, TAG_COIL_2):
            mesh.coil_terminals[ctag] = _coil_terminals(mesh, ctag, zs)
    return mesh


def _coil_terminals(mesh, ctag, zs):
    """Cut a coil ring open on the outer side of its leg and return its two terminal node sets.

    The coil elements of the outer winding side (|x| beyond the yoke) in the first layer
    of cells at z >= 0 become air.  The coil nodes on the two faces of that gap are the
    terminals, like the terminal surfaces a gmsh coil geometry carries
    (``laplace_subdomain_solver.py:71-115``).  Terminals are found topologically, so
    jittered nodes do not matter.
    """
    g = mesh.geometry
    ox = 0.5 * g.outer_w
    elems = mesh.domain_elements(ctag)
    cen = mesh.element_centroids(elems)
    outer = elems[np.abs(cen[:, 0]) > ox]
    cz = mesh.element_centroids(outer)[:, 2]
    k0 = int(np.searchsorted(zs, -1e-12))
    z_lo, z_hi = zs[k0], zs[k0 + 1]
    zmid = 0.5 * (z_lo + z_hi)
    gap = outer[np.abs(cz - zmid) < 0.5 * (z_hi - z_lo)]
    mesh.elem_domain[gap] = TAG_AIR
    gap_nodes = np.zeros(mesh.num_nodes, dtype=bool)
    gap_nodes[mesh.cells[gap].reshape(-1)] = True
    rest = mesh.domain_elements(ctag)
    cr = mesh.element_centroids(rest)[:, 2]
    below = np.zeros(mesh.num_nodes, dtype=bool)
    above = np.zeros(mesh.num_nodes, dtype=bool)
    below[mesh.cells[rest[cr < zmid]].reshape(-1)] = True
    above[mesh.cells[rest[cr > zmid]].reshape(-1)] = True
    t1 = np.flatnonzero(gap_nodes & below & ~above)
    t2 = np.flatnonzero(gap_nodes & above & ~below)
    return t1, t2


def bar_conductor_mesh(target_tets=20000, jitter=0.1, seed=3, box=(0.6, 0.6, 0.8), bar=0.1, ring=(0.3, 0.5),
                       ring_length=0.4):
    """A straight conductor bar along z through the whole box inside a square iron ring.

    The bar (|x|, |y| < bar/2, all z) is volume TAG_COIL_1; its terminals are its node sets on
    the two z faces of the box, which carry the Dirichlet condition, so the source current
    enters and leaves through the boundary (a consistent total-potential problem).  The iron
    ring (inner/outer half widths ring, |z| < ring_length/2) is TAG_IRON, the rest TAG_AIR.
    """
    bx, by, bz = (0.5 * b for b in box)
    hb, ri, ro, lz = 0.5 * bar, 0.5 * ring[0], 0.5 * ring[1], 0.5 * ring_length
    xb = sorted({-bx, -ro, -ri, -hb, hb, ri, ro, bx})
    zb = sorted({-bz, -lz, lz, bz})
    lo, hi = 0.002, 0.5
    for _ in range(60):
        mid = np.sqrt(lo * hi)
        xs, zs = _graded_lines(xb, mid, mid, (-bx, bx)), _graded_lines(zb, mid, mid, (-bz, bz))
        if 6 * (len(xs) - 1) ** 2 * (len(zs) - 1) > target_tets:
            lo = mid
        else:
            hi = mid
    xs, zs = _graded_lines(xb, hi, hi, (-bx, bx)), _graded_lines(zb, hi, hi, (-bz, bz))
    ys = xs.copy()
    cx, cz = 0.5 * (xs[1:] + xs[:-1]), 0.5 * (zs[1:] + zs[:-1])
    X, Y, Z = np.meshgrid(cx, cx, cz, indexing="ij")
    dom = np.full(X.shape, TAG_AIR, dtype=np.int32)
    ring_m = (np.maximum(np.abs(X), np.abs(Y)) > ri) & (np.maximum(np.abs(X), np.abs(Y)) < ro) & (np.abs(Z) < lz)
    dom[ring_m] = TAG_IRON
    dom[(np.abs(X) < hb) & (np.abs(Y) < hb)] = TAG_COIL_1
    fixed = [np.flatnonzero(np.isin(np.round(a, 12), np.round(b, 12))) for a, b in ((xs, xb), (ys, xb), (zs, zb))]
    mesh = tensor_grid_mesh(xs, ys, zs, dom, jitter=jitter, seed=seed, fixed_planes=fixed)
    coil_nodes = mesh.domain_nodes_mask(TAG_COIL_1)
    z = mesh.nodes[:, 2]
    mesh.coil_terminals = {TAG_COIL_1: (np.flatnonzero(coil_nodes & (np.abs(z + bz) < 1e-12)),
                                        np.flatnonzero(coil_nodes & (np.abs(z - bz) < 1e-12)))}
    return mesh


def kuhn_microbench_mesh(nx=120, ny=120, nz=116, jitter=0.2, iron_fraction=0.4, seed=11):
    """Unit-spacing structured grid split into 6 tets per cell, jittered nodes, seeded
    per-element iron/air flags (iron with probability ``iron_fraction``)."""
    xs, ys, zs = (np.arange(n + 1, dtype=np.float64) for n in (nx, ny, nz))
    dom = np.full((nx, ny, nz), TAG_AIR, dtype=np.int32)
    mesh = tensor_grid_mesh(xs, ys, zs, dom, jitter=jitter, seed=seed)
    rng = np.random.default_rng(seed + 1)
    mesh.elem_domain = np.where(rng.random(mesh.num_elements) < iron_fraction, TAG_IRON, TAG_AIR).astype(np.int32)
    return mesh
