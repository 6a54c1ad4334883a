"""Reference-element data for first-order tetrahedra.

gmsh supplies these tables to the reference (``snoopy/finite_element.py:153-220``:
``get_quadrature_rule``, ``evaluate_basis``, ``evaluate_basis_derivative``,
``get_curl_edge_basis_functions``).  gmsh is not a dependency here, so this module
states them from the mathematics:

* reference tetrahedron with vertices (0,0,0), (1,0,0), (0,1,0), (0,0,1) and
  barycentric coordinates l0 = 1-u-v-w, l1 = u, l2 = v, l3 = w;
* lowest-order Nedelec (Whitney) edge functions w_ab = l_a grad l_b - l_b grad l_a,
  whose curl is the constant 2 grad l_a x grad l_b;
* local edges in the order (0,1), (0,2), (0,3), (1,2), (1,3), (2,3), each directed
  from its lower to its higher local vertex.

The table layouts are the ones the reference's C kernels index
(``fem_c/ctools.c:373-413`` for ``d_phi``, ``ctools.c:1058-1060`` for ``curls``):

* ``d_phi``  float64[Q, 4, 3]  gradient of each Lagrange function at each point;
* ``curls``  float64[n_orient, Q, 6, 3]  reference curls per orientation;
* ``w``      float64[Q]; ``q`` float64[Q*3] (u, v, w per point).

Orientation convention (this package's own; gmsh uses another one): orientation
``o`` of an element is a 6-bit mask, bit j set when local edge j runs against the
global edge direction (global edges run from the lower to the higher global node
index).  ``curls[o, :, j] = (-1)^bit_j * curls[0, :, j]``; 64 orientations.
"""

import math

import numpy as np

# local edge -> (local vertex a, local vertex b)
TET_EDGES = np.array([[0, 1], [0, 2], [0, 3], [1, 2], [1, 3], [2, 3]], dtype=np.int64)

# gradients of the barycentric coordinates on the reference tetrahedron
_GRAD_L = np.array([[-1.0, -1.0, -1.0],
                    [1.0, 0.0, 0.0],
                    [0.0, 1.0, 0.0],
                    [0.0, 0.0, 1.0]])

N_ORIENT = 64
NUM_EL_DOFS = 6
NUM_NODES = 4


def _conical_product_rule(n):
    """Stroud's conical product rule on the reference tetrahedron.

    n Gauss-Jacobi points per collapsed direction give n**3 points, exact for
    polynomials of total degree 2n-1 (Stroud, Approximate Calculation of
    Multiple Integrals, 1971, rule Tn:2n-1).
    """
    from scipy.special import roots_jacobi

    # map Gauss-Jacobi on [-1, 1] with weight (1-x)^alpha to [0, 1]
    xa, wa = roots_jacobi(n, 2.0, 0.0)
    xb, wb = roots_jacobi(n, 1.0, 0.0)
    xc, wc = roots_jacobi(n, 0.0, 0.0)
    a, b, c = (xa + 1) / 2, (xb + 1) / 2, (xc + 1) / 2
    wa, wb, wc = wa / 8.0, wb / 4.0, wc / 2.0
    pts, wts = [], []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                u = a[i]
                v = b[j] * (1 - a[i])
                w = c[k] * (1 - a[i]) * (1 - b[j])
                pts.append((u, v, w))
                wts.append(wa[i] * wb[j] * wc[k])
    return np.array(pts), np.array(wts)


def quadrature_rule(order):
    """Quadrature on the reference tetrahedron exact to total degree ``order``.

    Returns ``(w, q)`` like the reference's ``FiniteElement.get_quadrature_rule``
    (``snoopy/finite_element.py:153-166``): weights float64[Q] summing to 1/6 and
    points flattened float64[Q*3].

    order 1: centroid; order 2: the symmetric 4-point rule; order 3: the 5-point
    rule with a negative centroid weight; higher orders: Stroud's conical product
    rule with ceil((order+1)/2)**3 points.
    """
    order = int(order)
    if order <= 1:
        pts = np.array([[0.25, 0.25, 0.25]])
        wts = np.array([1.0 / 6.0])
    elif order == 2:
        a = (5.0 + 3.0 * math.sqrt(5.0)) / 20.0
        b = (5.0 - math.sqrt(5.0)) / 20.0
        pts = np.array([[b, b, b], [a, b, b], [b, a, b], [b, b, a]])
        wts = np.full(4, 1.0 / 24.0)
    elif order == 3:
        pts = np.array([[0.25, 0.25, 0.25],
                        [1.0 / 6, 1.0 / 6, 1.0 / 6],
                        [0.5, 1.0 / 6, 1.0 / 6],
                        [1.0 / 6, 0.5, 1.0 / 6],
                        [1.0 / 6, 1.0 / 6, 0.5]])
        wts = np.array([-4.0 / 5.0, 9.0 / 20.0, 9.0 / 20.0, 9.0 / 20.0, 9.0 / 20.0]) / 6.0
    else:
        pts, wts = _conical_product_rule((order + 2) // 2)
    return wts.astype(np.float64), pts.reshape(-1).astype(np.float64)


def barycentric(q):
    """Barycentric coordinates float64[Q, 4] of flattened local points ``q``."""
    p = np.asarray(q, dtype=np.float64).reshape(-1, 3)
    lam = np.empty((p.shape[0], 4))
    lam[:, 0] = 1.0 - p[:, 0] - p[:, 1] - p[:, 2]
    lam[:, 1:] = p
    return lam


def evaluate_basis(q):
    """Lagrange P1 basis at the points: float64[Q, 4] (``finite_element.py:34-57``)."""
    return barycentric(q)


def evaluate_basis_derivative(q):
    """Gradients of the P1 basis at the points: float64[Q, 4, 3] (``finite_element.py:59-83``)."""
    nq = np.asarray(q).reshape(-1, 3).shape[0]
    return np.ascontiguousarray(np.broadcast_to(_GRAD_L, (nq, 4, 3))).astype(np.float64)


def reference_curls():
    """Curls of the six Whitney functions on the reference element, float64[6, 3]."""
    out = np.empty((6, 3))
    for j, (a, b) in enumerate(TET_EDGES):
        out[j] = 2.0 * np.cross(_GRAD_L[a], _GRAD_L[b])
    return out


def orientation_signs(o):
    """Edge signs float64[..., 6] of orientation mask(s) ``o``."""
    o = np.asarray(o, dtype=np.int64)
    bits = (o[..., None] >> np.arange(6)) & 1
    return 1.0 - 2.0 * bits


def curl_edge_basis_functions(q):
    """Curl tables float64[64, Q, 6, 3] and the number of orientations.

    Mirrors ``FiniteElement.get_curl_edge_basis_functions``
    (``snoopy/finite_element.py:195-220``) for first-order tetrahedra.
    """
    nq = np.asarray(q).reshape(-1, 3).shape[0]
    c0 = reference_curls()
    signs = orientation_signs(np.arange(N_ORIENT))  # [64, 6]
    curls = signs[:, None, :, None] * c0[None, None, :, :]
    curls = np.broadcast_to(curls, (N_ORIENT, nq, 6, 3))
    return np.ascontiguousarray(curls), N_ORIENT


def edge_basis_functions(q):
    """Whitney functions on the reference element, float64[Q, 6, 3] (orientation 0)."""
    lam = barycentric(q)
    out = np.empty((lam.shape[0], 6, 3))
    for j, (a, b) in enumerate(TET_EDGES):
        out[:, j, :] = lam[:, a, None] * _GRAD_L[b] - lam[:, b, None] * _GRAD_L[a]
    return out


class FiniteElement:
    """First-order tetrahedron with the reference's ``FiniteElement`` method names.

    ``gmsh_code`` is accepted for signature compatibility (gmsh element type 4 is
    the 4-node tetrahedron); only that type is supported.
    """

    def __init__(self, gmsh_code=4):
        if int(gmsh_code) != 4:
            raise ValueError(f"element type {gmsh_code} not supported: only 4-node tetrahedra (type 4)")
        self.gmsh_code = 4
        self.num_nodes = 4

    def get_number_of_nodes(self):
        return 4

    def get_quadrature_rule(self, order):
        return quadrature_rule(order)

    def evaluate_basis(self, q):
        return evaluate_basis(q)

    def evaluate_basis_derivative(self, q):
        return evaluate_basis_derivative(q)

    def get_curl_edge_basis_functions(self, mesh, loc, element_type, element_order):
        if int(element_order) != 1:
            raise ValueError("only first-order edge elements are supported")
        return curl_edge_basis_functions(loc)
