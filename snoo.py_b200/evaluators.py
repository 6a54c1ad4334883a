"""Field-map evaluation with the reference's interface (``snoopy/evaluators.py``).

Points are located on the device mesh index (``mesh_index.MeshIndex``: bucket grid + barycentric
test) instead of gmsh's ``get_element_by_coordinates``; ``gmsh_model`` is the ``TetMesh`` the
solvers use.  A point counts as inside the volumes ``vol_tags`` when the element holding it
belongs to one of them (the reference asks gmsh's ``is_inside`` per volume first).
"""

import numpy as np

from . import _lib
from . import finite_element as fe
from .device import torch, upload, zeros


def _located(mesh, positions, vol_tags):
    """Device element ids (-1 outside the volumes), barycentric coordinates and the index of
    each point's volume in ``vol_tags`` (-1 outside)."""
    pts = upload(np.asarray(positions, dtype=np.float64).reshape(-1, 3), np.float64)
    elem, bary = mesh.index().locate_device(pts)
    el = elem.cpu().numpy().astype(np.int64)
    dom = np.full(len(el), -1, dtype=np.int32)
    ok = el >= 0
    tags = list(vol_tags)
    lookup = {t: i for i, t in enumerate(tags)}
    dom[ok] = [lookup.get(int(t), -1) for t in mesh.elem_domain[el[ok]]]
    el[dom < 0] = -1
    return upload(el, np.int32), bary, upload(dom, np.int32), el


def evaluate_curl_curl_solution(positions, gmsh_model, vol_tags, solution, glob_ids=None):
    """B = curl A at ``positions`` [M, 3] inside the volumes ``vol_tags`` (0 elsewhere), for the
    vector potential ``solution`` (``evaluators.py:155-295``).  ``glob_ids`` is accepted for the
    reference's signature; the mesh's own edge ids are used."""
    mesh = gmsh_model
    el_d, _, _, _ = _located(mesh, positions, vol_tags)
    n = int(el_d.numel())
    w, q = fe.quadrature_rule(1)
    d_phi = upload(fe.evaluate_basis_derivative(q), np.float64)
    curls, n_orient = fe.curl_edge_basis_functions(q)
    curls_d = upload(curls, np.float64)
    nodes_d = upload(mesh.nodes, np.float64)
    cells_d, gids_d, or_d = (upload(mesh.cells, np.int32), upload(mesh.elem_edges, np.int32),
                             upload(mesh.orientations, np.int32))
    x_d = solution if hasattr(solution, "data_ptr") else upload(solution, np.float64)
    B = zeros(3 * n)
    _lib.call("snp_b_at_elements", n, _lib.ptr(el_d), _lib.ptr(nodes_d), _lib.ptr(cells_d), _lib.ptr(gids_d),
              _lib.ptr(or_d), _lib.ptr(curls_d), n_orient, _lib.ptr(d_phi), len(w), _lib.ptr(x_d), _lib.ptr(B),
              _lib.stream_ptr())
    return B[: 3 * n].cpu().numpy().reshape(-1, 3)


def evaluate_interpolation(positions, gmsh_model, vol_tags, nodal_values):
    """Linear interpolation of nodal values at ``positions`` (``evaluators.py:297-410``):
    a point in volume ``vol_tags[j]`` interpolates ``nodal_values[j]`` ([N] or [N, C]).
    Returns [M, C] (C = 1 for scalar values); 0 outside the volumes."""
    mesh = gmsh_model
    t = torch()
    el_d, bary, dom_d, _ = _located(mesh, positions, vol_tags)
    first = np.asarray(nodal_values[0] if not hasattr(nodal_values[0], "data_ptr") else nodal_values[0].cpu().numpy())
    nc = 1 if first.ndim == 1 else first.shape[1]
    stack = []
    for v in nodal_values:
        v_d = v if hasattr(v, "data_ptr") else upload(np.asarray(v, dtype=np.float64), np.float64)
        if int(v_d.numel()) != mesh.num_nodes * nc:
            raise ValueError(f"every nodal value set needs {mesh.num_nodes} x {nc} values")
        stack.append(v_d.reshape(-1))
    nodal_d = t.cat(stack) if len(stack) > 1 else stack[0].contiguous()
    out = mesh.index().interpolate(el_d, bary, nodal_d, nc, len(stack), dom_d)
    return out.cpu().numpy()


def evaluate_fem_solution_node_interpolation(gmsh_model, points, solver, coil_list, x, domain_list):
    """B at ``points`` by interpolating nodal averages (``evaluators.py:413-454``): per domain of
    ``domain_list`` the element fields averaged at the nodes plus the coils' field at the nodes."""
    nodes = solver.curl_curl_factory.nodes
    b_coil = 0.0 * nodes
    for coil in coil_list:
        b_coil = b_coil + coil.compute_B(nodes)
    b_node_list = [solver.curl_curl_factory.compute_nodal_fields(x, [indx]) + b_coil for indx in domain_list]
    return evaluate_interpolation(points, gmsh_model, domain_list, b_node_list)
