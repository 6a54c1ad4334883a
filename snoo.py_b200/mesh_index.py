"""Device mesh index: point location and nodal averaging for field maps.

Replaces gmsh's ``get_element_by_coordinates`` (``snoopy/evaluators.py:155-295, 297-410``)
and the Python loop of ``CurlCurlAssembler.compute_nodal_fields``
(``snoopy/curl_curl_assembler.py:2089-2196``) with the ``snp_mesh_index_*`` kernels: a
uniform bucket grid over element centroids (cell edge >= the largest element extent, so the
element holding a point lies in the 27 buckets around it) and the node -> element incidence.
"""

import ctypes

import numpy as np

from . import _lib
from .device import torch, upload, zeros


class MeshIndex:
    """Owner of an ``snp_mesh_index`` over nodes [N, 3] and cells [E, 4] (0-based)."""

    def __init__(self, nodes, cells, stream=None):
        _lib.require_cuda()
        nodes_d = nodes if hasattr(nodes, "data_ptr") else upload(nodes, np.float64)
        cells_d = cells if hasattr(cells, "data_ptr") else upload(cells, np.int32)
        self.n_nodes = int(nodes_d.numel() // 3)
        self.n_elems = int(cells_d.numel() // 4)
        h = ctypes.c_void_p()
        _lib.call("snp_mesh_index_create", _lib.ptr(nodes_d), self.n_nodes, _lib.ptr(cells_d), self.n_elems,
                  _lib.stream_ptr(stream), ctypes.byref(h))
        self.handle = h
        self.stream = stream

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.load().snp_mesh_index_destroy(h)
            except Exception:
                pass
            self.handle = None

    def info(self):
        nb = (ctypes.c_int32 * 3)()
        bmin = (ctypes.c_double * 3)()
        h = (ctypes.c_double * 3)()
        mx = ctypes.c_int32()
        _lib.call("snp_mesh_index_info", self.handle, nb, bmin, h, ctypes.byref(mx))
        return {"nb": tuple(nb), "bmin": tuple(bmin), "h": tuple(h), "max_bucket": int(mx.value)}

    def locate_device(self, points_d, tol=1e-12):
        """Device element ids (int32, -1 outside) and barycentric coordinates [P, 4]."""
        t = torch()
        n = int(points_d.numel() // 3)
        elem = t.empty(max(n, 1), dtype=t.int32, device=points_d.device)[:n]
        bary = zeros(4 * n)[: 4 * n]
        _lib.call("snp_mesh_index_locate", self.handle, _lib.ptr(points_d), n, float(tol), _lib.ptr(elem),
                  _lib.ptr(bary), _lib.stream_ptr(self.stream))
        return elem, bary.view(n, 4)

    def locate(self, points, tol=1e-12):
        """Element index (int64, -1 outside) and barycentric coordinates [P, 4] as numpy."""
        pts = upload(np.asarray(points, dtype=np.float64).reshape(-1, 3), np.float64)
        elem, bary = self.locate_device(pts, tol)
        return elem.cpu().numpy().astype(np.int64), bary.cpu().numpy()

    def nodal_average(self, elem_values_d, n_comp, elem_mask_d=None):
        """Device [N, n_comp]: per node, the mean of ``elem_values_d`` [E, n_comp] over its elements
        (those with a nonzero mask entry when a uint8 mask [E] is given); 0 where none."""
        if int(elem_values_d.numel()) < self.n_elems * int(n_comp):
            raise ValueError("elem_values needs E x n_comp values")
        if elem_mask_d is not None and int(elem_mask_d.numel()) < self.n_elems:
            raise ValueError("elem_mask needs one entry per element")
        out = zeros(self.n_nodes * n_comp)[: self.n_nodes * n_comp]
        _lib.call("snp_mesh_index_nodal_average", self.handle, _lib.ptr(elem_values_d), int(n_comp),
                  _lib.ptr(elem_mask_d), _lib.ptr(out), _lib.stream_ptr(self.stream))
        return out.view(self.n_nodes, n_comp)

    def interpolate(self, elem_d, bary_d, nodal_d, n_comp, n_sets=1, point_set_d=None):
        """Device [P, n_comp]: barycentric interpolation of nodal values (``n_sets`` stacked arrays of
        N x n_comp; ``point_set_d`` int32 [P] picks the array per point, -1 gives 0)."""
        n = int(elem_d.numel())
        if int(bary_d.numel()) < 4 * n or int(nodal_d.numel()) < int(n_sets) * self.n_nodes * int(n_comp):
            raise ValueError("bary needs 4 values per point and nodal n_sets x N x n_comp values")
        if point_set_d is not None and int(point_set_d.numel()) < n:
            raise ValueError("point_set needs one entry per point")
        out = zeros(n * n_comp)[: n * n_comp]
        _lib.call("snp_mesh_index_interpolate", self.handle, n, _lib.ptr(elem_d), _lib.ptr(bary_d), _lib.ptr(nodal_d),
                  int(n_comp), int(n_sets), _lib.ptr(point_set_d), _lib.ptr(out), _lib.stream_ptr(self.stream))
        return out.view(n, n_comp)
