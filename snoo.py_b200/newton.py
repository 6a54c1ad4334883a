"""Device Newton solver: Python owner of the native ``snp_solver`` handle."""

import ctypes
import os

import numpy as np

from . import _lib
from .device import torch, upload, zeros

MODE_REFERENCE = 0  # increment test + scipy-style CG (red_mvp_solver.py:121-224)
MODE_RESIDUAL = 1   # ||F_free|| <= tol * ||F_free(x0)||

BLOCK_MAX = 8    # DoFs per block-Jacobi block
BLOCK_TILE = 256  # blocks never cross a multiple of this (the DoF pass's shared-memory tile)


def dof_blocks(keys, free, max_block=BLOCK_MAX, tile=BLOCK_TILE):
    """Block-Jacobi partition: maximal runs of consecutive free DoFs with equal ``keys`` (for
    edge DoFs numbered by their lower node, the edges that share that node), cut into pieces of
    at most ``max_block`` DoFs and at multiples of ``tile``; a constrained DoF is a block of its
    own.  Returns uint16 [n]: offset of the DoF in its block | block size << 8."""
    keys = np.asarray(keys)
    free = np.asarray(free).astype(bool)
    n = len(keys)
    idx = np.arange(n)
    start = np.ones(n, dtype=bool)
    if n > 1:
        start[1:] = (keys[1:] != keys[:-1]) | ~free[1:] | ~free[:-1]
    start[::tile] = True
    run_start = idx[start][np.cumsum(start) - 1]
    start |= (idx - run_start) % max_block == 0
    block = np.cumsum(start) - 1
    starts = idx[start]
    sizes = np.diff(np.r_[starts, n])
    return ((idx - starts[block]) | (sizes[block] << 8)).astype(np.uint16)


class DeviceNewton:
    """Newton solver over a ``CurlCurlAssembler``'s materials, Dirichlet mask and source fields.

    Everything (mesh arrays, CSR pattern, Jacobian, work vectors) lives on the device; a
    solve returns a float64 CUDA tensor.
    """

    def __init__(self, assembler, free_mask, source_fields=(), quad_order=2, rhs_extra=None, stream=None):
        _lib.require_cuda()
        if stream is not None:
            # inputs uploaded on torch's current stream must be complete before the solver's
            # own stream copies them
            torch().cuda.synchronize()
        self.assembler = assembler
        self.n = assembler.num_dofs
        d = assembler._device_state()
        tb = assembler.tables(quad_order)
        self.tables = tb
        self.free_mask = free_mask if hasattr(free_mask, "data_ptr") else upload(np.asarray(free_mask, dtype=np.uint8), np.uint8)
        self._stream = stream
        h = ctypes.c_void_p()
        _lib.call("snp_solver_create", self.n, _lib.ptr(d["nodes"]), assembler.nodes.shape[0], _lib.ptr(tb.curls_d),
                  tb.n_orient, _lib.ptr(tb.d_phi_d), _lib.ptr(tb.w_d), tb.nq, _lib.ptr(self.free_mask),
                  _lib.stream_ptr(stream), ctypes.byref(h))
        self.handle = h
        bs = assembler.upload_source_fields(source_fields)
        for n, m in enumerate(d["mats"]):
            n_int, rc, rx = d["rel"][n]
            _lib.call("snp_solver_add_material", self.handle, _lib.ptr(m["cells"]), _lib.ptr(m["gids"]),
                      _lib.ptr(m["orient"]), m["count"], n_int, _lib.ptr(rc), _lib.ptr(rx), _lib.ptr(bs[n]))
        # diluted steel (CurlCurlAssemblerDiluted): the factor s(z) enters every assembly
        for n, dil in enumerate(getattr(assembler, "dilutions", [])[: len(d["mats"])]):
            if dil is not None:
                coef = (ctypes.c_double * 4)(dil.c_num, dil.m_num, dil.c_den, dil.m_den)
                _lib.call("snp_solver_set_dilution", self.handle, n, _lib.ptr(tb.phi_d), coef)
        if rhs_extra is not None:
            r = rhs_extra if hasattr(rhs_extra, "data_ptr") else upload(rhs_extra, np.float64)
            _lib.call("snp_solver_set_rhs", self.handle, _lib.ptr(r))
        _lib.call("snp_solver_finalize", self.handle)
        # block Jacobi over the edges that share their lower node (DoF i = mesh edge i), unless
        # SNP_PRECOND=jacobi or the layout is not matrix-free
        self.block_jacobi = False
        mesh = getattr(assembler, "mesh", None)
        edges = getattr(mesh, "edges", None)
        if (os.environ.get("SNP_PRECOND", "block").lower() != "jacobi" and edges is not None
                and len(edges) == self.n and self.jacobian_layout == "elem"):
            fm = self.free_mask.cpu().numpy().astype(bool)
            self._set_blocks(dof_blocks(edges[:, 0], fm))
        p = ctypes.c_void_p()
        _lib.call("snp_solver_pattern", self.handle, ctypes.byref(p))
        from .device import Pattern

        self.pattern = Pattern(None, 0, 6, self.n, handle=p, owned=False)

    def solve(self, x0=None, mode=MODE_RESIDUAL, tol=1e-8, cg_maxiter=-1, max_newton=25, cg_rtol=None, precision=0,
              verbose=False, x_out=None, raise_on_failure=True, line_search=None, res_ref=0.0):
        """Run Newton from ``x0`` (zeros if None).  Returns (x CUDA tensor, stats dict).

        ``line_search`` (default: on in residual mode, off in reference mode) takes the step
        length where the energy slope F(x + a h).h has halved.  ``res_ref`` > 0 (residual mode)
        replaces ||F_free(x0)|| in the stopping rule, e.g. ||F_free(0)|| so that a warm start is
        held to the zero-start target; a start whose residual exceeds it is replaced by 0."""
        if line_search is None:
            line_search = mode == MODE_RESIDUAL
        t = torch()
        if x_out is None:
            x = zeros(self.n)[: self.n]
        else:
            x = x_out
        if x0 is not None:
            src = x0 if hasattr(x0, "data_ptr") else t.from_numpy(np.ascontiguousarray(x0, dtype=np.float64))
            x.copy_(src.to(x.device, non_blocking=True))
        else:
            x.zero_()
        if cg_rtol is None:
            cg_rtol = 1e-5 if mode == MODE_REFERENCE else 0.1
        if self._stream is not None:
            t.cuda.current_stream().synchronize()  # x was prepared on torch's stream
        opts = _lib.SolveOpts(int(mode), float(tol), int(cg_maxiter), int(max_newton), float(cg_rtol), int(precision),
                              1 if verbose else 0, 1 if line_search else 0, float(res_ref))
        st = _lib.SolveStats()
        rc = _lib.load().snp_solver_solve(self.handle, _lib.ptr(x), ctypes.byref(opts), ctypes.byref(st))
        self._leave()
        stats = st.as_dict()
        ref = res_ref if res_ref > 0 else stats["res0"]
        stats["rel_res"] = stats["res"] / ref if ref > 0 else 0.0
        if rc != 0 and (raise_on_failure or rc not in (3,)):
            _lib.check(rc)
        stats["converged"] = rc == 0
        return x, stats

    def _enter(self):
        """Work queued on torch's current stream (inputs of the next call) precedes the solver's
        own stream."""
        if self._stream is not None:
            self._stream.wait_stream(torch().cuda.current_stream())

    def _leave(self):
        """Torch's current stream waits for what the last call queued on the solver's stream."""
        if self._stream is not None:
            torch().cuda.current_stream().wait_stream(self._stream)

    def assemble(self, x, K=False, J=True, rhs=False, F=True):
        x_d = x if hasattr(x, "data_ptr") else upload(x, np.float64)
        nnz = self.pattern.nnz
        out = {"K": zeros(nnz) if K else None, "J": zeros(nnz) if J else None, "rhs": zeros(self.n) if rhs else None,
               "F": zeros(self.n) if F else None}
        self._enter()
        _lib.call("snp_solver_assemble", self.handle, _lib.ptr(x_d), _lib.ptr(out["K"]), _lib.ptr(out["J"]),
                  _lib.ptr(out["rhs"]), _lib.ptr(out["F"]), _lib.stream_ptr(self._stream))
        self._leave()
        return out

    @property
    def jacobian_layout(self):
        """Storage of the residual-mode Newton loop's Jacobian, chosen when the solver was
        finalized from the environment variable SNP_JACOBIAN: "elem" (matrix-free element
        tensors, the default), "csr" or "sell" (SELL-C-sigma, C=32, sigma=256)."""
        v = ctypes.c_int(-1)
        _lib.call("snp_solver_jacobian_layout", self.handle, ctypes.byref(v))
        return {0: "csr", 1: "sell", 2: "elem"}[v.value]

    def set_nodes(self, nodes_dev):
        """Move the mesh nodes (device float64 [N, 3]); topology, pattern and materials stay."""
        self._enter()
        _lib.call("snp_solver_set_nodes", self.handle, _lib.ptr(nodes_dev), _lib.stream_ptr(self._stream))
        self._leave()

    def set_source(self, material, B_s_dev):
        """Replace material ``material``'s source field (device float64 [E_m * Q * 3])."""
        self._enter()
        _lib.call("snp_solver_set_source", self.handle, int(material), _lib.ptr(B_s_dev), _lib.stream_ptr(self._stream))
        self._leave()

    def residual_norm(self, x):
        """||F_free(x)|| (float64), via the matrix-free assembly."""
        t = torch()
        F = zeros(self.n)[: self.n]
        self.assemble_tensors(x, "fp64", F)
        fm = self.free_mask.to(t.bool)
        return float(t.linalg.vector_norm(F[fm]).item())

    def assemble_tensors(self, x, precision="fp64", F=None):
        """Matrix-free Newton assembly at x (element tensors of J(x), and F(x) into ``F`` when
        given); afterwards ``jacobian_apply(..., precision)`` applies J(x)."""
        x_d = x if hasattr(x, "data_ptr") else upload(x, np.float64)
        self._enter()
        _lib.call("snp_solver_assemble_tensors", self.handle, _lib.ptr(x_d), {"fp64": 0, "mixed": 1}[precision],
                  _lib.ptr(F), _lib.stream_ptr(self._stream))
        self._leave()
        return F

    def jacobian_apply(self, x, y, precision="fp64"):
        """y = J x on the free DoFs with the Newton Jacobian of the last solve of that precision
        ("fp64": float64 vectors; "mixed": the float32 Jacobian and float32 vectors)."""
        prec = {"fp64": 0, "mixed": 1}[precision]
        self._enter()
        _lib.call("snp_solver_jacobian_apply", self.handle, prec, _lib.ptr(x), _lib.ptr(y),
                  _lib.stream_ptr(self._stream))
        self._leave()
        return y

    def reduced_system(self, V, F=None, precision="fp64"):
        """Galerkin system in the span of V (CUDA float32 [n, m], row-major, m <= 128) with the
        Jacobian of the last ``assemble_tensors`` of that precision: (V^T J V [m, m], V^T F [m]
        or None), float64 on the device, summed in a fixed order."""
        t = torch()
        assert V.dtype == t.float32 and V.is_cuda and V.dim() == 2 and V.stride(1) == 1 and V.shape[0] == self.n
        m = int(V.shape[1])
        Jr = t.empty((m, m), dtype=t.float64, device="cuda")
        g = t.empty(m, dtype=t.float64, device="cuda") if F is not None else None
        self._enter()
        _lib.call("snp_solver_reduced_system", self.handle, {"fp64": 0, "mixed": 1}[precision], _lib.ptr(V), m,
                  int(V.stride(0)), _lib.ptr(F), _lib.ptr(Jr), _lib.ptr(g), _lib.stream_ptr(self._stream))
        self._leave()
        return Jr, g

    def _set_blocks(self, meta):
        if meta is None:
            _lib.call("snp_solver_set_block_jacobi", self.handle, None)
            self.block_jacobi = False
            return
        meta = np.ascontiguousarray(meta, dtype=np.uint16)
        assert meta.shape == (self.n,)
        _lib.call("snp_solver_set_block_jacobi", self.handle, meta.ctypes.data_as(ctypes.c_void_p))
        self.block_jacobi = True

    def set_preconditioner(self, kind="block", meta=None):
        """Residual-mode Krylov preconditioner: "block" (block Jacobi; ``meta`` from
        ``dof_blocks``, default the edges sharing their lower node) or "jacobi" (point Jacobi,
        as the reference)."""
        if kind == "jacobi":
            self._set_blocks(None)
        else:
            if meta is None:
                fm = self.free_mask.cpu().numpy().astype(bool)
                meta = dof_blocks(self.assembler.mesh.edges[:, 0], fm)
            self._set_blocks(meta)

    def set_krylov(self, method="cg", restart=30):
        """Krylov method of the residual-mode Newton steps: "cg" (default) or "gmres"
        (restarted GMRES(``restart``), right-preconditioned, float64 solves only)."""
        _lib.call("snp_solver_set_krylov", self.handle, {"cg": 0, "gmres": 1}[method], int(restart))

    def precond_apply(self, r, precision="fp64"):
        """z = M r (CUDA float64 [n]) with the block Jacobi of the last ``assemble_tensors`` of
        that precision; returns (z, number of blocks that fell back to point Jacobi)."""
        t = torch()
        z = t.empty_like(r)
        fb = ctypes.c_int32(0)
        self._enter()
        _lib.call("snp_solver_precond_apply", self.handle, {"fp64": 0, "mixed": 1}[precision], _lib.ptr(r),
                  _lib.ptr(z), ctypes.byref(fb), _lib.stream_ptr(self._stream))
        self._leave()
        return z, int(fb.value)

    def set_galerkin_basis(self, V=None, steps=1):
        """Attach a basis (CUDA float32 [n, m], row-major, m <= 128) whose Galerkin Newton step
        corrects every kept start of the residual-mode solves (up to ``steps`` steps, each kept
        only when it lowers ||F_free||); None detaches.  The tensor is held while attached."""
        t = torch()
        if V is None:
            _lib.call("snp_solver_set_galerkin_basis", self.handle, None, 0, 0, 0)
            self._galerkin_V = None
            return
        assert V.dtype == t.float32 and V.is_cuda and V.dim() == 2 and V.stride(1) == 1 and V.shape[0] == self.n
        _lib.call("snp_solver_set_galerkin_basis", self.handle, _lib.ptr(V), int(V.shape[1]), int(V.stride(0)),
                  int(steps))
        self._galerkin_V = V

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None and _lib._lib is not None:
                _lib.load().snp_solver_destroy(self.handle)
        except Exception:
            pass
        self.handle = None
