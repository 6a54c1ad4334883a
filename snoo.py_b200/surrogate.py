"""Learned warm start for the nonlinear solve.

A small MLP maps a magnet's design parameters to the POD coefficients of its converged
edge-DoF vector; Newton then starts from the reconstruction instead of from zero.  The
network is trained on solutions this solver generates over a fixed-topology family
(``morph.YokeMorphFamily``).  Zero-start Newton stays the yardstick: a warm-started solve is held
to the zero-start residual target ||F_free(x)|| <= tol ||F_free(0)||, and a prediction whose
residual exceeds ||F_free(0)|| is dropped for x = 0, so the network changes iteration counts,
never the converged answer.

The MLP (9 -> 256 -> 256 -> 256 -> 128, GELU) keeps FP32 master weights and BF16 copies; its
forward and backward passes run on this library's tcgen05 GEMM (BF16 operands, FP32
accumulation, fused bias/GELU epilogue) and element-wise kernels; Adam updates the FP32
weights.  The POD basis is a setup step (float64 Gram matrix and eigendecomposition through
torch's cuBLAS/cuSOLVER calls).
"""

import ctypes
import math
import time

import numpy as np

from . import _lib
from .device import torch, upload, zeros

IN_PAD = 16  # the 9 inputs padded to a multiple of 8 (zero columns) for the GEMM's K


def _p(t):
    return _lib.ptr(t) if t is not None else None


class MLP:
    """Dense GELU network on the library's BF16 tensor-core GEMM."""

    def __init__(self, sizes=(9, 256, 256, 256, 128), seed=0):
        t = torch()
        self.sizes = list(sizes)
        self.in_dim = sizes[0]
        dims = [IN_PAD] + list(sizes[1:])
        self.dims = dims
        g = np.random.default_rng(seed)
        self.W, self.b, self.Wb, self.WTb, self.mW, self.vW, self.mb, self.vb = ([] for _ in range(8))
        for l in range(len(dims) - 1):
            fan_in = sizes[l]
            w = np.zeros((dims[l + 1], dims[l]), dtype=np.float32)
            w[:, :fan_in] = g.normal(0.0, math.sqrt(2.0 / fan_in), size=(dims[l + 1], fan_in))
            self.W.append(t.from_numpy(w).cuda())
            self.b.append(t.zeros(dims[l + 1], dtype=t.float32, device="cuda"))
            self.Wb.append(self.W[-1].to(t.bfloat16))
            self.WTb.append(self.W[-1].t().contiguous().to(t.bfloat16))
            self.mW.append(t.zeros_like(self.W[-1]))
            self.vW.append(t.zeros_like(self.W[-1]))
            self.mb.append(t.zeros_like(self.b[-1]))
            self.vb.append(t.zeros_like(self.b[-1]))
        self.step_count = 0
        self.err = t.zeros(1, dtype=t.int32, device="cuda")

    @property
    def n_layers(self):
        return len(self.W)

    def _gemm(self, A, B, C=None, H=None, bias=None, act=0):
        M, K = A.shape
        N = B.shape[0]
        _lib.call("snp_gemm_bf16", M, N, K, _p(A), A.stride(0), _p(B), B.stride(0), _p(bias), act, _p(C),
                  N if C is None else C.stride(0), _p(H), N if H is None else H.stride(0), _p(self.err),
                  _lib.stream_ptr())

    def input_bf16(self, X):
        """[B, in_dim] float -> [B, 16] BF16 with zero padding."""
        t = torch()
        Xp = t.zeros((X.shape[0], IN_PAD), dtype=t.float32, device="cuda")
        Xp[:, : self.in_dim] = X if hasattr(X, "data_ptr") else t.as_tensor(X, dtype=t.float32, device="cuda")
        return Xp.to(t.bfloat16)

    def forward(self, Xb, keep=False):
        """Xb: [B, 16] BF16.  Returns the FP32 output [B, out]; keeps activations when ``keep``."""
        t = torch()
        B = Xb.shape[0]
        H = Xb
        self.cache = [(None, Xb)]
        for l in range(self.n_layers):
            last = l == self.n_layers - 1
            Z = t.empty((B, self.dims[l + 1]), dtype=t.float32, device="cuda")
            Hn = None if last else t.empty((B, self.dims[l + 1]), dtype=t.bfloat16, device="cuda")
            self._gemm(H, self.Wb[l], C=Z, H=Hn, bias=self.b[l], act=0 if last else 1)
            if keep:
                self.cache.append((Z, Hn))
            H = Hn if not last else Z
        if not keep:
            self.cache = None
        return H

    def backward(self, dY):
        """dY: FP32 [B, out] gradient of the loss w.r.t. the output (B a multiple of 8).
        Returns per-layer (dW, db) in FP32."""
        t = torch()
        B = dY.shape[0]
        assert B % 8 == 0, "backward needs the batch padded to a multiple of 8"
        grads = [None] * self.n_layers
        dZ = dY
        dZb = t.empty(dY.shape, dtype=t.bfloat16, device="cuda")  # output layer: dZ = dY
        _lib.call("snp_f32_to_bf16", dY.numel(), _p(dY), _p(dZb), _lib.stream_ptr())
        for l in range(self.n_layers - 1, -1, -1):
            Hprev = self.cache[l][1]  # BF16 [B, in]
            dZT = t.empty((dZb.shape[1], B), dtype=t.bfloat16, device="cuda")
            _lib.call("snp_transpose_bf16", B, dZb.shape[1], _p(dZb), dZb.shape[1], _p(dZT), B, _lib.stream_ptr())
            HT = t.empty((Hprev.shape[1], B), dtype=t.bfloat16, device="cuda")
            _lib.call("snp_transpose_bf16", B, Hprev.shape[1], _p(Hprev), Hprev.shape[1], _p(HT), B,
                      _lib.stream_ptr())
            dW = t.empty_like(self.W[l])
            self._gemm(dZT, HT, C=dW)  # [out, in] = dZ^T H
            db = t.empty_like(self.b[l])
            _lib.call("snp_col_sum", B, dZ.shape[1], _p(dZ), dZ.shape[1], _p(db), _lib.stream_ptr())
            grads[l] = (dW, db)
            if l > 0:
                dH = t.empty((B, self.dims[l]), dtype=t.float32, device="cuda")
                self._gemm(dZb, self.WTb[l], C=dH)  # [B, in] = dZ W
                Zprev = self.cache[l][0]
                dZ = t.empty_like(dH)
                dZb = t.empty((B, self.dims[l]), dtype=t.bfloat16, device="cuda")
                _lib.call("snp_gelu_backward", dH.numel(), _p(dH), _p(Zprev), _p(dZb), _p(dZ), _lib.stream_ptr())
        return grads

    def adam(self, grads, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        for l, (dW, db) in enumerate(grads):
            _lib.call("snp_adam_step", self.W[l].numel(), _p(self.W[l]), _p(dW), _p(self.mW[l]), _p(self.vW[l]),
                      _p(self.Wb[l]), lr, beta1, beta2, eps, self.step_count, _lib.stream_ptr())
            _lib.call("snp_adam_step", self.b[l].numel(), _p(self.b[l]), _p(db), _p(self.mb[l]), _p(self.vb[l]),
                      None, lr, beta1, beta2, eps, self.step_count, _lib.stream_ptr())
            rows, cols = self.Wb[l].shape
            _lib.call("snp_transpose_bf16", rows, cols, _p(self.Wb[l]), cols, _p(self.WTb[l]), rows, _lib.stream_ptr())

    def train_step(self, Xb, T, lr):
        """One Adam step on the mean-squared error of a batch (B a multiple of 8)."""
        t = torch()
        Y = self.forward(Xb, keep=True)
        dY = t.empty_like(Y)
        _lib.call("snp_mse_grad", Y.numel(), _p(Y), _p(T), 2.0 / Y.numel(), _p(dY), None, _lib.stream_ptr())
        grads = self.backward(dY)
        self.adam(grads, lr=lr)
        return Y

    def check_errors(self):
        torch().cuda.synchronize()
        if int(self.err.item()) != 0:
            raise _lib.SnpError(1, "tensor-core GEMM wait timed out")


def pod(snapshots, n_modes):
    """POD of snapshot rows [S, n] (float32 or float64 CUDA tensor): mean [n], orthonormal modes
    [n, n_modes] (float64) from the float64 Gram matrix, and the snapshots' coefficients."""
    t = torch()
    S = snapshots.shape[0]
    mean = snapshots.mean(0, dtype=t.float64)
    G = t.zeros((S, S), dtype=t.float64, device="cuda")
    chunk = max(1, int(2e9 // (8 * snapshots.shape[1])))
    for i in range(0, S, chunk):
        Di = snapshots[i:i + chunk].double() - mean
        for j in range(0, S, chunk):
            Dj = snapshots[j:j + chunk].double() - mean
            G[i:i + chunk, j:j + chunk] = Di @ Dj.T
    G = 0.5 * (G + G.T)
    evals, evecs = t.linalg.eigh(G)
    order = t.argsort(evals, descending=True)[:n_modes]
    lam = evals[order].clamp_min(1e-300)
    V = evecs[:, order]
    U = t.zeros((snapshots.shape[1], n_modes), dtype=t.float64, device="cuda")
    for i in range(0, S, chunk):
        U += (snapshots[i:i + chunk].double() - mean).T @ V[i:i + chunk]
    U /= lam.sqrt()
    coeffs = t.zeros((S, n_modes), dtype=t.float64, device="cuda")
    for i in range(0, S, chunk):
        coeffs[i:i + chunk] = (snapshots[i:i + chunk].double() - mean) @ U
    energy = float((lam.sum() / evals.clamp_min(0).sum()).item())
    return mean, U, coeffs, energy


class MorphedSolver:
    """One device Newton solver serving every member of a ``YokeMorphFamily``: moving a member
    in replaces the node coordinates and the coil source field, nothing else."""

    def __init__(self, family, quad_order=2, max_newton=60, stream=None):
        from . import materials as MAT
        from . import mesh as M
        from .red_mvp_solver import RedMVPSolver

        self.family = family
        self.solver = RedMVPSolver(family.mesh, family._base_coils, [M.TAG_IRON], [M.TAG_AIR],
                                   [MAT.atan_reluctance()], max_newton_iterations=max_newton, quad_order=quad_order)
        self.solver.verbose = False
        if stream is not None:
            self.solver.stream = stream
        self.eng = self.solver.newton_engine()
        self.n = family.mesh.num_dofs
        self.max_newton = max_newton
        self._zero = zeros(self.n)[: self.n]

    def set_member(self, p):
        """Move the solver to member p; returns ||F_free(0)|| of that member."""
        from .fem_c import biot_savart_device

        t = torch()
        asm = self.solver.curl_curl_factory
        nodes = upload(np.ascontiguousarray(self.family.nodes(p)), np.float64)
        d = asm._device_state()
        d["nodes"].copy_(nodes)
        self.eng.set_nodes(nodes)
        pts = asm.get_quadrature_points_device(self.solver.quad_order, 0)
        Bs = zeros(pts.numel())[: pts.numel()]
        for segs, current, rad in self.family.coil_segments(p):
            Bs += biot_savart_device(upload(segs, np.float64), pts, current, rad)[: pts.numel()]
        self.eng.set_source(0, Bs)
        t.cuda.synchronize()
        self._nodes, self._Bs = nodes, Bs  # keep the uploads referenced while the stream uses them
        return self.eng.residual_norm(self._zero)

    def attach_basis(self, V=None, steps=1):
        """Galerkin-correct every kept start in the span of V (``WarmStart.galerkin_basis``)
        inside the solve (``snp_solver_set_galerkin_basis``); None detaches."""
        self.eng.set_galerkin_basis(V, steps)

    def solve(self, x0=None, rtol=1e-8, precision="mixed", res_ref=0.0):
        prec = {"fp64": 0, "mixed": 1}[precision]
        return self.eng.solve(x0, mode=1, tol=rtol, max_newton=self.max_newton, precision=prec, cg_maxiter=50000,
                              res_ref=res_ref)


def solve_members_at_once(msolvers, x0s, res_refs, rtol=1e-8, precision="mixed", n_threads=0):
    """One Newton solve per ``MorphedSolver`` (each already moved to its member, each on its own
    CUDA stream), all at once through ``snp_solver_solve_many``: every solve runs on a host
    thread of its own, so the GPU overlaps their kernels.  ``x0s``: starting vectors (CUDA
    float64 [n]) or None for zero starts; ``res_refs``: each member's ||F_free(0)||.
    Returns the answers (new CUDA tensors) and per-solve stats dicts."""
    k = len(msolvers)
    t = torch()
    xs = []
    for ms, x0 in zip(msolvers, x0s):
        x = zeros(ms.n)[: ms.n]
        if x0 is not None:
            x.copy_(x0)
        xs.append(x)
    t.cuda.synchronize()
    prec = {"fp64": 0, "mixed": 1}[precision]
    handles = (ctypes.c_void_p * k)(*[ms.eng.handle.value for ms in msolvers])
    xp = (ctypes.c_void_p * k)(*[x.data_ptr() for x in xs])
    opts = (_lib.SolveOpts * k)(*[_lib.SolveOpts(1, float(rtol), 50000, int(ms.max_newton), 0.1, prec, 0, 1,
                                                 float(ref)) for ms, ref in zip(msolvers, res_refs)])
    stats = (_lib.SolveStats * k)()
    status = (ctypes.c_int32 * k)()
    rc = _lib.load().snp_solver_solve_many(handles, k, xp, opts, stats, int(n_threads), status)
    t.cuda.synchronize()
    out = []
    for i in range(k):
        d = stats[i].as_dict()
        d["rel_res"] = d["res"] / res_refs[i] if res_refs[i] > 0 else 0.0
        d["status"] = int(status[i])
        out.append(d)
    if rc != 0:
        _lib.check(rc)
    return xs, out


def basis_combine(V, coef, mean=None):
    """mean + coef @ V^T on this library's kernel (``snp_basis_combine``): V CUDA float32 [n, m]
    row-major, coef CUDA float64 [P, m]; returns CUDA float64 [P, n]."""
    t = torch()
    assert V.dtype == t.float32 and V.is_cuda and V.stride(1) == 1 and coef.dtype == t.float64
    n, m = int(V.shape[0]), int(V.shape[1])
    coef = coef.reshape(-1, m).contiguous()
    P = int(coef.shape[0])
    out = t.empty((P, n), dtype=t.float64, device="cuda")
    for p0 in range(0, P, 32):
        p1 = min(P, p0 + 32)
        _lib.call("snp_basis_combine", n, _lib.ptr(V), m, int(V.stride(0)), _lib.ptr(coef[p0:p1]), p1 - p0,
                  _lib.ptr(mean), _lib.ptr(out[p0:p1]), n, _lib.stream_ptr())
    return out


class WarmStart:
    """Snapshots -> POD -> MLP; predicts starting vectors for new family members."""

    def __init__(self, msolver, n_modes=128, hidden=256, seed=0):
        self.ms = msolver
        self.n_modes = n_modes
        self.mlp = MLP((9, hidden, hidden, hidden, n_modes), seed=seed)
        self.timings = {}

    def generate(self, params, precision="mixed", rtol=1e-8, members_at_once=1):
        """Solve every member (zero start); returns float32 snapshots [S, n] and per-solve stats.
        ``members_at_once`` > 1 solves groups of members together in the batched solver
        (``batch.BatchSolver`` over that many ``MorphedSolver`` copies of the family)."""
        t = torch()
        snaps = t.empty((len(params), self.ms.n), dtype=t.float32, device="cuda")
        stats = []
        t0 = time.perf_counter()
        if members_at_once <= 1:
            for i, p in enumerate(params):
                ref = self.ms.set_member(p)
                x, st = self.ms.solve(None, rtol=rtol, precision=precision, res_ref=ref)
                snaps[i] = x.float()
                stats.append(st)
        else:
            from .batch import BatchSolver

            k = int(members_at_once)
            members = [MorphedSolver(self.ms.family, max_newton=self.ms.max_newton) for _ in range(k)]
            engines = {}
            for c0 in range(0, len(params), k):
                chunk = list(range(c0, min(c0 + k, len(params))))
                m = len(chunk)
                if m not in engines:
                    engines[m] = BatchSolver(members[:m])
                refs = [ms.set_member(params[i]) for ms, i in zip(members[:m], chunk)]
                st = engines[m].solve(rtol, precision=precision, res_refs=refs)
                for x, i in zip(engines[m].xs, chunk):
                    snaps[i] = x.float()
                stats += st
            del engines, members
        t.cuda.synchronize()
        self.timings["generate_s"] = time.perf_counter() - t0
        return snaps, stats

    def fit(self, params, snapshots, epochs=None, batch=256, lr=2e-3, seed=0, steps=6000):
        """POD of the snapshots, then Adam with a cosine-decayed learning rate for ``epochs``
        passes over the data (default: as many as make about ``steps`` steps)."""
        t = torch()
        t0 = time.perf_counter()
        self.mean, self.U, coeffs, self.pod_energy = pod(snapshots, self.n_modes)
        # one scale for every mode (not a per-mode standardisation): the network's squared
        # error then equals the DoF-space error of the reconstruction (the modes are
        # orthonormal), so training weights each mode by its energy
        self.c_mu = coeffs.mean(0)
        self.c_sd = ((coeffs - self.c_mu) ** 2).mean().sqrt().clamp_min(1e-30)
        T = ((coeffs - self.c_mu) / self.c_sd).float()
        X = self.mlp.input_bf16(t.as_tensor(np.asarray(params), dtype=t.float32, device="cuda"))
        S = len(params)
        batch = max(8, min(batch, (S // 8) * 8))
        if epochs is None:
            epochs = max(1, -(-steps // max(1, S // batch)))
        rng = np.random.default_rng(seed)
        self.history = []
        for ep in range(epochs):
            lr_ep = lr * 0.5 * (1.0 + math.cos(math.pi * ep / epochs))
            perm = rng.permutation(S)
            for i in range(0, S - batch + 1, batch):
                idx = t.as_tensor(perm[i:i + batch], device="cuda")
                Y = self.mlp.train_step(X[idx].contiguous(), T[idx].contiguous(), lr_ep)
            if ep % max(1, epochs // 10) == 0 or ep == epochs - 1:
                self.history.append((ep, float(((Y - T[idx]) ** 2).mean().item())))
        self.mlp.check_errors()
        self.timings["fit_s"] = time.perf_counter() - t0
        return self

    def predict(self, params, check=True):
        """Starting vectors [P, n] (float64, device) for parameter rows.  ``check=False`` skips
        the synchronising check of the GEMM's error flag (call ``mlp.check_errors()`` later)."""
        t = torch()
        X = self.mlp.input_bf16(t.as_tensor(np.atleast_2d(params), dtype=t.float32, device="cuda"))
        Y = self.mlp.forward(X)
        if check:
            self.mlp.check_errors()
        c = (Y.double() * self.c_sd + self.c_mu).contiguous()
        return basis_combine(self.basis_f32(), c, self.mean)

    def basis_f32(self):
        """All POD modes as a row-major float32 [n, modes] CUDA tensor (cached): the operand of
        the reconstruction kernel."""
        if getattr(self, "_U32", None) is None or self._U32.shape != self.U.shape:
            self._U32 = self.U.float().contiguous()
        return self._U32

    def project(self, x):
        """Best POD approximation of a solution (the surrogate's floor)."""
        return self.mean + ((x.double() - self.mean) @ self.U) @ self.U.T

    def galerkin_basis(self, modes):
        """The first ``modes`` POD modes as a row-major float32 [n, modes] CUDA tensor (cached)."""
        modes = int(min(modes, self.U.shape[1]))
        if getattr(self, "_gb", None) is None or self._gb.shape[1] != modes:
            self._gb = self.U[:, :modes].float().contiguous()
        return self._gb

    def correct(self, x0, msolver=None, modes=64, precision="mixed", steps=1):
        """Galerkin Newton step(s) on a warm start in the span V of the first ``modes`` POD
        modes: assemble J(x) and F(x) (matrix-free, ``precision``), solve (V^T J V) c = -V^T F
        (both from ``snp_solver_reduced_system``), x += V c.  The member must already be set on
        ``msolver`` (default: the training solver).  Returns a new float64 vector; the Newton
        solve that follows still checks it by its residual.  A singular reduced system leaves
        x unchanged."""
        t = torch()
        ms = msolver or self.ms
        V = self.galerkin_basis(modes)
        x = x0.double().clone()
        F = zeros(ms.n)[: ms.n]
        for _ in range(steps):
            ms.eng.assemble_tensors(x, precision, F)
            Jr, g = ms.eng.reduced_system(V, F, precision)
            c, info = t.linalg.solve_ex(Jr, -g)
            c = t.where(info == 0, c, t.zeros_like(c))
            x += (V @ c.float()).double()
        return x
