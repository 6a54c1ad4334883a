"""Many magnet variants solved together.

Each variant is its own device solver (its own mesh, materials, source and CSR/element
topology) created on its own CUDA stream.  Two ways to solve them together:

* ``BatchSolver``: one batched solver over all variants (``snp_batch_*``): concatenated element
  and DoF arrays with per-variant offsets, one launch per pass over all variants, per-variant
  Newton / CG / line-search state on the device, the whole Newton loop one CUDA graph, launch
  shapes from its autotuner.  A variant's answer does not depend on what else is batched.
* ``solve_many``: ``snp_solver_solve_many`` runs every variant's own Newton solve on a host
  thread of its own so the GPU overlaps the variants' kernels.  Every instance's solve is
  deterministic, so these answers are identical to one-at-a-time solves.

Variant family (seeded): window-frame yokes with outer width U[0.4, 0.9] m, aperture width
U[0.1, 0.4] m (capped so each leg keeps 5 cm), length U[0.3, 2.0] m, coil current density
U[1, 5] A/mm^2, iron saturation Js U[1.6, 2.1] T and mu_r U[1000, 5000], meshed at
U[30k, 600k] tets.  Even-numbered instances use the reduced-potential path (racetrack
filament coils, Biot-Savart source field); odd-numbered ones the total-potential path with a
conductor bar through an iron ring of the same widths and length, whose source rhs comes from
the grad-grad Laplace solve of the conductor's electric potential.
"""

import ctypes

import numpy as np

from . import _lib
from . import materials as MAT
from . import mesh as M
from .device import torch, zeros

RANGES = {"outer_w": (0.4, 0.9), "ap_w": (0.1, 0.4), "length": (0.3, 2.0), "J": (1e6, 5e6), "Js": (1.6, 2.1),
          "mu_r": (1000.0, 5000.0), "tets": (30e3, 600e3)}


def sample_variants(n=128, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        v = {k: float(rng.uniform(*r)) for k, r in RANGES.items()}
        v["ap_w"] = min(v["ap_w"], v["outer_w"] - 0.1)
        v["tets"] = int(v["tets"])
        v["kind"] = "reduced" if i % 2 == 0 else "total"
        v["index"] = i
        out.append(v)
    return out


class Instance:
    """One variant: its solver object, Newton engine, stream and solution buffer."""

    def __init__(self, v, quad_order=2, max_newton=60):
        from .mvp_solver import MVPSolver
        from .red_mvp_solver import RedMVPSolver

        t = torch()
        self.v = v
        self.stream = t.cuda.Stream()
        rel = MAT.atan_reluctance(mu_r=v["mu_r"], Js=v["Js"])
        if v["kind"] == "reduced":
            ow, ap, L = v["outer_w"], v["ap_w"], v["length"]
            g = M.WindowFrameGeometry(outer_w=ow, outer_h=ow, ap_w=ap, ap_h=ap * 2.0 / 3.0, length=L,
                                      box=(ow + 0.4, ow + 0.4, L + 0.7), current_density=v["J"])
            self.mesh = M.window_frame_mesh(v["tets"], jitter=0.15, seed=7 + v["index"], geometry=g)
            self.solver = RedMVPSolver(self.mesh, g.coils(), [M.TAG_IRON], [M.TAG_AIR], [rel],
                                       max_newton_iterations=max_newton, quad_order=quad_order)
            self.solver.verbose = False
            self.solver.stream = self.stream
            self.eng = self.solver.newton_engine()
        else:
            ow, ap, L = v["outer_w"], v["ap_w"], v["length"]
            box = (ow + 0.3, ow + 0.3, L + 0.4)
            self.mesh = M.bar_conductor_mesh(v["tets"], seed=3 + v["index"], box=box, bar=0.5 * ap,
                                             ring=(ap, ow), ring_length=L)
            t1, t2 = self.mesh.coil_terminals[M.TAG_COIL_1]
            self.solver = MVPSolver(self.mesh, [M.TAG_COIL_1], [M.TAG_IRON], [M.TAG_AIR], [(t1, t2)], [rel],
                                    quad_order=quad_order, max_newton_iterations=max_newton)
            self.solver.verbose = False
            self.solver.stream = self.stream
            self.phi = v["J"] * box[2]  # potential difference driving J along the bar
            self.eng = self.solver._engine([self.phi])
        self.n = self.mesh.num_dofs
        self.x = zeros(self.n)[: self.n]
        self.max_newton = max_newton

    @property
    def num_elements(self):
        return self.mesh.num_elements

    def opts(self, rtol, precision):
        return _lib.SolveOpts(1, float(rtol), 50000, int(self.max_newton), 0.1, {"fp64": 0, "mixed": 1}[precision], 0,
                              1, 0.0)


def solve_many(instances, rtol=1e-8, precision="fp64", n_threads=0):
    """Zero-start Newton on every instance at once; returns per-instance stats dicts."""
    t = torch()
    for ins in instances:
        ins.x.zero_()
    t.cuda.synchronize()
    k = len(instances)
    handles = (ctypes.c_void_p * k)(*[ins.eng.handle.value for ins in instances])
    xs = (ctypes.c_void_p * k)(*[ins.x.data_ptr() for ins in instances])
    opts = (_lib.SolveOpts * k)(*[ins.opts(rtol, precision) for ins in instances])
    stats = (_lib.SolveStats * k)()
    status = (ctypes.c_int32 * k)()
    rc = _lib.load().snp_solver_solve_many(handles, k, xs, opts, stats, int(n_threads), status)
    t.cuda.synchronize()
    out = []
    for i in range(k):
        d = stats[i].as_dict()
        d["rel_res"] = d["res"] / d["res0"] if d["res0"] > 0 else 0.0
        d["status"] = int(status[i])
        out.append(d)
    if rc != 0:
        _lib.check(rc)
    return out


class BatchSolver:
    """Many problems in one batched device solver (``snp_batch_*``): their element and DoF arrays
    concatenated, one launch per pass over all of them, each problem's Newton / CG / line-search
    state on the device and the whole Newton loop as one CUDA graph.

    ``members``: objects with a Newton engine ``eng`` (``Instance``, ``surrogate.MorphedSolver``)
    or engines themselves; a member's ``x`` (when it has one) receives its answer, otherwise
    the batch holds a buffer (``xs``).  The members' own solvers stay the source of their
    meshes, materials and source fields, so they must outlive this object.  Every member's
    answer is bitwise the one it gets in a batch of its own."""

    def __init__(self, members, max_newton=60):
        t = torch()
        t.cuda.synchronize()
        self.members = list(members)
        self.engines = [m.eng if hasattr(m, "eng") else m for m in self.members]
        self.xs = [m.x if hasattr(m, "x") else zeros(e.n)[: e.n] for m, e in zip(self.members, self.engines)]
        self.max_newton = [int(getattr(m, "max_newton", max_newton)) for m in self.members]
        k = len(self.engines)
        handles = (ctypes.c_void_p * k)(*[e.handle.value for e in self.engines])
        h = ctypes.c_void_p()
        _lib.call("snp_batch_create", handles, k, ctypes.byref(h))
        self.handle = h

    def tune(self, precision="fp64"):
        """Run the autotuner (element-pass block size, assembly grid) on this batch."""
        _lib.call("snp_batch_tune", self.handle, {"fp64": 0, "mixed": 1}[precision])
        return self.info()

    def info(self):
        inf = _lib.BatchInfo()
        _lib.call("snp_batch_get_info", self.handle, ctypes.byref(inf))
        return inf.as_dict()

    def solve(self, rtol=1e-8, precision="fp64", x0s=None, res_refs=None, raise_on_failure=True):
        """Residual-mode Newton of every member at once, from zero or from ``x0s`` (CUDA float64
        vectors or None); ``res_refs`` (per member, > 0) replaces ||F_free(x0)|| in the stopping
        rule and drops starts worse than x = 0.  Answers in ``xs``; returns per-member stats."""
        t = torch()
        k = len(self.engines)
        for i, x in enumerate(self.xs):
            if x0s is not None and x0s[i] is not None:
                x.copy_(x0s[i])
            else:
                x.zero_()
        t.cuda.synchronize()
        xp = (ctypes.c_void_p * k)(*[x.data_ptr() for x in self.xs])
        prec = {"fp64": 0, "mixed": 1}[precision]
        opts = (_lib.SolveOpts * k)()
        for i in range(k):
            ref = float(res_refs[i]) if res_refs is not None else 0.0
            opts[i] = _lib.SolveOpts(1, float(rtol), 50000, self.max_newton[i], 0.1, prec, 0, 1, ref)
        stats = (_lib.SolveStats * k)()
        status = (ctypes.c_int32 * k)()
        rc = _lib.load().snp_batch_solve(self.handle, xp, opts, stats, status)
        out = []
        for i in range(k):
            d = stats[i].as_dict()
            ref = res_refs[i] if (res_refs is not None and res_refs[i] > 0) else d["res0"]
            d["rel_res"] = d["res"] / ref if ref > 0 else 0.0
            d["status"] = int(status[i])
            out.append(d)
        if rc != 0 and raise_on_failure:
            _lib.check(rc)
        return out

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None and _lib._lib is not None:
                _lib.load().snp_batch_destroy(self.handle)
        except Exception:
            pass
        self.handle = None


def solve_one_by_one(instances, rtol=1e-8, precision="fp64"):
    """The same solves, one instance after another (each on its own stream)."""
    t = torch()
    out = []
    for ins in instances:
        ins.x.zero_()
        t.cuda.synchronize()
        _, st = ins.eng.solve(None, mode=1, tol=rtol, max_newton=ins.max_newton, cg_maxiter=50000,
                              precision={"fp64": 0, "mixed": 1}[precision], x_out=ins.x)
        out.append(st)
    t.cuda.synchronize()
    return out
