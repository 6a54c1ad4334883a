"""Benchmark: nonlinear magnetostatic solves per second to a 1e-8 relative Newton residual.

Workload (seeded, synthetic; no dataset): window-frame iron yoke (outer 0.6 x 0.6 m, aperture
0.3 x 0.2 m, 0.5 m long) in a 1.0 x 1.0 x 1.2 m air box, two racetrack filament coils around
the vertical legs at J = 3 A/mm^2, iron reluctivity from the atan B(H) law (mu_r 3000,
Js 1.9 T) as a 40-knot PCHIP, first-order Nedelec tetrahedra (~1.2M tets), 4-point rule,
n x A = 0 on the box, reduced vector potential formulation.  One step = one full Newton
solve from A = 0 until ||F_free|| <= 1e-8 ||F_free(0)|| (F = K(A) A - rhs(A)).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun): every rank solves its own copy (independent replicas, weak scaling);
the only communication is the timing barrier and a max over ranks.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Nonlinear solves/s to 1e-8 residual @1.2M tets: plain FP64 vs mixed+warm-start"
UNIT = "solves/s"
RTOL = 1e-8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--tets", type=int, default=1_200_000)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the assembly microbenchmark, the 4M-tet mixed-precision accuracy run and the "
                         "warm-start study at the bench size")
    ap.add_argument("--batched", action="store_true",
                    help="only the batched-variants study (128 seeded yoke variants, 30k-600k tets, half "
                         "reduced, half total potential); prints its own JSON line")
    ap.add_argument("--warm-start-family", action="store_true",
                    help="only the learned-warm-start study on the 300k-tet morphed family "
                         "(4000 training / 500 held-out members); prints its own JSON line")
    ap.add_argument("--assembly-grid", type=int, default=0, metavar="G",
                    help="only the assembly microbenchmark on a G x G x round(G*116/120) grid x 6 tets "
                         "(120: the 10M-tet configuration); prints its own JSON line")
    ap.add_argument("--gemm", type=int, nargs=3, default=None, metavar=("M", "N", "K"),
                    help="only the surrogate's BF16 tensor-core GEMM C = A B^T at M x N x K; prints its "
                         "own JSON line")
    return ap.parse_args()


def workload(tets):
    from snoopy_b200 import materials as MAT
    from snoopy_b200 import mesh as M

    msh = M.window_frame_mesh(tets, jitter=0.15, seed=7)
    return msh, msh.geometry.coils(), MAT.atan_reluctance()


def oracle_problem(tets):
    """The workload set up for the CPU oracle with the reference's C kernels (``oracle/_ref``):
    mesh, coils, reluctance, quadrature tables, the per-material assembler, the free-DoF mask,
    the iron quadrature points and the source fields there."""
    import oracle as O

    import snoopy_b200 as S
    from snoopy_b200 import finite_element as FE
    from snoopy_b200 import mesh as M

    msh, coils, rel = workload(tets)
    w, q = FE.quadrature_rule(2)
    dphi = FE.evaluate_basis_derivative(q)
    phi = FE.evaluate_basis(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    iron = msh.domain_elements(M.TAG_IRON)
    air = msh.domain_elements(M.TAG_AIR)
    mats = [dict(cells=msh.cells[iron], glob_ids=msh.elem_edges[iron], orientations=msh.orientations[iron],
                 reluctance=rel),
            dict(cells=msh.cells[air], glob_ids=msh.elem_edges[air], orientations=msh.orientations[air],
                 reluctance=S.ConstantReluctance(0.25 / np.pi * 1e7))]
    pts = np.einsum("qi,eid->eqd", phi, msh.nodes[msh.cells[iron]]).reshape(-1, 3)
    Bs = sum(O.compute_B_line_segs_cpp(c.get_segments(), pts, c.current, c.rad, backend="ref") for c in coils)
    A = O.OracleCurlCurlAssembler(msh.nodes, mats, msh.num_dofs, w, q, dphi, curls, backend="ref")
    mask = np.ones(msh.num_dofs, bool)
    mask[msh.get_edge_boundary_dofs() - 1] = False
    return dict(msh=msh, coils=coils, rel=rel, w=w, q=q, dphi=dphi, phi=phi, curls=curls, A=A, mask=mask,
                iron_points=pts, sf=[Bs, np.zeros((0, 3))])


# ---------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples (every 200 ms) of SM clock, power and throttle reasons."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = np.array([float(r[1]) for r in rows])
        mx = float(rows[0][2])
        power = np.array([float(r[3]) for r in rows if r[3] not in ("[N/A]", "")] or [0.0])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        load = sm[sm > 0.5 * mx] if (sm > 0.5 * mx).any() else sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows),
                "power_w_max": float(power.max())}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------- our arm

def bytes_spmv(nnz, n, vb=8, xb=8):
    """Algorithmic bytes of y = A x on a CSR with int32 indices: values+columns nnz*(vb+4),
    row pointers (n+1)*4, x read once and y written once (2n*xb)."""
    return nnz * (vb + 4) + (n + 1) * 4 + 2 * n * xb


def bytes_pcg_iteration(nnz, n, vb=8, xb=8):
    """One Jacobi-PCG iteration: the SpMV plus 9n*xb of fused vector streams (update: r, q,
    dinv, x, p read; r, z, x written; direction update: p read and written, z read)."""
    return bytes_spmv(nnz, n, vb, xb) + 9 * n * xb


def bytes_elem_apply(ne, n, tb=8):
    """y = J x with the matrix-free Jacobian: per element its six DoF words, six tensor
    entries and six incidence-slot indices (6*4 + 6*tb + 6*4), per DoF the slot-range pointer,
    x read once and y written once.  The edge terms passed between the two passes through
    their slots (6*tb per element, written and read) are an intermediate and not counted."""
    return ne * (24 + 6 * tb + 24) + (n + 1) * 4 + 2 * n * tb


def bytes_elem_pcg_iteration(ne, n, tb=8, block_jacobi=False):
    """One matrix-free PCG iteration (element pass + DoF pass): the operator data as in
    bytes_elem_apply; per DoF {z, p}, {r, x} and 1/diag read once, {z, p} and {r, x} written
    once (9 words).  With block Jacobi the DoF pass reads the DoF's row of its block inverse
    (8 float32) and its block word (2 B) in place of 1/diag."""
    if block_jacobi:
        return ne * (24 + 6 * tb + 24) + (n + 1) * 4 + 8 * n * tb + 34 * n
    return ne * (24 + 6 * tb + 24) + (n + 1) * 4 + 9 * n * tb


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one matrix-free PCG iteration,
# k_epass1 + k_epass2 (point Jacobi) or k_epass1 + k_epass2_bj (block Jacobi), from ncu
# captures of the 1,164,240-tet workload (cold cache: ncu flushes L2 before every replay pass,
# so slot values and DoF states that stay in L2 between the two passes of a live run are
# counted as DRAM traffic here).  Summaries and commands: profiles/elem_pcg_passes_window_frame_1p2M.md
# and profiles/elem_pcg_block_jacobi_window_frame_1p2M.md.  Scaled by the element count.
MEASURED_TRAFFIC = {"ne": 1_164_240, "fp64": (143.15e6 + 129.10e6), "mixed": (100.94e6 + 62.43e6),
                    "fp64_bj": (135.04e6 + 7.03e6 + 152.77e6 + 16.10e6),
                    "mixed_bj": (95.13e6 + 4.47e6 + 103.08e6 + 2.18e6)}


def measured_traffic(layout, precision, ne, block_jacobi=False):
    key = precision + ("_bj" if block_jacobi else "")
    if layout != "elem" or key not in MEASURED_TRAFFIC:
        return None
    return MEASURED_TRAFFIC[key] * ne / MEASURED_TRAFFIC["ne"]


# ---------------------------------------------------------------------------- ranks

def max_over_ranks(value, device="cpu"):
    """The largest of a float over all ranks of the default process group (the value itself
    when no group is initialised): every multi-GPU time is the slowest rank's."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_throughput(units_per_rank, ms_local, device="cpu"):
    """Units processed by all ranks per second of the slowest rank's timed interval."""
    import torch.distributed as dist

    world = dist.get_world_size() if (dist.is_available() and dist.is_initialized()) else 1
    return world * units_per_rank / (max_over_ranks(ms_local, device) / 1e3)


def partition_by_size(sizes, world):
    """Greedy balance of independent instances over ranks: largest first, each to the rank
    with the least work so far (ties to the lower rank).  Returns each rank's indices."""
    parts = [[] for _ in range(world)]
    load = [0.0] * world
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    import snoopy_b200 as S
    from snoopy_b200 import _lib
    from snoopy_b200 import mesh as M
    from snoopy_b200.device import upload, zeros

    t_setup = time.perf_counter()
    msh, coils, rel = workload(args.tets)
    solver = S.RedMVPSolver(msh, coils, [M.TAG_IRON], [M.TAG_AIR], [rel], max_newton_iterations=60, quad_order=2)
    solver.verbose = False
    eng = solver.newton_engine()
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t_setup
    prec = {"fp64": 0, "mixed": 1}[args.precision]
    n = msh.num_dofs
    nnz = eng.pattern.nnz
    x = zeros(n)[:n]

    def one_solve():
        # the coils' source field is evaluated on every solve, as the reference's solve does
        # (red_mvp_solver.py:149-166), then the Newton solve from A = 0
        solver.compute_source_fields(refresh=True)
        return eng.solve(None, mode=1, tol=RTOL, max_newton=60, precision=prec, x_out=x, cg_maxiter=50000)[1]

    for _ in range(args.warmup):
        one_solve()
    clocks = ClockSampler(local)
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0.record(stream)
    stats = [one_solve() for _ in range(args.steps)]
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, "cuda")
    value = whole_job_throughput(args.steps, ms, "cuda")

    # dominant kernel: the PCG iteration (the two passes of the matrix-free operator, or the
    # assembled-matrix kernels), timed by the solver's CUDA events around every Krylov solve
    # of the timed region
    cg_its = sum(s["cg_iterations"] for s in stats)
    t_kry = sum(s["t_krylov_ms"] for s in stats)
    t_asm = sum(s["t_assemble_ms"] for s in stats)
    newton = sum(s["newton_iterations"] for s in stats)
    assemblies = sum(1 + s["newton_iterations"] + s["residual_evals"] for s in stats)
    peak, peak_kind = measured_peaks()
    it_ms = t_kry / max(cg_its, 1)
    vb, xb = (8, 8) if args.precision == "fp64" else (4, 4)
    layout = eng.jacobian_layout
    ne = msh.num_elements
    bj = bool(getattr(eng, "block_jacobi", False))
    if layout == "elem":
        b_it = bytes_elem_pcg_iteration(ne, n, vb, block_jacobi=bj)
        b_apply = bytes_elem_apply(ne, n, vb)
        kern_name = ("pcg_iteration (k_epass1 element pass + k_epass2_bj block-Jacobi DoF pass; the block build of "
                     "each Newton step, k_bj_entries + k_bj_invert, inside the timed Krylov region)" if bj else
                     "pcg_iteration (k_epass1 element pass + k_epass2 DoF pass)")
    else:
        b_it = bytes_pcg_iteration(nnz, n, vb, xb)
        b_apply = bytes_spmv(nnz, n, vb, xb)
        kern_name = "pcg_iteration (k_spmv+dot, k_update, k_pupdate)"
    achieved = b_it / (it_ms / 1e3) / 1e9

    def time_spmv(fn, reps=50):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(3):
            fn()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    # SpMV alone: the Krylov loop's own operator (the last Newton Jacobian in the solver's
    # layout and precision), and the CSR entry point on the float64 Jacobian
    xv = x if xb == 8 else x.to(torch.float32)
    yv = torch.empty_like(xv)
    spmv_ms = time_spmv(lambda: eng.jacobian_apply(xv, yv, args.precision))
    spmv_gbs = b_apply / (spmv_ms / 1e3) / 1e9
    J = eng.assemble(x, J=True, F=False)["J"]
    pat = eng.pattern
    fm = eng.free_mask
    y = zeros(n)
    csr_ms = time_spmv(lambda: _lib.call("snp_spmv", n, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(J),
                                         _lib.ptr(fm), _lib.ptr(x), _lib.ptr(y), _lib.stream_ptr()))
    csr_gbs = bytes_spmv(nnz, n) / (csr_ms / 1e3) / 1e9

    # end to end through the public API: host x0 (pinned) in, host solution out
    x0_host = torch.zeros(n, dtype=torch.float64).pin_memory()
    e2e_times = []
    for _ in range(max(args.e2e_steps, 1)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xs, _st = solver.solve_to_residual(RTOL, x_0=x0_host, precision=args.precision, max_newton=60)
        t1 = time.perf_counter()
        e2e_times.append(t1 - t0)
    e2e_s = float(np.median(e2e_times))
    e2e_value = whole_job_throughput(1, 1e3 * e2e_s, "cuda")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference's own work per solve (point-Jacobi CG), not this solver's counts
        cpu = cpu_baseline_sample(msh, coils, rel, REFERENCE_COUNTS["assemblies"], REFERENCE_COUNTS["cg"])

    launches = int(sum(s.get("kernel_launches", 0) for s in stats)) or None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded window-frame yoke mesh and coils, no dataset)",
        "config": {"workload": f"reduced-MVP Newton solve to rel. residual 1e-8, window-frame yoke, "
                               f"{msh.num_elements} tets / {n} edge DoFs, Q=4, {args.precision}",
                   "tets": msh.num_elements, "dofs": n, "nnz": nnz, "precision": args.precision,
                   "jacobian": layout,
                   "preconditioner": "block Jacobi (edges sharing a node)" if bj else "point Jacobi",
                   "newton_per_solve": newton / args.steps, "cg_per_solve": cg_its / args.steps,
                   "assemblies_per_solve": assemblies / args.steps,
                   "assembly_ms_per_solve": t_asm / args.steps, "krylov_ms_per_solve": t_kry / args.steps,
                   "setup_s": t_setup, "l2": "matrix values+indices > 126 MB L2 (no flush needed)",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"kernel": kern_name, "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "bytes_per_launch": b_it, "launch_ms": it_ms,
                     "traffic": measured_traffic(layout, args.precision, ne, layout == "elem" and bj),
                     "spmv_alone": {"achieved": spmv_gbs, "frac": spmv_gbs / peak, "ms": spmv_ms,
                                    "bytes": b_apply, "layout": layout},
                     "spmv_csr_f64": {"achieved": csr_gbs, "frac": csr_gbs / peak, "ms": csr_ms,
                                      "bytes": bytes_spmv(nnz, n)}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
        "cpu_baseline": cpu,
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_extras:
        del eng, solver, x, J, y, xv, yv, pat, fm
        torch.cuda.empty_cache()
        line["assembly_microbench"] = assembly_microbench()
        torch.cuda.empty_cache()
        line["mixed_precision_4m"] = mixed_precision_accuracy()
        torch.cuda.empty_cache()
        line["mixed_warm_start"] = warm_start_study(args.tets, n_train=160, n_test=8)
        torch.cuda.empty_cache()
        line["batched_variants_32"] = batched_study(32)
        torch.cuda.empty_cache()
        # the learned-warm-start configuration at its stated size: the morphed 300k-tet family,
        # 4000 training solves (generated 32 members at a time by the batched solver), 500 held out
        line["warm_start_family_300k"] = warm_start_study(300_000, n_train=4000, n_test=500, generate_at_once=32)
        torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def warm_start_study(base_tets, n_train, n_test, n_modes=128, hidden=256, epochs=None, seed=0, galerkin_modes=64,
                     generate_at_once=1):
    """Learned warm start on a morphed-yoke family (fixed topology, 8 shape parameters + coil
    current density).  Untimed: ``n_train`` zero-start mixed-precision solves, POD to
    ``n_modes`` modes, MLP training on the tensor-core kernels.  Timed (CUDA events around each
    solve; moving the solver to a member is not timed): ``n_test`` held-out members solved
    three ways to ||F_free|| <= 1e-8 ||F_free(0)||: plain float64 from zero, mixed precision
    from zero, and mixed precision from the network's prediction (inference and reconstruction
    inside the timed region), and that prediction moved by one Galerkin Newton step in the span
    of the first ``galerkin_modes`` POD modes inside the solve (``MorphedSolver.attach_basis``;
    0 skips it).  The members-at-once row uses the corrected starts when the correction runs."""
    import torch

    from snoopy_b200 import morph
    from snoopy_b200 import surrogate as SG

    t0 = time.perf_counter()
    fam = morph.YokeMorphFamily(base_tets=base_tets, seed=7)
    ms = SG.MorphedSolver(fam)
    P = fam.sample(n_train + n_test, seed=seed + 101)
    P_train, P_test = P[:n_train], P[n_train:]
    setup_s = time.perf_counter() - t0
    modes = min(n_modes, n_train - 1)
    ws = SG.WarmStart(ms, n_modes=modes, hidden=hidden, seed=seed)
    snaps, st_train = ws.generate(P_train, precision="mixed", members_at_once=generate_at_once)
    ws.fit(P_train, snaps, epochs=epochs, batch=min(256, (n_train // 8) * 8), lr=2e-3, seed=seed)
    del snaps
    torch.cuda.empty_cache()
    stream = torch.cuda.current_stream()
    rows = {"fp64_zero": [], "mixed_zero": [], "mixed_warm": []}
    galerkin_modes = min(galerkin_modes, modes)
    if galerkin_modes > 0:
        rows["mixed_warm_galerkin"] = []
    surr_err, proj_err, b_err = [], [], []
    warm_x, galerkin_x, b_refs = [], [], []
    probes = fam.geometry.aperture_probes(200, margin=0.03)
    el, _ = fam.mesh.locate(probes)
    for p in P_test:
        ref = ms.set_member(p)
        for name in rows:
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            x0 = ws.predict(p)[0] if name.startswith("mixed_warm") else None
            if name == "mixed_warm_galerkin":
                ms.attach_basis(ws.galerkin_basis(galerkin_modes))
            x, st = ms.solve(x0, rtol=RTOL, precision="fp64" if name == "fp64_zero" else "mixed", res_ref=ref)
            ms.attach_basis(None)
            e1.record(stream)
            torch.cuda.synchronize()
            rows[name].append((e0.elapsed_time(e1), st["newton_iterations"], st["cg_iterations"], st["rel_res"],
                               st["start_dropped"]))
            if name == "fp64_zero":
                x_ref = x.clone()
                B_ref = ms.solver.curl_curl_factory.compute_B_at_points(x, probes, el)
                b_refs.append(B_ref)
            elif name == "mixed_warm":
                warm_x.append(x.clone())
                nrm = float(torch.linalg.vector_norm(x_ref).item())
                surr_err.append(float(torch.linalg.vector_norm(x0 - x_ref).item()) / nrm)
                proj_err.append(float(torch.linalg.vector_norm(ws.project(x_ref) - x_ref).item()) / nrm)
                Bw = ms.solver.curl_curl_factory.compute_B_at_points(x, probes, el)
                b_err.append(float(np.linalg.norm(Bw - B_ref, axis=1).max() / np.linalg.norm(B_ref, axis=1).max()))
            elif name == "mixed_warm_galerkin":
                galerkin_x.append(x.clone())
                Bw = ms.solver.curl_curl_factory.compute_B_at_points(x, probes, el)
                b_err.append(float(np.linalg.norm(Bw - B_ref, axis=1).max() / np.linalg.norm(B_ref, axis=1).max()))
    out = {"workload": f"morphed window-frame yoke family, {fam.mesh.num_elements} tets / {fam.mesh.num_dofs} DoFs, "
                       f"8 shape parameters + J, {n_train} training / {n_test} held-out members",
           "setup_s": setup_s, "generate_s": ws.timings["generate_s"], "fit_s": ws.timings["fit_s"],
           "preconditioner": "block Jacobi" if getattr(ms.eng, "block_jacobi", False) else "point Jacobi",
           "pod_modes": modes, "pod_energy": ws.pod_energy, "train_loss_first_last": [ws.history[0][1], ws.history[-1][1]],
           "train_newton_mean": float(np.mean([s["newton_iterations"] for s in st_train])),
           "surrogate_rel_err_mean": float(np.mean(surr_err)), "pod_floor_rel_err_mean": float(np.mean(proj_err)),
           "warm_vs_fp64_B_err_max": float(np.max(b_err))}
    for name, r in rows.items():
        r = np.array(r, dtype=np.float64)
        out[name] = {"solves_per_s": len(r) / (r[:, 0].sum() / 1e3), "ms_mean": float(r[:, 0].mean()),
                     "newton_mean": float(r[:, 1].mean()), "cg_mean": float(r[:, 2].mean()),
                     "rel_res_max": float(r[:, 3].max()), "starts_dropped": int(r[:, 4].sum())}
    out["speedup_mixed_warm_vs_fp64_zero"] = out["mixed_warm"]["solves_per_s"] / out["fp64_zero"]["solves_per_s"]
    if galerkin_modes > 0:
        out["galerkin_modes"] = galerkin_modes
        out["speedup_mixed_warm_galerkin_vs_fp64_zero"] = (out["mixed_warm_galerkin"]["solves_per_s"]
                                                           / out["fp64_zero"]["solves_per_s"])
    # the same warm-started mixed solves, `batch` members at a time: one solver per member, each
    # on its own stream and host thread (snp_solver_solve_many); wall clock around each batch's
    # predictions and solves (moving the solvers to their members is not timed, as above).
    # Smaller meshes leave more of the GPU idle per solve, so they run more members at once (at
    # 287k tets a sweep gave 145 / 157 / 162 / 161 solves/s for 8 / 16 / 24 / 32 at once).
    batch = min(24 if fam.mesh.num_elements < 600_000 else 4, len(P_test))
    if batch > 1:
        extra = [SG.MorphedSolver(fam, stream=torch.cuda.Stream()) for _ in range(batch)]
        if galerkin_modes > 0:
            for m in extra:
                m.attach_basis(ws.galerkin_basis(galerkin_modes))
        # three passes over the held-out members (wall clock is host-sensitive: median of the three)
        walls, stats, same = [], [], True
        for rep in range(3):
            wall = 0.0
            for c0 in range(0, len(P_test), batch):
                chunk = list(range(c0, min(c0 + batch, len(P_test))))
                mss = extra[: len(chunk)]
                refs = [m.set_member(P_test[i]) for m, i in zip(mss, chunk)]
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                x0s = [ws.predict(P_test[i], check=False)[0] for i in chunk]  # row by row, as one at a time
                ws.mlp.check_errors()
                xs, st = SG.solve_members_at_once(mss, x0s, refs, rtol=RTOL, precision="mixed")
                torch.cuda.synchronize()
                wall += time.perf_counter() - t1
                if rep == 0:
                    stats += st
                one_at_a_time = galerkin_x if galerkin_modes > 0 else warm_x
                same = same and all(torch.equal(x, one_at_a_time[i]) for x, i in zip(xs, chunk))
            walls.append(wall)
        wall = float(np.median(walls))
        out["mixed_warm_batched"] = {
            "members_at_once": batch, "galerkin_modes": galerkin_modes, "solves_per_s": len(P_test) / wall,
            "passes_s": walls,
            "newton_mean": float(np.mean([s_["newton_iterations"] for s_ in stats])),
            "cg_mean": float(np.mean([s_["cg_iterations"] for s_ in stats])),
            "rel_res_max": float(max(s_["rel_res"] for s_ in stats)),
            "identical_to_one_at_a_time": bool(same)}
        out["speedup_mixed_warm_batched_vs_fp64_zero"] = (out["mixed_warm_batched"]["solves_per_s"]
                                                          / out["fp64_zero"]["solves_per_s"])
        del extra
    # the batched solver (snp_batch_*): every held-out member's warm start (network prediction,
    # then the Galerkin step on the host path) solved by one batched Newton loop, members in
    # groups of `eng_batch`; predictions, Galerkin steps and the batched solve are timed
    from snoopy_b200 import batch as BT

    eng_batch = min(32 if fam.mesh.num_elements < 600_000 else 8, len(P_test))
    if eng_batch > 1:
        members = [SG.MorphedSolver(fam) for _ in range(eng_batch)]
        engine = BT.BatchSolver(members)
        tuned = engine.tune("mixed")
        wall, stats, errs = 0.0, [], []
        for c0 in range(0, len(P_test), eng_batch):
            chunk = list(range(c0, min(c0 + eng_batch, len(P_test))))
            if len(chunk) < eng_batch:  # a smaller last group gets a batch of its own size
                engine = BT.BatchSolver(members[: len(chunk)])
            mss = members[: len(chunk)]
            refs = [m.set_member(P_test[i]) for m, i in zip(mss, chunk)]
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            x0s = []
            for m, i in zip(mss, chunk):
                x0 = ws.predict(P_test[i], check=False)[0]
                if galerkin_modes > 0:
                    x0 = ws.correct(x0, msolver=m, modes=galerkin_modes, precision="mixed")
                x0s.append(x0)
            ws.mlp.check_errors()
            st = engine.solve(RTOL, precision="mixed", x0s=x0s, res_refs=refs)
            torch.cuda.synchronize()
            wall += time.perf_counter() - t1
            stats += st
            for m, x, i in zip(mss, engine.xs, chunk):
                Bw = m.solver.curl_curl_factory.compute_B_at_points(x, probes, el)
                errs.append(float(np.linalg.norm(Bw - b_refs[i], axis=1).max()
                                  / np.linalg.norm(b_refs[i], axis=1).max()))
        out["mixed_warm_batched_engine"] = {
            "members_per_batch": eng_batch, "galerkin_modes": galerkin_modes, "solves_per_s": len(P_test) / wall,
            "newton_mean": float(np.mean([s_["newton_iterations"] for s_ in stats])),
            "cg_mean": float(np.mean([s_["cg_iterations"] for s_ in stats])),
            "rel_res_max": float(max(s_["rel_res"] for s_ in stats)),
            "starts_dropped": int(sum(s_["start_dropped"] for s_ in stats)),
            "B_err_vs_fp64_zero_max": float(max(errs)),
            "autotuner": {k: tuned[k] for k in ("pass1_block", "asm_waves", "graph")}}
        out["speedup_mixed_warm_batched_engine_vs_fp64_zero"] = (out["mixed_warm_batched_engine"]["solves_per_s"]
                                                                 / out["fp64_zero"]["solves_per_s"])
        del engine, members
    del ws, ms, fam
    return out


def mixed_precision_accuracy(tets=4_000_000, n_probes=1000):
    """The same window-frame yoke at ~4M tets solved to the 1e-8 Newton residual twice: in
    float64, and with float32 element tensors and float32 CG inside the float64 Newton loop
    (the Newton residual and update stay float64, so each Newton step refines the float32
    inner solve).  Reported: B error at 1000 seeded aperture probes of both solves against the
    CPU oracle's float64 solve (reference C kernels and scipy cg, converged to 1e-10; stored in
    tests/golden/config_c3.npz by tests/golden/make_config_golden.py), of the mixed solve against
    the float64 device solve, and Newton / CG counts and times of both."""
    import torch

    import snoopy_b200 as S
    from snoopy_b200 import mesh as M

    t0 = time.perf_counter()
    msh, coils, rel = workload(tets)
    solver = S.RedMVPSolver(msh, coils, [M.TAG_IRON], [M.TAG_AIR], [rel], max_newton_iterations=60, quad_order=2)
    solver.verbose = False
    solver.newton_engine()
    probes = msh.geometry.aperture_probes(n_probes)
    el, _ = msh.locate(probes)
    setup_s = time.perf_counter() - t0
    out = {"workload": f"window-frame yoke, {msh.num_elements} tets / {msh.num_dofs} edge DoFs, Q=4",
           "setup_s": setup_s, "probes": n_probes}
    B = {}
    for prec in ("fp64", "mixed"):
        # one untimed solve first: the first call of a precision loads its kernels and builds its
        # Krylov graph, which costs tens of milliseconds at this size
        solver.solve_to_residual(RTOL, precision=prec, max_newton=60, return_device=True)
        torch.cuda.synchronize()
        t = time.perf_counter()
        xs, st = solver.solve_to_residual(RTOL, precision=prec, max_newton=60, return_device=True)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t
        B[prec] = solver.evaluate_B(xs, probes, el)
        out[prec] = {"newton": st["newton_iterations"], "cg": st["cg_iterations"], "rel_res": st["rel_res"],
                     "solve_s": wall, "krylov_ms": st["t_krylov_ms"], "assembly_ms": st["t_assemble_ms"],
                     "pcg_iteration_us": 1e3 * st["t_krylov_ms"] / max(st["cg_iterations"], 1)}
    d = np.linalg.norm(B["mixed"] - B["fp64"], axis=1)
    out["b_err_max_rel"] = float(d.max() / np.linalg.norm(B["fp64"], axis=1).max())
    out["b_err_rms_rel"] = float(np.sqrt(np.mean(d ** 2)) / np.sqrt(np.mean(np.sum(B["fp64"] ** 2, axis=1))))
    fx_path = os.path.join(ROOT, "tests", "golden", "config_c3.npz")
    if os.path.exists(fx_path):
        fx = np.load(fx_path)
        if int(fx["tets"]) == msh.num_elements and np.array_equal(fx["elements"], el):
            Bo = fx["B"]
            scale = np.linalg.norm(Bo, axis=1).max()
            out["vs_fp64_oracle"] = {
                "oracle": f"CPU float64 Newton to rel. residual {float(fx['rel_res']):.1e} (reference C kernels, "
                          f"scipy Jacobi cg; {int(fx['newton'])} Newton steps, {int(fx['cg'])} CG iterations)",
                **{f"b_err_max_rel_{p}": float(np.linalg.norm(B[p] - Bo, axis=1).max() / scale) for p in B}}
    del solver
    return out


def assembly_microbench(reps=5, warmup=3, seed=5, grid=(120, 120, 116)):
    """Assembly-only microbenchmark: the structured 120 x 120 x 116 grid (``grid``) split into 6 tets
    per cell (10,022,400 tets), nodes jittered by U[-0.2, 0.2] x spacing, edge DoFs
    x ~ N(0, 1e-3), seeded 40% iron flags (PCHIP atan B-H) against air, no Dirichlet mask,
    4-point rule, float64.  Two Newton assemblies at x are timed (CUDA events, after warm-up):

    * csr: the drop-in path, J = K + dK into the fixed CSR plus the residual F
      (``snp_solver_assemble``): the element kernel stores each element's 21 matrix values and six
      residual terms, then every CSR entry and every F entry is summed from its contributions in
      element order, each value written once (deterministic); ``csr_atomic``: the same outputs
      from the element kernel adding into the CSR through the slot map with float64 atomics
      (``SNP_ASSEMBLY=atomic``, the value zeroing included);
    * tensors: the matrix-free path of the Newton loop, S_e per element plus F and diag(J)
      summed per DoF (``snp_solver_assemble_tensors``).

    Algorithmic bytes: csr E*(16 cells + 24 DoFs + 4 orientation + 144 slots) + 24N + 8n (x)
    + 8nnz (J) + 8n (F); tensors E*(16 + 24 + 4 + 48 S_e) + 24N + 8n + 16n (F, diag).
    Every element is read once per call; the 1.9e8-entry matrix and the slot map exceed L2.
    """
    import torch

    import snoopy_b200 as S
    from snoopy_b200 import _lib
    from snoopy_b200 import materials as MAT
    from snoopy_b200 import mesh as M
    from snoopy_b200.curl_curl_assembler import CurlCurlAssembler
    from snoopy_b200.device import upload, zeros
    from snoopy_b200.newton import DeviceNewton

    t0 = time.perf_counter()
    msh = M.kuhn_microbench_mesh(*grid)
    E, N, n = msh.num_elements, msh.nodes.shape[0], msh.num_dofs
    asm = CurlCurlAssembler(msh, [M.TAG_IRON, M.TAG_AIR], [MAT.atan_reluctance(), S.ConstantReluctance(1e7 / (4 * np.pi))])
    eng = DeviceNewton(asm, np.ones(n, dtype=np.uint8), (), quad_order=2)
    os.environ["SNP_ASSEMBLY"] = "atomic"
    try:
        eng_atomic = DeviceNewton(asm, np.ones(n, dtype=np.uint8), (), quad_order=2)
    finally:
        del os.environ["SNP_ASSEMBLY"]
    nnz = eng.pattern.nnz
    x = upload(np.random.default_rng(seed).normal(0.0, 1e-3, n), np.float64)
    J = zeros(nnz)
    F = zeros(n)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(warmup):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_csr = timed(lambda: _lib.call("snp_solver_assemble", eng.handle, _lib.ptr(x), None, _lib.ptr(J), None,
                                     _lib.ptr(F), _lib.stream_ptr()))
    ms_atomic = timed(lambda: _lib.call("snp_solver_assemble", eng_atomic.handle, _lib.ptr(x), None, _lib.ptr(J), None,
                                        _lib.ptr(F), _lib.stream_ptr()))
    ms_t = timed(lambda: eng.assemble_tensors(x, "fp64", F))
    peak, peak_kind = measured_peaks()
    b_csr = E * (16 + 24 + 4 + 144) + 24 * N + 8 * n + 8 * nnz + 8 * n
    b_t = E * (16 + 24 + 4 + 48) + 24 * N + 8 * n + 16 * n
    out = {"workload": f"Kuhn grid {grid[0]}x{grid[1]}x{grid[2]} x 6 = {E} tets, {N} nodes, {n} edge DoFs, nnz {nnz}, "
                       f"40% iron, x ~ N(0, 1e-3), Q=4, f64",
           "setup_s": setup_s, "peak_gbs": peak, "peak_kind": peak_kind}
    for name, ms, b in (("csr", ms_csr, b_csr), ("csr_atomic", ms_atomic, b_csr), ("tensors", ms_t, b_t)):
        gbs = b / (ms / 1e3) / 1e9
        out[name] = {"ms": ms, "gelem_per_s": E / (ms / 1e3) / 1e9, "bytes": b, "achieved_gbs": gbs,
                     "frac": gbs / peak}
    del eng, eng_atomic, asm, J, F, x
    return out


# ---------------------------------------------------------------------------- CPU reference

def reference_sample(msh, coils, rel, assemblies_per_solve, cg_per_solve, n_cg_sample=10, quad_order=2):
    """Time the reference's CPU path on the full workload and project one solve.

    Times one assembly through the reference's own C kernels (oracle/_ref,
    compute_K_dK_Hcurl[_red] via the Cython layer's marshalling) with scipy's COO->CSR, the
    per-material ``K +=`` adds, ``dK + K``, the Dirichlet fancy-indexing and the Jacobi
    preconditioner, then ``n_cg_sample`` iterations of scipy's cg on that system.  A solve is
    the source field, ``assemblies_per_solve`` assemblies (one per Newton step, one at the
    start, one per extra line-search trial) and ``cg_per_solve`` CG iterations.
    """
    import oracle as O
    from scipy.sparse import diags
    from scipy.sparse.linalg import cg

    import snoopy_b200 as S
    from snoopy_b200 import finite_element as FE
    from snoopy_b200 import mesh as M

    backend = "ref" if O.ref_available() else "oracle"
    w, q = FE.quadrature_rule(quad_order)
    dphi = FE.evaluate_basis_derivative(q)
    phi = FE.evaluate_basis(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    iron = msh.domain_elements(M.TAG_IRON)
    air = msh.domain_elements(M.TAG_AIR)
    mats = [dict(cells=msh.cells[iron], glob_ids=msh.elem_edges[iron], orientations=msh.orientations[iron],
                 reluctance=rel),
            dict(cells=msh.cells[air], glob_ids=msh.elem_edges[air], orientations=msh.orientations[air],
                 reluctance=S.ConstantReluctance(0.25 / np.pi * 1e7))]
    t0 = time.perf_counter()
    P = np.einsum("qi,eid->eqd", phi, msh.nodes[msh.cells[iron]]).reshape(-1, 3)
    Bs = sum(O.compute_B_line_segs_cpp(c.get_segments(), P, c.current, c.rad, backend=backend) for c in coils)
    t_src = time.perf_counter() - t0
    A = O.OracleCurlCurlAssembler(msh.nodes, mats, msh.num_dofs, w, q, dphi, curls, backend=backend)
    mask = np.ones(msh.num_dofs, bool)
    mask[msh.get_edge_boundary_dofs() - 1] = False
    x = np.random.default_rng(0).normal(0.0, 1e-3, msh.num_dofs)
    x[~mask] = 0.0
    t0 = time.perf_counter()
    K, J, rhs = A.compute_stiffness_and_jacobi_matrix_c(x, [Bs, np.zeros((0, 3))])
    F = K @ x - rhs
    J_c = J[mask, :][:, mask]
    M_ = diags(1.0 / J_c.diagonal(), shape=J_c.shape)
    t_asm = time.perf_counter() - t0
    t0 = time.perf_counter()
    cg(J_c, -F[mask], rtol=1e-30, atol=0.0, M=M_, maxiter=n_cg_sample)
    t_it = (time.perf_counter() - t0) / n_cg_sample
    t_solve = t_src + assemblies_per_solve * t_asm + cg_per_solve * t_it
    return {"value": 1.0 / t_solve, "unit": UNIT, "cores": 1, "kind": "reference" if backend == "ref" else "port",
            "sample": (f"1 full Newton assembly ({t_asm:.2f} s: reference C kernels + scipy COO->CSR, sparse adds, "
                       f"masking) and {n_cg_sample} scipy Jacobi-CG iterations ({t_it * 1e3:.1f} ms each) on the "
                       f"{msh.num_elements}-tet system; solve projected as source field + "
                       f"{assemblies_per_solve:.1f} assemblies + {cg_per_solve:.0f} CG iterations"),
            "t_assembly_s": t_asm, "t_cg_iteration_s": t_it, "t_source_s": t_src, "t_solve_projected_s": t_solve}


def cpu_baseline_sample(msh, coils, rel, assemblies_per_solve, cg_per_solve):
    try:
        return reference_sample(msh, coils, rel, assemblies_per_solve, cg_per_solve)
    except Exception as exc:  # the baseline must not take the GPU line down
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {exc}"}


# Work per solve of this workload, measured by running the whole solve on the CPU with the
# reference's kernels and scipy's cg (oracle.newton_residual with forcing="ew" and
# line_search="energy", the device solver's algorithm) on the 1.16M-tet mesh: 13 Newton steps,
# 2868 CG iterations and 22 assemblies, 278 s on one core.  The device solver needs 13 steps and
# 2652 CG iterations with the same point Jacobi, 13-14 steps and about 1313 with its block
# Jacobi; the reference arm and the cpu_baseline object project the measured per-iteration
# times with the oracle's counts.
REFERENCE_COUNTS = {"newton": 13.0, "assemblies": 22.0, "cg": 2868.0}


def host_info():
    """Host CPU of the machine the reference arm runs on: model, logical CPUs this process may
    use, and the numerical libraries of the CPU path."""
    import platform

    import scipy

    model = platform.processor() or ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count() or 1
    mem_gb = None
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable"):
                mem_gb = int(line.split()[1]) / 2**20
                break
    except OSError:
        pass
    return {"cpu_model": model, "logical_cpus": os.cpu_count(), "usable_cpus": usable, "mem_available_gb": mem_gb,
            "numpy": np.__version__, "scipy": scipy.__version__}


# Host memory one worker of the reference arm holds at the ~1.2M-tet workload (reference
# triplets, scipy's COO->CSR copies of K, dK and J, the masked Jacobian), measured peak ~4 GB.
REFERENCE_WORKER_GB = 6.0


def _reference_worker(tets, solve_ids, warmup, barrier, out_q):
    """One host process of the reference arm: build the workload and the oracle problem (the
    reference's C kernels), run ``warmup`` bounded samples, wait for the others, then run each
    listed solve completely and report its time."""
    from threadpoolctl import threadpool_limits

    threadpool_limits(1)
    import oracle as O
    from scipy.sparse import diags
    from scipy.sparse.linalg import cg

    P = oracle_problem(tets)
    msh, A, mask = P["msh"], P["A"], P["mask"]
    sample = None
    for k in range(warmup):
        # bounded warm-up: one assembly and 10 Jacobi-CG iterations at a seeded state
        x = np.random.default_rng(k).normal(0.0, 1e-3, msh.num_dofs)
        x[~mask] = 0.0
        t0 = time.perf_counter()
        K, J, rhs = A.compute_stiffness_and_jacobi_matrix_c(x, P["sf"])
        F = K @ x - rhs
        J_c = J[mask, :][:, mask]
        M_ = diags(1.0 / J_c.diagonal(), shape=J_c.shape)
        t1 = time.perf_counter()
        cg(J_c, -F[mask], rtol=1e-30, atol=0.0, M=M_, maxiter=10)
        t2 = time.perf_counter()
        sample = {"t_assembly_s": t1 - t0, "t_cg_iteration_s": (t2 - t1) / 10}
        del K, J, rhs, F, J_c, M_
    barrier.wait()
    for sid in solve_ids:
        t0 = time.perf_counter()
        # the source field at the iron quadrature points, evaluated per solve as
        # red_mvp_solver.py:149-166 does (reference Biot-Savart kernel)
        Bs = sum(O.compute_B_line_segs_cpp(c.get_segments(), P["iron_points"], c.current, c.rad, backend="ref")
                 for c in P["coils"])
        t_src = time.perf_counter() - t0
        x, st = O.newton_residual(A, mask, [Bs, np.zeros((0, 3))], rtol=RTOL, forcing="ew", line_search="energy",
                                  cg_rtol=0.1, max_newton_iterations=60)
        t1 = time.perf_counter()
        out_q.put({"solve": sid, "s": t1 - t0, "t_source_s": t_src, "newton": st["newton"], "cg": int(sum(st["cg"])),
                   "assemblies": st["assemblies"], "rel_res": st["rel_res"], "sample": sample})


def run_reference(args):
    """The reference arm: complete CPU Newton solves of the workload with the reference's own C
    kernels (``oracle/_ref``: compute_K_dK_Hcurl[_red] and compute_B_line_segs through the Cython
    layer's marshalling), scipy's COO->CSR and sparse adds, and scipy's Jacobi-preconditioned
    ``cg`` (``red_mvp_solver.py:178-222``), driven by the same inexact Newton as the device solver
    (Eisenstat-Walker inner tolerances, energy line search) from A = 0 to the 1e-8 relative
    residual.  Each step is one complete solve; the steps run in parallel host processes, one
    single-threaded solve per core, so the value is the host's whole-machine throughput."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp

    import oracle as O

    info = host_info()
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's C kernels) is not built"}),
              flush=True)
        return
    # one single-threaded process per solve while memory allows: with more solves than cores the
    # processes share the cores (the wall time is then that of the whole host doing all of them,
    # not of two uneven waves)
    mem_cap = int((info["mem_available_gb"] or 64.0) // REFERENCE_WORKER_GB) or 1
    procs = max(1, min(args.steps, mem_cap))
    shares = [list(range(p, args.steps, procs)) for p in range(procs)]
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs + 1)
    q = ctx.Queue()
    t_setup = time.perf_counter()
    workers = [ctx.Process(target=_reference_worker, args=(args.tets, shares[p], args.warmup, barrier, q))
               for p in range(procs)]
    for w in workers:
        w.start()
    barrier.wait()
    t_setup = time.perf_counter() - t_setup
    t0 = time.perf_counter()
    res = [q.get() for _ in range(args.steps)]
    t1 = time.perf_counter()
    for w in workers:
        w.join()
    wall = t1 - t0
    value = args.steps / wall
    per = np.array([r["s"] for r in res])
    smp = next((r["sample"] for r in res if r["sample"]), None)
    counts = {k: float(np.mean([r[k] for r in res])) for k in ("newton", "cg", "assemblies")}
    projected = None
    if smp:
        projected = (float(np.mean([r["t_source_s"] for r in res])) + counts["assemblies"] * smp["t_assembly_s"]
                     + counts["cg"] * smp["t_cg_iteration_s"])
    tets_msg = f"{args.tets}"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"reduced-MVP Newton solve to rel. residual 1e-8, window-frame yoke, "
                                   f"~{tets_msg} target tets, Q=4, fp64",
                       "solves": args.steps, "processes": procs, "counts_per_solve": counts,
                       "max_rel_res": float(max(r["rel_res"] for r in res)), "setup_s": t_setup},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": min(procs, info["usable_cpus"]), "kind": "reference",
                             "sample": (f"{args.steps} complete solves (reference C kernels, scipy CSR and Jacobi cg, "
                                        f"source field per solve) on {procs} single-threaded processes; one solve "
                                        f"{per.mean():.1f} s mean ({per.min():.1f}-{per.max():.1f} s); warm-up: "
                                        f"{args.warmup} bounded samples per process (one assembly + 10 CG "
                                        f"iterations)"),
                             "solve_s_mean": float(per.mean()), "solve_s_min": float(per.min()),
                             "solve_s_max": float(per.max()), "single_core_solves_per_s": float(1.0 / per.mean()),
                             "projected_solve_s": projected, "host": info},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batched_study(n=128, rank=0, world=1, one_by_one=True):
    """Seeded yoke variants (the batched workload: 30k-600k tets, half reduced, half
    total potential), every instance solved to the 1e-8 residual, in float64 and in mixed
    precision, three ways:

    * one after another (each instance's own solver);
    * ``snp_solver_solve_many``: every instance's own Newton solve on a host thread and stream
      of its own, overlapping on the GPU;
    * the batched solver (``snp_batch_*``): one launch per pass over the concatenated element
      and DoF arrays of all instances, the Newton loop one CUDA graph, launch shapes from its
      autotuner (tuned once per precision before the timed solve).

    Throughput is instances per second of wall time (host clock around each whole batch, after a
    synchronize).  Each way's answers are checked: solve_many bitwise against one-at-a-time, the
    batched solver bitwise against batches of one (the first two instances) and by field
    against one-at-a-time."""
    import torch

    from snoopy_b200 import batch as B
    from snoopy_b200 import mesh as M

    t0 = time.perf_counter()
    V = B.sample_variants(n, seed=0)
    if world > 1:  # independent instances: each rank takes a greedy size-balanced share
        V = [V[i] for i in partition_by_size([v["tets"] for v in V], world)[rank]]
    inst = [B.Instance(v) for v in V]
    engine = B.BatchSolver(inst)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    tets = sum(i.num_elements for i in inst)
    dofs = sum(i.n for i in inst)
    res = {}
    import torch.distributed as dist

    def barrier():
        if world > 1:
            dist.barrier()

    def iron_B(ins, x):
        sel = ins.mesh.domain_elements(M.TAG_IRON)[::7]
        return ins.solver.curl_curl_factory.compute_B_at_points(x, ins.mesh.element_centroids()[sel], sel)

    for prec in ("fp64", "mixed"):
        B.solve_many(inst[:8], precision=prec)  # warm-up: graphs and work buffers of a few instances
        r = {}
        x_seq = None
        if one_by_one:
            barrier()
            t = time.perf_counter()
            B.solve_one_by_one(inst, precision=prec)
            t_seq = max_over_ranks(time.perf_counter() - t, "cuda")
            x_seq = [i.x.clone() for i in inst]
            r.update({"one_by_one_s": t_seq, "one_by_one_per_s": n / t_seq})
        barrier()
        t = time.perf_counter()
        par = B.solve_many(inst, precision=prec)
        t_par = max_over_ranks(time.perf_counter() - t, "cuda")
        if x_seq is None:
            x_seq = [i.x.clone() for i in inst]
        r.update({"solve_many_s": t_par, "solve_many_per_s": n / t_par,
                  "solve_many_identical_to_one_by_one": all(bool(torch.equal(a, i.x)) for a, i in zip(x_seq, inst)),
                  "solve_many_max_rel_res": max(s["rel_res"] for s in par)})
        # the batched solver: tune, one untimed solve (graph instantiation), then the timed one
        info = engine.tune(prec)
        engine.solve(precision=prec)
        barrier()
        t = time.perf_counter()
        eng = engine.solve(precision=prec)
        t_eng = max_over_ranks(time.perf_counter() - t, "cuda")
        x_eng = [i.x.clone() for i in inst]
        field = max(float(np.abs(iron_B(i, xe) - iron_B(i, xs)).max() / np.abs(iron_B(i, xs)).max())
                    for i, xe, xs in zip(inst, x_eng, x_seq))
        alone = True
        for k in range(min(2, len(inst))):
            B.BatchSolver([inst[k]]).solve(precision=prec)
            alone = alone and bool(torch.equal(inst[k].x, x_eng[k]))
        r.update({"batched_engine_s": t_eng, "batched_engine_per_s": n / t_eng,
                  "batched_engine_max_rel_res": max(s["rel_res"] for s in eng),
                  "batched_engine_identical_to_batch_of_one": alone,
                  "batched_engine_field_vs_one_by_one": field,
                  "batched_engine_kernel_launches": int(eng[0]["kernel_launches"]),
                  "batched_engine_newton_max": int(max(s["newton_iterations"] for s in eng)),
                  "autotuner": {k: info[k] for k in ("pass1_block", "asm_waves", "tuned_pass1_us", "tuned_asm_us",
                                                     "graph")},
                  "newton_mean": float(np.mean([s["newton_iterations"] for s in eng])),
                  "cg_mean": float(np.mean([s["cg_iterations"] for s in eng]))})
        if one_by_one:
            r["batched_engine_speedup_vs_one_by_one"] = r["one_by_one_s"] / t_eng
        res[prec] = r
        del x_seq, x_eng
    del engine, inst
    return {"instances": n, "ranks": world, "tets_this_rank": tets, "dofs_this_rank": dofs, "setup_s": setup_s,
            "note": ("instances split over ranks by size, max time over ranks" if world > 1 else "one GPU"),
            **res}


def run_batched(args, n=128):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    res = batched_study(n, rank, world)
    if rank == 0:
        line = {"metric": "batched nonlinear solves/s, 128 seeded yoke variants (30k-600k tets) to 1e-8 residual",
                "value": res["mixed"]["batched_engine_per_s"], "unit": "solves/s", "higher_is_better": True,
                "n_gpus": world, "scaling": "strong", "dtype": "f32+f64", "data": "synthetic (seeded variant family)",
                "config": res}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_warm_start_family(args):
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    res = warm_start_study(300_000, n_train=4000, n_test=500, generate_at_once=32)
    line = {"metric": "warm-started vs zero-start nonlinear solves/s, morphed 300k-tet yoke family",
            "value": res["mixed_warm"]["solves_per_s"], "unit": UNIT, "higher_is_better": True, "n_gpus": 1,
            "dtype": "f32+f64 (bf16 MLP)", "data": "synthetic (seeded morphed-yoke family)", "config": res}
    print(json.dumps(line), flush=True)


def run_assembly_grid(a):
    g = a.assembly_grid
    out = assembly_microbench(reps=max(a.steps, 1), warmup=max(a.warmup, 1), grid=(g, g, max(2, round(g * 116 / 120))))
    print(json.dumps({"metric": "assembly microbenchmark", **out}), flush=True)


def run_gemm(a):
    """snp_gemm_bf16 (tcgen05 MMA, TMA-fed) on seeded BF16 operands: CUDA-event time per call
    after warm-up and dense TFLOP/s (2 M N K per call) against the measured BF16 peak."""
    import torch

    from snoopy_b200 import _lib

    M, N, K = a.gemm
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.empty(M, N, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")

    def call():
        _lib.call("snp_gemm_bf16", M, N, K, _lib.ptr(A), K, _lib.ptr(B), K, None, 0, _lib.ptr(C), N, None, N,
                  _lib.ptr(err), _lib.stream_ptr())

    for _ in range(max(a.warmup, 1)):
        call()
    reps = max(a.steps, 1) * 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        call()
    e1.record()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ms = e0.elapsed_time(e1) / reps
    ref = A.float() @ B.float().T
    rel = float(((C - ref).abs().max() / ref.abs().max()).item())
    tf = 2.0 * M * N * K / (ms / 1e3) / 1e12
    peak = None
    try:
        pk = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")))
        peak = pk.get("bf16_tflops")
    except Exception:
        pass
    print(json.dumps({"metric": "bf16 GEMM", "M": M, "N": N, "K": K, "ms": ms, "tflops": tf,
                      "peak_tflops": peak, "frac": (tf / peak) if peak else None, "max_rel_err_vs_fp32": rel}),
          flush=True)


if __name__ == "__main__":
    a = parse()
    if a.assembly_grid:
        run_assembly_grid(a)
    elif a.gemm:
        run_gemm(a)
    elif a.warm_start_family:
        run_warm_start_family(a)
    elif a.batched:
        run_batched(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
