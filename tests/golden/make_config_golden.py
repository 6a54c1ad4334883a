"""Generate the configuration-level fixtures in this directory: the CPU oracle's converged
float64 field at 1000 seeded aperture probes, for the benchmark's window-frame yoke at three
sizes.

For each size the script builds the same seeded mesh, coils and B-H law as ``bench.workload``
(``bench.oracle_problem``),
runs the oracle's residual Newton (``oracle.newton_residual``: the reference's own C kernels
from ``oracle/_ref`` for every assembly and Biot-Savart evaluation, scipy's Jacobi-preconditioned
``cg`` as ``snoopy/red_mvp_solver.py:199-203`` calls it, Eisenstat-Walker inner tolerances and
the energy line search) from A = 0 to a relative residual of 1e-10, and stores B = curl A + B_s
at the probes (``oracle.probe_B``) with the located elements and the solve's counts:

* ``config_c1.npz``  ~40k tets   (the CPU-runnable configuration)
* ``config_c2.npz``  ~1.2M tets  (the benchmark workload)
* ``config_c3.npz``  ~4M tets    (the mixed-precision configuration)

Only these small arrays are stored: the meshes are rebuilt from their seeds by whoever compares.

Usage: ``python tests/golden/make_config_golden.py [c1 c2 c3]`` (needs ``oracle/_ref``; the
~4M-tet solve takes about half an hour and 20 GB of host memory).  Sizes run in parallel
processes.
"""

import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (ROOT, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

CONFIGS = {"c1": 40_000, "c2": 1_200_000, "c3": 4_000_000}
RTOL = 1e-10
N_PROBES = 1000


def make(name):
    import numpy as np

    import bench
    import oracle as O

    t0 = time.perf_counter()
    P = bench.oracle_problem(CONFIGS[name])
    msh = P["msh"]
    t1 = time.perf_counter()
    x, st = O.newton_residual(P["A"], P["mask"], P["sf"], rtol=RTOL, forcing="ew", line_search="energy", cg_rtol=0.1,
                              max_newton_iterations=80)
    t2 = time.perf_counter()
    assert st["rel_res"] <= RTOL, st["rel_res"]
    probes = msh.geometry.aperture_probes(N_PROBES)
    B, el = O.probe_B(msh.nodes, msh.cells, msh.elem_edges, msh.orientations, P["curls"], P["phi"], P["dphi"], P["q"],
                      P["w"], msh.num_dofs, x, probes, P["coils"])
    out = os.path.join(HERE, f"config_{name}.npz")
    np.savez_compressed(out, probes=probes, elements=el.astype(np.int32), B=B, rtol=RTOL, rel_res=st["rel_res"],
                        newton=st["newton"], cg=int(sum(st["cg"])), assemblies=st["assemblies"],
                        tets=msh.num_elements, dofs=msh.num_dofs, solve_s=t2 - t1, setup_s=t1 - t0)
    print(f"{name}: {msh.num_elements} tets, {msh.num_dofs} DoFs, Newton {st['newton']}, CG {sum(st['cg'])}, "
          f"rel. residual {st['rel_res']:.2e}, solve {t2 - t1:.0f} s -> {out}", flush=True)


if __name__ == "__main__":
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    names = [a for a in sys.argv[1:] if a in CONFIGS] or list(CONFIGS)
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=make, args=(n,)) for n in names]
    for p in procs:
        p.start()
    for p in procs:
        p.join()
    sys.exit(max(p.exitcode for p in procs))
