"""The batched Newton solver (snp_batch_*, ``batch.BatchSolver``): variants of the batched
family solved by one set of launches with the whole Newton loop in one CUDA graph.

* every variant converges to the 1e-8 relative residual, and its field matches the
  single-problem solver's (both stop at 1e-8, so the fields agree to that level);
* a variant's answer is bitwise independent of its batchmates, of their order, of the
  autotuner's launch shapes and of whether the loop runs as a graph or host-driven;
* float32 Jacobian and CG inside the float64 Newton loop reach the same field;
* the oracle on the reference's C kernels finds the batched answers at the 1e-8 residual;
* warm starts: a converged start needs no step, a start worse than x = 0 is dropped.
"""

import os

import numpy as np
import pytest

from helpers import oracle_relative_residual, rel_max
from snoopy_b200 import batch as B
from snoopy_b200 import mesh as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def family():
    V = B.sample_variants(6, seed=3)
    for v in V:
        v["tets"] = min(v["tets"], 40000)
    return [B.Instance(v) for v in V]


@pytest.fixture(scope="module")
def batched(family):
    bs = B.BatchSolver(family)
    st = bs.solve(1e-8)
    xs = [ins.x.clone() for ins in family]
    return bs, st, xs


def _iron_B(ins, x):
    msh = ins.mesh
    sel = msh.domain_elements(M.TAG_IRON)[::3]
    return ins.solver.curl_curl_factory.compute_B_at_points(x, msh.element_centroids()[sel], sel)


def test_batch_converges_and_matches_single_solver(family, batched):
    bs, st, xs = batched
    assert bs.info()["graph"] == 1
    assert {ins.v["kind"] for ins in family} == {"reduced", "total"}
    seq = B.solve_one_by_one(family, rtol=1e-8)
    for ins, s_b, s_1, xb in zip(family, st, seq, xs):
        assert s_b["status"] == 0 and s_b["rel_res"] <= 1e-8, (ins.v, s_b)
        assert s_1["rel_res"] <= 1e-8
        assert abs(s_b["newton_iterations"] - s_1["newton_iterations"]) <= 2
        assert rel_max(_iron_B(ins, xb), _iron_B(ins, ins.x)) < 1e-6


def test_batch_answer_independent_of_batchmates(family, batched):
    bs, st, xs = batched
    # alone
    for k in (0, 3):
        one = B.BatchSolver([family[k]])
        s1 = one.solve(1e-8)[0]
        assert bool((family[k].x == xs[k]).all()), k
        assert s1["newton_iterations"] == st[k]["newton_iterations"]
        assert s1["cg_iterations"] == st[k]["cg_iterations"]
    # reversed order
    rev = B.BatchSolver(family[::-1])
    rev.solve(1e-8)
    for ins, x in zip(family, xs):
        assert bool((ins.x == x).all())


def test_batch_tuner_and_host_loop_change_no_bits(family, batched):
    bs, st, xs = batched
    info = bs.tune("fp64")
    assert info["pass1_block"] in (128, 256, 512) and info["asm_waves"] in (1, 2)
    assert min(info["tuned_pass1_us"]) > 0 and min(info["tuned_asm_us"]) > 0
    bs.solve(1e-8)
    for ins, x in zip(family, xs):
        assert bool((ins.x == x).all())
    os.environ["SNP_BATCH_GRAPH"] = "0"
    try:
        host = B.BatchSolver(family)
    finally:
        del os.environ["SNP_BATCH_GRAPH"]
    assert host.info()["graph"] == 0
    host.solve(1e-8)
    for ins, x in zip(family, xs):
        assert bool((ins.x == x).all())


def test_batch_mixed_precision_reaches_the_field(family, batched):
    bs, st, xs = batched
    sm = bs.solve(1e-8, precision="mixed")
    for ins, s, x64 in zip(family, sm, xs):
        assert s["status"] == 0 and s["rel_res"] <= 1e-8, s
        assert rel_max(_iron_B(ins, ins.x), _iron_B(ins, x64)) < 1e-6


def test_batch_answers_at_the_oracle_residual(oracle_mod, family, batched):
    bs, st, xs = batched
    for k in (0, 1):  # one reduced, one total-potential variant
        assert oracle_relative_residual(oracle_mod, family[k], xs[k].cpu().numpy()) <= 1.5e-8


def test_batch_warm_starts(family, batched):
    import torch

    bs, st, xs = batched
    res0 = [s["res0"] for s in st]
    # converged starts: no Newton step; a start far worse than zero: dropped for x = 0
    bad = torch.full_like(xs[1], 10.0)
    x0s = [x.clone() for x in xs]
    x0s[1] = bad
    sw = bs.solve(1e-8, x0s=x0s, res_refs=res0)
    for k, (ins, s) in enumerate(zip(family, sw)):
        assert s["status"] == 0 and s["rel_res"] <= 1e-8
        if k == 1:
            assert s["start_dropped"] == 1 and s["newton_iterations"] == st[1]["newton_iterations"]
        else:
            assert s["start_dropped"] == 0 and s["newton_iterations"] == 0


def test_batch_needs_block_jacobi(family):
    from snoopy_b200 import _lib

    ins = family[2]
    ins.eng.set_preconditioner("jacobi")
    try:
        with pytest.raises(_lib.SnpError) as e:
            B.BatchSolver([ins])
        assert "block-Jacobi" in str(e.value)
    finally:
        ins.eng.set_preconditioner("block")
