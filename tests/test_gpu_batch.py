"""Many variants solved concurrently (snp_solver_solve_many) against the same solves one at
a time: every instance converges and the answers are bitwise identical (each solve is
deterministic, whatever the GPU overlaps it with)."""

import numpy as np
import pytest

from snoopy_b200 import batch as B

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def instances():
    V = B.sample_variants(6, seed=3)
    for v in V:
        v["tets"] = min(v["tets"], 40000)
    return [B.Instance(v) for v in V]


def test_batched_and_one_by_one_agree(instances):
    seq = B.solve_one_by_one(instances, rtol=1e-8)
    x_seq = [ins.x.cpu().numpy().copy() for ins in instances]
    par = B.solve_many(instances, rtol=1e-8)
    for ins, s1, s2, x1 in zip(instances, seq, par, x_seq):
        assert s1["rel_res"] <= 1e-8 and s2["rel_res"] <= 1e-8, (ins.v, s1["rel_res"], s2["rel_res"])
        assert s1["newton_iterations"] == s2["newton_iterations"]
        assert s1["cg_iterations"] == s2["cg_iterations"]
        assert np.array_equal(x1, ins.x.cpu().numpy())
    kinds = {ins.v["kind"] for ins in instances}
    assert kinds == {"reduced", "total"}


def test_batched_with_fewer_threads(instances):
    ref = [ins.x.cpu().numpy().copy() for ins in instances]
    st = B.solve_many(instances, rtol=1e-8, n_threads=2)
    assert all(s["status"] == 0 for s in st)
    for ins, x in zip(instances, ref):
        assert np.array_equal(x, ins.x.cpu().numpy())
