"""The learned warm start: device MLP gradients against the CPU oracle, training, and the
warm-started Newton against zero-start Newton on a morphed yoke family."""

import numpy as np
import pytest
import torch

import mlp_oracle as MO
from snoopy_b200 import morph
from snoopy_b200 import surrogate as SG

pytestmark = pytest.mark.gpu


def _set_weights(mlp, W, b):
    for l in range(mlp.n_layers):
        w = np.zeros(tuple(mlp.W[l].shape), dtype=np.float32)
        w[:, : W[l].shape[1]] = W[l]
        mlp.W[l].copy_(torch.from_numpy(w))
        mlp.b[l].copy_(torch.from_numpy(b[l].astype(np.float32)))
        mlp.Wb[l].copy_(mlp.W[l].to(torch.bfloat16))
        mlp.WTb[l].copy_(mlp.W[l].t().contiguous().to(torch.bfloat16))


def test_mlp_gradients_match_oracle():
    rng = np.random.default_rng(1)
    sizes = (9, 64, 64, 32)
    mlp = SG.MLP(sizes, seed=0)
    W = [rng.normal(0, np.sqrt(2.0 / sizes[i]), (sizes[i + 1], sizes[i])).astype(np.float32) for i in range(3)]
    b = [rng.normal(0, 0.1, sizes[i + 1]).astype(np.float32) for i in range(3)]
    _set_weights(mlp, W, b)
    B = 64
    X = rng.uniform(-1, 1, (B, 9)).astype(np.float32)
    T = rng.normal(0, 1, (B, 32)).astype(np.float32)
    Xb = mlp.input_bf16(torch.from_numpy(X).cuda())
    Tt = torch.from_numpy(T).cuda()
    Y = mlp.forward(Xb, keep=True)
    dY = torch.empty_like(Y)
    from snoopy_b200 import _lib
    _lib.call("snp_mse_grad", Y.numel(), _lib.ptr(Y), _lib.ptr(Tt), 2.0 / Y.numel(), _lib.ptr(dY), None,
              _lib.stream_ptr())
    grads = mlp.backward(dY)
    mlp.check_errors()
    Wp = [np.concatenate([W[0], np.zeros((64, 7), np.float32)], axis=1)] + W[1:]
    Xp = np.concatenate([X, np.zeros((B, 7), np.float32)], axis=1)
    Yo, _ = MO.forward(Wp, b, Xp, bf=True)
    assert np.abs(Y.cpu().numpy() - Yo).max() <= 2e-2 * np.abs(Yo).max()
    go, _ = MO.backward(Wp, b, Xp, T.astype(np.float64), bf=True)
    for l in range(3):
        dW = grads[l][0].cpu().numpy().astype(np.float64)
        db = grads[l][1].cpu().numpy().astype(np.float64)
        rel_w = np.linalg.norm(dW - go[l][0]) / np.linalg.norm(go[l][0])
        rel_b = np.linalg.norm(db - go[l][1]) / np.linalg.norm(go[l][1])
        assert rel_w < 2e-2 and rel_b < 2e-2, (l, rel_w, rel_b)
    assert np.all(grads[0][0].cpu().numpy()[:, 9:] == 0.0)  # padded input columns


def test_mlp_training_reduces_loss():
    rng = np.random.default_rng(2)
    mlp = SG.MLP((9, 128, 128, 16), seed=3)
    A = rng.normal(0, 1, (9, 16))
    X = rng.uniform(-1, 1, (512, 9)).astype(np.float32)
    T = np.sin(X @ A).astype(np.float32)
    Xb = mlp.input_bf16(torch.from_numpy(X).cuda())
    Tt = torch.from_numpy(T).cuda()
    first = None
    for step in range(300):
        Y = mlp.train_step(Xb, Tt, lr=2e-3)
        if first is None:
            first = float(((Y - Tt) ** 2).mean())
    mlp.check_errors()
    last = float(((mlp.forward(Xb) - Tt) ** 2).mean())
    assert last < 0.1 * first, (first, last)


@pytest.fixture(scope="module")
def family_setup():
    fam = morph.YokeMorphFamily(base_tets=20000, seed=5)
    ms = SG.MorphedSolver(fam)
    P = fam.sample(56, seed=11)
    return fam, ms, P[:48], P[48:]


def test_warm_start_cuts_newton_and_keeps_the_answer(family_setup):
    fam, ms, P_train, P_test = family_setup
    ws = SG.WarmStart(ms, n_modes=16, hidden=64, seed=0)
    snaps, st_train = ws.generate(P_train, precision="fp64")
    assert all(s["rel_res"] <= 1e-8 for s in st_train)
    ws.fit(P_train, snaps, epochs=400, batch=48, lr=3e-3)
    assert ws.history[-1][1] < ws.history[0][1]
    probes = fam.geometry.aperture_probes(200, margin=0.03)
    n_zero, n_warm = [], []
    for p in P_test:
        ref = ms.set_member(p)
        el, _ = fam.mesh.locate(probes)  # topology is fixed; locate on the base mesh is close enough inside the aperture
        x0 = ws.predict(p)[0]
        xz, sz = ms.solve(None, rtol=1e-8, precision="fp64", res_ref=ref)
        Bz = ms.solver.curl_curl_factory.compute_B_at_points(xz, probes, el)
        xw, sw = ms.solve(x0, rtol=1e-8, precision="fp64", res_ref=ref)
        Bw = ms.solver.curl_curl_factory.compute_B_at_points(xw, probes, el)
        assert sz["rel_res"] <= 1e-8 and sw["rel_res"] <= 1e-8
        err = np.linalg.norm(Bw - Bz, axis=1).max() / np.linalg.norm(Bz, axis=1).max()
        assert err < 1e-6, err
        n_zero.append(sz["newton_iterations"])
        n_warm.append(sw["newton_iterations"])
    assert np.mean(n_warm) < np.mean(n_zero), (n_warm, n_zero)


def test_bad_start_is_dropped(family_setup):
    fam, ms, P_train, P_test = family_setup
    ref = ms.set_member(P_test[0])
    bad = torch.full((ms.n,), 1e3, dtype=torch.float64, device="cuda")
    x, st = ms.solve(bad, rtol=1e-8, precision="fp64", res_ref=ref)
    assert st["start_dropped"] == 1 and st["rel_res"] <= 1e-8


def test_members_solved_at_once_match_one_at_a_time(family_setup):
    """Warm-started solves of several members at once (one solver, stream and host thread each)
    give bitwise the answers of solving them one after another."""
    fam, ms, P_train, P_test = family_setup
    rng = np.random.default_rng(3)
    mss = [SG.MorphedSolver(fam, stream=torch.cuda.Stream()) for _ in range(3)]
    refs = [m.set_member(p) for m, p in zip(mss, P_test[:3])]
    x0s = [torch.as_tensor(rng.normal(0, 1e-4, ms.n), device="cuda") for _ in range(3)]
    xs, st = SG.solve_members_at_once(mss, x0s, refs, rtol=1e-8, precision="mixed")
    for x, s, x0, p, r in zip(xs, st, x0s, P_test[:3], refs):
        ref = ms.set_member(p)
        assert ref == r
        x1, s1 = ms.solve(x0, rtol=1e-8, precision="mixed", res_ref=ref)
        assert s["rel_res"] <= 1e-8 and s["status"] == 0
        assert s["newton_iterations"] == s1["newton_iterations"] and s["cg_iterations"] == s1["cg_iterations"]
        assert torch.equal(x, x1)


def test_reduced_system_matches_products(family_setup):
    """V^T J V and V^T F from the fused kernel against column-by-column Jacobian products,
    for 80 columns (a full and a partial 64-column block) in float64 and float32."""
    fam, ms, P_train, P_test = family_setup
    ref = ms.set_member(P_test[1])
    x, _ = ms.solve(None, rtol=1e-4, precision="fp64", res_ref=ref)
    eng = ms.eng
    fm = eng.free_mask.bool()
    g = torch.Generator(device="cuda").manual_seed(5)
    V = torch.randn((ms.n, 80), generator=g, device="cuda", dtype=torch.float32)
    F = torch.zeros(ms.n, dtype=torch.float64, device="cuda")
    for prec, dt, tol in (("fp64", torch.float64, 1e-12), ("mixed", torch.float32, 1e-5)):
        eng.assemble_tensors(x, prec, F)
        Jr, gr = eng.reduced_system(V, F, prec)
        JV = torch.empty((ms.n, 80), dtype=torch.float64, device="cuda")
        for j in range(80):
            y = torch.zeros(ms.n, dtype=dt, device="cuda")
            eng.jacobian_apply(V[:, j].to(dt).contiguous(), y, prec)
            JV[:, j] = y.double()
        Vf = torch.where(fm[:, None], V.double(), torch.zeros_like(JV))
        A = Vf.T @ JV
        assert torch.allclose(Jr, Jr.T, rtol=0, atol=1e-12 * float(Jr.abs().max()))
        assert float((Jr - A).abs().max()) <= tol * float(A.abs().max()), prec
        b = Vf.T @ torch.where(fm, F, torch.zeros_like(F))
        assert float((gr - b).abs().max()) <= 1e-12 * float(b.abs().max()), prec
    # a basis view with a leading dimension larger than its width
    eng.assemble_tensors(x, "fp64", F)
    Jr_all, _ = eng.reduced_system(V, None, "fp64")
    Jr_view, _ = eng.reduced_system(V[:, :20], None, "fp64")
    assert float((Jr_view - Jr_all[:20, :20]).abs().max()) <= 1e-12 * float(Jr_all.abs().max())


def test_galerkin_correction_cuts_the_residual(family_setup):
    """One Galerkin Newton step in a POD basis moves a start (the POD mean) closer to the
    member's solution, and Newton from it reaches the same field."""
    fam, ms, P_train, P_test = family_setup
    ws = SG.WarmStart(ms, n_modes=16, hidden=32, seed=0)
    snaps, _ = ws.generate(P_train[:24], precision="fp64")
    ws.mean, ws.U, _, _ = SG.pod(snaps, 16)
    eng = ms.eng
    for p in P_test[:3]:
        ref = ms.set_member(p)
        x0 = ws.mean.clone()
        x1 = ws.correct(x0, modes=16, precision="mixed")
        r0, r1 = eng.residual_norm(x0), eng.residual_norm(x1)
        assert r1 < 0.5 * r0, (r0, r1)
        xz, sz = ms.solve(None, rtol=1e-8, precision="fp64", res_ref=ref)
        xg, sg = ms.solve(x1, rtol=1e-8, precision="fp64", res_ref=ref)
        assert sg["start_dropped"] == 0 and sg["rel_res"] <= 1e-8
        assert sg["cg_iterations"] < sz["cg_iterations"]


def test_galerkin_correction_inside_the_solve(family_setup):
    """The same step taken inside snp_solver_solve (attached basis): applied to the start,
    fewer CG iterations to the same target, and members solved at once give bitwise the
    one-at-a-time answers.  No res_ref, so both starts are kept and held to ||F_free(mean)||."""
    fam, ms, P_train, P_test = family_setup
    ws = SG.WarmStart(ms, n_modes=16, hidden=32, seed=0)
    snaps, _ = ws.generate(P_train[:24], precision="fp64")
    ws.mean, ws.U, _, _ = SG.pod(snaps, 16)
    V = ws.galerkin_basis(16)
    corrected = []
    for p in P_test[:3]:
        ms.set_member(p)
        x0, s0 = ms.solve(ws.mean, rtol=1e-8, precision="mixed")
        ms.attach_basis(V)
        x1, s1 = ms.solve(ws.mean, rtol=1e-8, precision="mixed")
        ms.attach_basis(None)
        assert s0["galerkin_steps"] == 0 and s1["galerkin_steps"] == 1
        assert s1["res0"] == s0["res0"] and s1["res"] <= 1e-8 * s1["res0"]
        assert s1["cg_iterations"] < s0["cg_iterations"], (s0["cg_iterations"], s1["cg_iterations"])
        corrected.append((x1, s1))
    mss = [SG.MorphedSolver(fam, stream=torch.cuda.Stream()) for _ in range(3)]
    for m in mss:
        m.attach_basis(V)
    for m, p in zip(mss, P_test[:3]):
        m.set_member(p)
    xs, st = SG.solve_members_at_once(mss, [ws.mean] * 3, [0.0] * 3, rtol=1e-8, precision="mixed")
    for x, s, (x1, s1) in zip(xs, st, corrected):
        assert s["galerkin_steps"] == 1 and s["cg_iterations"] == s1["cg_iterations"]
        assert torch.equal(x, x1)
