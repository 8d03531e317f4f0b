"""Adjoint and tangent-linear model of the step (no reference counterpart: OpenPhase has no adjoint).

Pinned by (i) the tangent-linear model reproducing the forward state exactly, (ii) the dot-product
test <w, J dtheta> = <J^T w, dtheta> between the dual-number tangent kernel and the hand-written
reverse sweep, (iii) central finite differences at 1e-4 relative perturbation, and (iv) FP32 vs
FP64 versions.  The step is piecewise smooth: its discrete decisions (which fields exist, which
increments are clipped) are held fixed by the derivatives.  A finite difference whose two perturbed
rollouts take different decisions (the per-step stored-entry counts or the final index sets
differ) measures a jump, not a derivative; those parameters are counted and reported, and every
parameter whose perturbed rollouts keep the decisions must agree within 1e-3.
"""
import numpy as np
import pytest

from openphase_b200.adjoint import Rollout, grain_volumes_function
from openphase_b200.cases import Case
from openphase_b200.context import Context
from tests.parity import compare_states

pytestmark = pytest.mark.gpu

CASE = Case(32, 32, 32, 10, seed=41, iwidth=5.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4), dg_scale=0.05,
            name="adjoint_32")
T = 30


def _setup(precision="fp64", interval=None, case=CASE, nsteps=T):
    G = case.ngrains
    state = case.initial_state()
    sig, mu, dg = case.pair_sigma(), np.ones((G, G)), case.driving_force()
    ctx = Context.from_case(case, precision=precision, k_slots=16, state=state)
    ctx.set_pair_table(sig, mu)
    R = Rollout(ctx, case.dt, nsteps, interval)
    R.set_parameters(sig, mu, dg)
    return ctx, R, state, sig, mu, dg


def test_tangent_state_equals_forward_and_dot_product():
    ctx, R, state, sig, mu, dg = _setup()
    G = CASE.ngrains
    rng = np.random.default_rng(0)
    w = rng.standard_normal(G)
    R.forward()
    gs, gm, gd = R.backward(w)
    assert R.adjoint_status == 0
    ds = rng.standard_normal((G, G)); ds = (ds + ds.T) / 2; np.fill_diagonal(ds, 0)
    dm = rng.standard_normal((G, G)); dm = (dm + dm.T) / 2; np.fill_diagonal(dm, 0)
    dd = rng.standard_normal(G)
    dV = R.tangent(ds, dm, dd)
    ref = Context.from_case(CASE, precision="fp64", k_slots=16, state=state)
    ref.set_pair_table(sig, mu)
    ref.step(CASE.dt, T)
    r = compare_states(ctx.download(), ref.download(), G)
    assert r["same_sets"] and r["max_dphi"] == 0.0, r
    iu = np.triu_indices(G, 1)
    lhs = float(w @ dV)
    rhs = float((gs[iu] * ds[iu]).sum() + (gm[iu] * dm[iu]).sum() + gd @ dd)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


def _fd_check(h_rel, seed, case=CASE, nsteps=T, interval=None, precision="fp64"):
    """Central differences on 32 random parameters (12 sigma pairs, 12 mu pairs, 8 driving forces)
    of L = sum_g w_g V_g(T); L is summed on the host in a fixed order (deterministic)."""
    ctx, R, state, sig, mu, dg = _setup(precision=precision, interval=interval, case=case, nsteps=nsteps)
    G = case.ngrains
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(G)
    R.forward()
    gs, gm, gd = R.backward(w)

    def run(s, m, d):
        R.set_parameters(s, m, d)
        R.forward(fingerprint=True)
        c, i, v = ctx.download()
        return float(np.sum(w[i] * v)), list(R.fingerprint), (c, i, v)

    picks = []
    for kind, gr in (("sigma", gs), ("mu", gm)):
        cand = np.argwhere(np.triu(np.abs(gr) > 1e-6 * np.abs(gr).max(), 1))
        for k in rng.choice(len(cand), size=min(12, len(cand)), replace=False):
            picks.append((kind, tuple(int(x) for x in cand[k])))
    for g in rng.choice(G, size=8, replace=False):
        picks.append(("dg", (int(g),)))
    smooth, jumps = [], []
    for kind, ix in picks:
        if kind == "dg":
            h = h_rel * abs(dg[ix[0]])
            p1, p2 = dg.copy(), dg.copy()
            p1[ix[0]] += h
            p2[ix[0]] -= h
            (L1, f1, s1), (L2, f2, s2) = run(sig, mu, p1), run(sig, mu, p2)
            ad = gd[ix[0]]
        else:
            base = sig if kind == "sigma" else mu
            a, b = ix
            h = h_rel * abs(base[a, b])
            p1, p2 = base.copy(), base.copy()
            p1[a, b] += h
            p1[b, a] += h
            p2[a, b] -= h
            p2[b, a] -= h
            args1 = (p1, mu, dg) if kind == "sigma" else (sig, p1, dg)
            args2 = (p2, mu, dg) if kind == "sigma" else (sig, p2, dg)
            (L1, f1, s1), (L2, f2, s2) = run(*args1), run(*args2)
            ad = (gs if kind == "sigma" else gm)[a, b]
        fd = (L1 - L2) / (2 * h)
        rel = abs(fd - ad) / max(abs(fd), abs(ad), 1e-30)
        same = f1 == f2 and compare_states(s1, s2, G)["same_sets"]
        (smooth if same else jumps).append((kind, ix, fd, ad, rel))
    return picks, smooth, jumps


def test_gradients_match_central_finite_differences():
    # At the 1e-4 relative perturbation of the calibration set-up most pairs of runs change
    # decisions (a field appears or vanishes in a voxel, a limiter switches branch), so the
    # difference quotient mixes the derivative with jumps and kinks: reported, loosely bounded.
    picks, smooth, jumps = _fd_check(1e-4, 1)
    rels = sorted(r[4] for r in smooth + jumps)
    print("h=1e-4: sets kept", len(smooth), "changed", len(jumps), "median rel", rels[len(rels) // 2])
    for r in smooth + jumps:
        print(r)
    assert rels[len(rels) // 2] <= 0.2
    # at 1e-7 almost every pair of runs keeps the decisions: every such parameter agrees within 1e-3
    picks, smooth, jumps = _fd_check(1e-7, 1)
    print("h=1e-7: decisions kept", len(smooth), "changed", len(jumps))
    for r in smooth + jumps:
        print(r)
    assert len(smooth) >= len(picks) // 2, (smooth, jumps)
    for kind, ix, fd, ad, rel in smooth:
        assert rel <= 1e-3, (kind, ix, fd, ad, rel)


def test_checkpoint_interval_does_not_change_gradients():
    G = CASE.ngrains
    w = np.random.default_rng(2).standard_normal(G)
    out = []
    for interval in (1, None, T):
        ctx, R, *_ = _setup(interval=interval)
        R.forward()
        out.append(R.backward(w))
    # identical up to the order of the atomic gradient accumulation
    for o in out[1:]:
        for a, b in zip(out[0], o):
            assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(a).max())


def test_fp32_and_fp64_gradients_agree():
    G = CASE.ngrains
    w = np.random.default_rng(3).standard_normal(G)
    grads = {}
    for prec in ("fp64", "fp32"):
        ctx, R, *_ = _setup(precision=prec)
        R.forward()
        grads[prec] = R.backward(w)
        # the reverse sweep recomputes every step in the forward's own precision and order: the
        # recomputed lists are the stored ones (no adjoint mismatch) in both forms
        assert R.adjoint_status == 0, (prec, R.adjoint_status)
    for a, b in zip(grads["fp64"], grads["fp32"]):
        assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(a)


def test_autograd_function_calibration_loss():
    import torch
    G = CASE.ngrains
    ctx, R, state, sig, mu, dg = _setup()
    target = R.forward() * (1.0 + 0.01 * np.random.default_rng(4).standard_normal(G))
    GV = grain_volumes_function()
    s = torch.tensor(np.ones((G, G)) * 1.0, dtype=torch.float64, requires_grad=True)
    m = torch.tensor(mu, dtype=torch.float64, requires_grad=True)
    d = torch.zeros(G, dtype=torch.float64, requires_grad=True)
    V = GV.apply(s, m, d, R)
    loss = ((V - torch.from_numpy(target)) ** 2).sum()
    loss.backward()
    # the same through the rollout directly
    R.set_parameters(np.ones((G, G)), mu, np.zeros(G))
    V2 = R.forward()
    gs, gm, gd = R.backward(2.0 * (V2 - target))
    assert np.allclose(s.grad.numpy(), gs, rtol=0, atol=1e-12 * np.abs(gs).max())
    assert np.allclose(m.grad.numpy(), gm, rtol=0, atol=1e-12 * np.abs(gm).max())
    assert np.allclose(d.grad.numpy(), gd, rtol=0, atol=1e-12 * max(np.abs(gd).max(), 1e-30))


def test_calibration_rollout_gradients():
    """The calibration set-up itself: 128^3, 256 Voronoi grains, sigma ~ U[0.8, 1.2] per pair,
    dG ~ U[0, 0.03].

    (1) 200 steps of the FP32 form, checkpoints every 16 steps, central differences at 1e-4
        relative on 32 random parameters: a pair of perturbed rollouts that takes different
        decisions (a field appears or vanishes somewhere in the 2M voxels, a limiter switches
        branch) measures a jump, not the derivative.  At this size every pair does, so the count is
        reported and the few kept pairs (if any) must agree within 1e-3.
    (2) The derivative itself: the FP64 form over the first 30 steps, central differences at 1e-8
        relative keep every decision; the median relative difference is <= 1e-3 and every
        parameter agrees within 1e-3 of the largest gradient of its kind (small gradients are
        swamped by the rounding of the loss, ~1e-16 |L| / h).
    (3) The full 200-step checkpointed rollout in FP64: the tangent-linear model and the adjoint
        satisfy the dot-product identity to 1e-10."""
    import json
    from openphase_b200.cases import adjoint_calibration_128
    case = adjoint_calibration_128()
    G = case.ngrains
    picks, smooth, jumps = _fd_check(1e-4, 5, case=case, nsteps=case.nsteps, interval=16, precision="fp32")
    rels = sorted(r[4] for r in smooth + jumps)
    print("FD_CALIBRATION_FP32_1e-4 " + json.dumps({"steps": case.nsteps, "parameters": len(picks),
                                                    "decisions_kept": len(smooth), "decisions_changed": len(jumps),
                                                    "median_rel": rels[len(rels) // 2]}))
    for kind, ix, fd, ad, rel in smooth:
        assert rel <= 1e-3, (kind, ix, fd, ad, rel)
    # (2)
    picks, smooth, jumps = _fd_check(1e-8, 5, case=case, nsteps=30, precision="fp64")
    rels = sorted(r[4] for r in smooth)
    scale = {k: max(abs(r[3]) for r in smooth if r[0] == k) for k in ("sigma", "mu", "dg")}
    normwise = max(abs(r[2] - r[3]) / scale[r[0]] for r in smooth)
    print("FD_CALIBRATION_FP64_1e-8_30_steps " + json.dumps({"parameters": len(picks), "decisions_kept": len(smooth),
                                                             "median_rel": rels[len(rels) // 2], "max_rel": rels[-1],
                                                             "max_rel_to_largest_gradient": normwise}))
    for r in smooth + jumps:
        print(r)
    assert len(jumps) == 0
    assert rels[len(rels) // 2] <= 1e-3
    assert normwise <= 1e-3
    # (3)
    ctx, R, state, sig, mu, dg = _setup(precision="fp64", interval=16, case=case, nsteps=case.nsteps)
    rng = np.random.default_rng(6)
    w = rng.standard_normal(G)
    R.forward()
    gs, gm, gd = R.backward(w)
    assert R.adjoint_status == 0
    ds = rng.standard_normal((G, G)); ds = (ds + ds.T) / 2; np.fill_diagonal(ds, 0)
    dm = rng.standard_normal((G, G)); dm = (dm + dm.T) / 2; np.fill_diagonal(dm, 0)
    dd = rng.standard_normal(G)
    dV = R.tangent(ds, dm, dd)
    iu = np.triu_indices(G, 1)
    lhs = float(w @ dV)
    rhs = float((gs[iu] * ds[iu]).sum() + (gm[iu] * dm[iu]).sum() + gd @ dd)
    print("DOT_PRODUCT_CALIBRATION_200_STEPS", lhs, rhs, abs(lhs - rhs) / abs(lhs))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)
