"""LES path: rk_4_main with flag_les = 1 (Vreman sgs_visc after each step, mu_sgs in the
diffusion and in the CFL dt) against the oracle.  FP64 bound 1e-12 relative per field (as the
rest of the FP64 path); the mixed path against FP64 within 1e-7 on the state after 3 steps of
this coarse 4^3 case (the stage RHS error of the mixed path is <= 1e-6; the state error is of
order dt times that)."""
import numpy as np
import pytest

from _util import rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


@pytest.fixture(scope="module")
def env(oracle):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    m = M.periodic_box(4, jitter=0.05, seed=4)
    prm = M.TGVParams(flag_les=1, Re=800.0)
    om = oracle.OracleMesh(m)
    gm = S.Sod2dMesh(m, prm)
    st0 = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=6)
    dt = oracle.adapt_dt(om, st0, prm)
    return dict(M=M, S=S, m=m, prm=prm, om=om, gm=gm, st0=st0, dt=dt, torch=torch)


def test_les_steps_fp64_vs_oracle(env, oracle):
    S, gm, om, prm, dt = env["S"], env["gm"], env["om"], env["prm"], env["dt"]
    ref = env["st0"].copy()
    oracle.rk4(om, prm, ref, dt, nsteps=3)
    assert np.abs(ref.mu_sgs).max() > 0  # the SGS viscosity is active
    s = S.Sod2dState.from_host(env["st0"], gm.nelem)
    s.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    h = s.to_host()
    for k in ("rho", "q", "E", "u", "pr", "Tem", "mu_fluid", "mu_e", "mu_sgs"):
        err = rel_l2(h[k], getattr(ref, k))
        assert err < TOL64, f"{k}: rel L2 {err:.3e}"


def test_les_dt_uses_new_mu_sgs(env, oracle):
    """dt after a step (adapt_dt_cfl with the updated mu_sgs, CFDSolverBase.f90:1592)."""
    S, gm, om, prm, dt = env["S"], env["gm"], env["om"], env["prm"], env["dt"]
    ref = env["st0"].copy()
    oracle.rk4(om, prm, ref, dt, nsteps=1)
    dt_ref = oracle.adapt_dt(om, ref, prm)
    s = S.Sod2dState.from_host(env["st0"], gm.nelem)
    s.dt.fill_(dt)
    gm.rk_4_main(s, precision=S.FP64, update_dt=True)
    assert abs(float(s.dt.item()) - dt_ref) <= 1e-13 * dt_ref


def test_les_graph_matches_eager_and_mixed_close(env):
    S, gm, torch = env["S"], env["gm"], env["torch"]
    a = S.Sod2dState.from_host(env["st0"], gm.nelem); a.dt.fill_(env["dt"])
    b = S.Sod2dState.from_host(env["st0"], gm.nelem); b.dt.fill_(env["dt"])
    c = S.Sod2dState.from_host(env["st0"], gm.nelem); c.dt.fill_(env["dt"])
    for _ in range(3):
        gm.rk_4_main(a, precision=S.FP64, update_dt=True)
        gm.rk_4_main(c, precision=S.MIXED, update_dt=True)
    gm.rk4_steps(b, 3, precision=S.FP64)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "mu_sgs", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    for k in ("rho", "q", "E"):
        assert float((getattr(c, k) - getattr(a, k)).norm() / getattr(a, k).norm()) < 1e-7, k


def _step_jvp(oracle, om, prm, st, dt, v):
    """One rk_4_main step and its JVP by composing oracle_rhs_jvp with the frozen mu_sgs."""
    def _with(base, rho, q, E):
        s = base.copy()
        s.rho = np.ascontiguousarray(rho); s.q = np.asfortranarray(q); s.E = np.ascontiguousarray(E)
        return s
    y0 = (st.rho, st.q, st.E)
    acc_y = [a.copy() for a in y0]
    acc_v = [a.copy() for a in v]
    ys, vs = y0, v
    a_next = [0.5, 0.5, 1.0, None]
    b = [1 / 6, 1 / 3, 1 / 3, 1 / 6]
    for s in range(4):
        R, dR = oracle.rhs_jvp(om, prm, _with(st, *ys), vs[0], vs[1], vs[2], mu_sgs=st.mu_sgs)
        Rc = (R[0], np.asfortranarray(R[1:4].T), R[4])
        dRc = (dR[0], np.asfortranarray(dR[1:4].T), dR[4])
        for f in range(3):
            acc_y[f] = acc_y[f] - dt * b[s] * Rc[f]
            acc_v[f] = acc_v[f] - dt * b[s] * dRc[f]
        if a_next[s] is not None:
            ys = tuple(y0[f] - dt * a_next[s] * Rc[f] for f in range(3))
            vs = tuple(v[f] - dt * a_next[s] * dRc[f] for f in range(3))
    return acc_y, acc_v


def test_les_step_vjp_dot_product(env, oracle):
    """Step adjoint with the frozen mu_sgs: <w, J v> (oracle dual numbers) == <J^T w, v>,
    bound 1e-11 relative to sum |w_i (J v)_i| (the adjoint tests' dot-product bound)."""
    S, gm, om, prm, dt, torch = env["S"], env["gm"], env["om"], env["prm"], env["dt"], env["torch"]
    st = env["st0"].copy()
    oracle.rk4(om, prm, st, dt, nsteps=1)  # mu_e and mu_sgs > 0
    assert np.abs(st.mu_sgs).max() > 0
    rng = np.random.default_rng(31)
    rnd = lambda a: rng.standard_normal(a.shape) * np.abs(a).mean()
    v = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    y1, dy1 = _step_jvp(oracle, om, prm, st, dt, v)
    s = S.Sod2dState.from_host(st, gm.nelem)
    s.dt.fill_(dt)
    gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    h = s.to_host()
    for got, ref in ((h["rho"], y1[0]), (h["q"], y1[1]), (h["E"], y1[2])):
        assert rel_l2(got, ref) < TOL64
    wb = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dtd = torch.full((1,), dt, dtype=torch.float64, device="cuda")
    out = gm.rk4_step_vjp(dev(st.rho), dev(st.q.T), dev(st.E), dev(st.mu_e.T), dev(st.mu_factor), dtd,
                          dev(wb[0]), dev(wb[1].T), dev(wb[2]), mu_sgs=dev(st.mu_sgs.T))
    g = [o.cpu().numpy() for o in out]
    g[1] = g[1].T
    terms = [wb[f] * dy1[f] for f in range(3)]
    lhs = sum(t.sum() for t in terms)
    rhs = sum((g[f] * v[f]).sum() for f in range(3))
    assert abs(lhs - rhs) <= 1e-11 * sum(np.abs(t).sum() for t in terms), (lhs, rhs)
    # without mu_sgs the adjoint is that of another map: the SGS terms are seen
    out0 = gm.rk4_step_vjp(dev(st.rho), dev(st.q.T), dev(st.E), dev(st.mu_e.T), dev(st.mu_factor), dtd,
                           dev(wb[0]), dev(wb[1].T), dev(wb[2]))
    assert not torch.equal(out0[0], out[0])


def test_les_rollout_gradient_fd(env):
    """Loss 1/2 sum |q_K|^2 after K = 4 LES steps (checkpoints every 2) against central
    differences of the frozen-coefficient map (mu_e, mu_sgs, dt frozen), h = 1e-4 and 1e-6,
    bound 1e-6 relative."""
    from sod2d_refmap_b200.adjoint import Sod2dRollout, replay, trajectory_coefficients, _clone_state
    S, gm, torch, dt = env["S"], env["gm"], env["torch"], env["dt"]
    K = 4
    s = S.Sod2dState.from_host(env["st0"], gm.nelem)
    s.dt.fill_(dt)
    gm.rk_4_main(s, precision=S.FP64, update_dt=True)  # a state whose mu_sgs is already > 0
    rho = s.rho.clone().requires_grad_(True)
    q = s.q.clone().requires_grad_(True)
    E = s.E.clone().requires_grad_(True)
    rK, qK, EK = Sod2dRollout.apply(gm, s, rho, q, E, K, 2)
    (0.5 * (qK * qK).sum()).backward()
    rng = np.random.default_rng(9)
    v = [torch.from_numpy(rng.standard_normal(t.shape)).cuda() * t.abs().mean() for t in (s.rho, s.q, s.E)]
    dL = float(sum((g * d).sum() for g, d in zip((rho.grad, q.grad, E.grad), v)).item())
    mus, dts, sgs = trajectory_coefficients(gm, s, K, with_sgs=True)

    def L_at(h):
        t = _clone_state(s)
        t.rho.add_(h * v[0]); t.q.add_(h * v[1]); t.E.add_(h * v[2])
        replay(gm, t, mus, dts, mu_sgs_seq=sgs)
        return 0.5 * float((t.q * t.q).sum().item())
    for h in (1e-4, 1e-6):
        fd = (L_at(h) - L_at(-h)) / (2 * h)
        assert abs(fd - dL) <= 1e-6 * abs(dL), (h, fd, dL)
