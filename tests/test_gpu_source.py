"""Constant momentum source term (the source_term argument of rk_4_main, mom_source_const_vect,
elem_source.f90:20-55) on the device against the oracle: the stage residual and three RK4 steps
(FP64 1e-12 per field; mixed vs FP64 1e-7; graph == eager bitwise, and a graph sees values
changed in place), and the step adjoint (recorded == recomputed stage states; a 4-step rollout
against central differences at h = 1e-5 and 1e-6, 1e-6)."""
import numpy as np
import pytest

from _util import rel_l2, t2n

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


@pytest.fixture(scope="module")
def env(oracle):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    m = M.periodic_box(3, jitter=0.05, seed=12)
    prm = M.TGVParams(Re=800.0)
    st0 = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=12)
    rng = np.random.default_rng(12)
    src = np.asfortranarray(np.column_stack([np.full(m.npoin, 0.2), 0.05 * rng.standard_normal((m.npoin, 2))]))
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    gm = S.Sod2dMesh(m, prm)
    s_dev = torch.from_numpy(np.ascontiguousarray(src.T)).cuda()
    gm.set_source_term(s_dev)
    return dict(torch=torch, M=M, S=S, m=m, prm=prm, st0=st0, src=src, om=om, dt=dt, gm=gm, s_dev=s_dev)


def test_stage_residual_and_steps(env, oracle):
    S, gm, om, prm, dt, st0, src = (env[k] for k in ("S", "gm", "om", "prm", "dt", "st0", "src"))
    ref = oracle.rk4(om, prm, st0.copy(), dt, nsteps=1, capture_stage=1, source=src)
    s = S.Sod2dState.from_host(st0, gm.nelem)
    out = gm.rhs(s, precision=S.FP64)
    assert rel_l2(t2n(out["Rmom"]), ref["Rmom"]) < TOL64
    for k in ("Rmass", "Rener"):
        assert rel_l2(out[k].cpu().numpy(), ref[k]) < TOL64, k
    plain = oracle.rk4(om, prm, st0.copy(), dt, nsteps=1, capture_stage=1)
    assert rel_l2(plain["Rmom"], ref["Rmom"]) > 1e-6  # the source reaches the residual
    ref3 = st0.copy()
    oracle.rk4(om, prm, ref3, dt, nsteps=3, source=src)
    a = S.Sod2dState.from_host(st0, gm.nelem)
    a.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(a, precision=S.FP64, update_dt=False)
    h = a.to_host()
    for k in ("rho", "q", "E", "u", "pr", "eta", "mu_fluid", "mu_e"):
        assert rel_l2(h[k], getattr(ref3, k)) < TOL64, k


def test_graph_mixed_and_in_place_values(env):
    torch, S, gm, dt, st0 = (env[k] for k in ("torch", "S", "gm", "dt", "st0"))
    a = S.Sod2dState.from_host(st0, gm.nelem); a.dt.fill_(dt)
    b = S.Sod2dState.from_host(st0, gm.nelem); b.dt.fill_(dt)
    c = S.Sod2dState.from_host(st0, gm.nelem); c.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    gm.rk4_steps(b, 3, precision=S.FP64)
    for _ in range(3):
        gm.rk_4_main(c, precision=S.MIXED, update_dt=True)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    for k in ("rho", "q", "E"):
        assert float((getattr(c, k) - getattr(a, k)).norm() / getattr(a, k).norm()) < 1e-7, k
    # values changed in place reach an already captured graph (the mesh keeps the pointer)
    gm.rk4_steps(b, 1, precision=S.FP64)  # captures the 1-step graph
    gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    keep = env["s_dev"].clone()
    env["s_dev"].mul_(2.0)
    gm.rk4_steps(b, 1, precision=S.FP64)  # replays it
    gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    torch.cuda.synchronize()
    env["s_dev"].copy_(keep)
    assert torch.equal(a.q, b.q)
    # without the source the step differs
    gm.set_source_term(None)
    d = S.Sod2dState.from_host(st0, gm.nelem); d.dt.fill_(dt)
    e = S.Sod2dState.from_host(st0, gm.nelem); e.dt.fill_(dt)
    gm.rk_4_main(d, precision=S.FP64, update_dt=False)
    gm.set_source_term(env["s_dev"])
    gm.rk_4_main(e, precision=S.FP64, update_dt=False)
    assert not torch.equal(d.q, e.q)


def test_step_adjoint_with_source(env):
    from sod2d_refmap_b200.adjoint import Sod2dRollout, replay, trajectory_coefficients, _clone_state
    torch, S, gm, dt, st0 = (env[k] for k in ("torch", "S", "gm", "dt", "st0"))
    s = S.Sod2dState.from_host(st0, gm.nelem)
    s.dt.fill_(dt)
    gm.rk_4_main(s, precision=S.FP64, update_dt=True)
    # recorded and recomputed stage states give the same VJP (the adjoint's own stage gather
    # applies the source)
    stages = torch.zeros(15 * gm.npoin, dtype=torch.float64, device="cuda")
    t = _clone_state(s)
    y0 = (t.rho.clone(), t.q.clone(), t.E.clone(), t.mu_e.clone())
    gm.rk_4_main_record(t, stages, update_dt=False)
    rng = np.random.default_rng(5)
    bars = [torch.from_numpy(rng.standard_normal(x.shape)).cuda() for x in (s.rho, s.q, s.E)]
    g1 = gm.rk4_step_vjp(*y0, s.mu_factor, s.dt, *bars, stages=stages)
    g2 = gm.rk4_step_vjp(*y0, s.mu_factor, s.dt, *bars, stages=None)
    for x, y in zip(g1, g2):
        assert torch.equal(x, y)
    K = 4
    rho = s.rho.clone().requires_grad_(True)
    q = s.q.clone().requires_grad_(True)
    E = s.E.clone().requires_grad_(True)
    rK, qK, EK = Sod2dRollout.apply(gm, s, rho, q, E, K, 2)
    (0.5 * (qK * qK).sum()).backward()
    v = [torch.from_numpy(rng.standard_normal(x.shape)).cuda() * x.abs().mean() for x in (s.rho, s.q, s.E)]
    dL = float(sum((g * d).sum() for g, d in zip((rho.grad, q.grad, E.grad), v)).item())
    mus, dts = trajectory_coefficients(gm, s, K)

    def L_at(h):
        u = _clone_state(s)
        u.rho.add_(h * v[0]); u.q.add_(h * v[1]); u.E.add_(h * v[2])
        replay(gm, u, mus, dts)
        return 0.5 * float((u.q * u.q).sum().item())
    # h = 1e-4 leaves an O(h^2) truncation of ~1e-6 relative on this forced flow
    for h in (1e-5, 1e-6):
        fd = (L_at(h) - L_at(-h)) / (2 * h)
        assert abs(fd - dL) <= 1e-6 * abs(dL), (h, fd, dL)
