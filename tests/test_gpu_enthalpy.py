"""flag_total_enthalpy: convection by full_convec_ijk_H (elem_convec.f90:20-208) as rk_4_main
selects it (time_integ.f90:361-365), against the oracle.  FP64 bound 1e-12 relative per field
(the rest of the FP64 path); the mixed path against FP64 with the bounds of the enthalpy path's
mixed test on the same 4^3 mesh (stage RHS 1e-3, state after 10 steps 1e-6); the adjoints by
dot-product tests against the oracle's dual-number JVP (1e-11)."""
import dataclasses

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
    m = M.periodic_box(4, jitter=0.05, seed=5)
    prm = dataclasses.replace(M.TGVParams(), flag_total_enthalpy=1)
    om = oracle.OracleMesh(m)
    gm = S.Sod2dMesh(m, prm)
    st0 = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=5)
    dt = oracle.adapt_dt(om, st0, prm)
    st1 = st0.copy()
    oracle.rk4(om, prm, st1, dt, nsteps=1)  # a state with mu_e > 0
    return dict(M=M, S=S, m=m, prm=prm, om=om, gm=gm, st0=st0, st1=st1, dt=dt, torch=torch)


def test_full_convec_ijk_H_entry(env, oracle):
    torch, gm, om, st = env["torch"], env["gm"], env["om"], env["st1"]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).cuda()
    Rm, Rmo, Re = gm.full_convec_ijk_H(dev(st.u), dev(st.q), dev(st.rho), dev(st.pr), dev(st.E))
    rRm, rRmo, rRe = oracle.convec_H(om, st.u, st.q, st.rho, st.pr, st.E)
    assert rel_l2(Rm.cpu().numpy(), rRm) < TOL64
    assert rel_l2(t2n(Rmo), rRmo) < TOL64
    assert rel_l2(Re.cpu().numpy(), rRe) < TOL64


def test_stage_rhs_and_steps_fp64(env, oracle):
    S, gm, om, prm, dt = env["S"], env["gm"], env["om"], env["prm"], env["dt"]
    st = env["st1"].copy()
    ref = oracle.rk4(om, prm, st.copy(), dt, nsteps=1, capture_stage=1)
    s = S.Sod2dState.from_host(env["st1"], gm.nelem)
    out = gm.rhs(s, precision=S.FP64)
    for k in ("Rmass", "Rener"):
        assert rel_l2(out[k].cpu().numpy(), ref[k]) < TOL64, k
    assert rel_l2(t2n(out["Rmom"]), ref["Rmom"]) < TOL64
    # the energy residual differs from the enthalpy form's (the flag reaches the kernel)
    gm.set_params(dataclasses.replace(prm, flag_total_enthalpy=0))
    out_h = gm.rhs(s, precision=S.FP64)
    gm.set_params(prm)
    assert rel_l2(out_h["Rener"].cpu().numpy(), ref["Rener"]) > 1e-9
    ref3 = env["st0"].copy()
    oracle.rk4(om, prm, ref3, dt, nsteps=3)
    a = S.Sod2dState.from_host(env["st0"], gm.nelem)
    a.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(a, precision=S.FP64, update_dt=False)
    h = a.to_host()
    for k in ("rho", "q", "E", "u", "pr", "eta", "mu_fluid", "mu_e"):
        assert rel_l2(h[k], getattr(ref3, k)) < TOL64, k


def test_mixed_and_graph(env):
    S, gm, torch, dt = env["S"], env["gm"], env["torch"], env["dt"]
    s = S.Sod2dState.from_host(env["st1"], gm.nelem)
    r64 = gm.rhs(s, precision=S.FP64)
    r32 = gm.rhs(s, precision=S.MIXED)
    for k in r64:
        assert rel_l2(t2n(r32[k]), t2n(r64[k])) < 1e-3, k
    a = S.Sod2dState.from_host(env["st0"], gm.nelem); a.dt.fill_(dt)
    b = S.Sod2dState.from_host(env["st0"], gm.nelem); b.dt.fill_(dt)
    c = S.Sod2dState.from_host(env["st0"], gm.nelem); c.dt.fill_(dt)
    for _ in range(10):
        gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    gm.rk4_steps(b, 10, precision=S.FP64)
    gm.rk4_steps(c, 10, precision=S.MIXED)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    for k in ("rho", "q", "E"):
        assert rel_l2(t2n(getattr(c, k)), t2n(getattr(a, k))) < 1e-6, k


def test_adjoint_total_enthalpy(env, oracle):
    """The RHS and step adjoints of the total-enthalpy path: dot-product tests against the
    oracle's dual-number JVP of the same map (bound 1e-11 relative to sum |w_i (J v)_i|)."""
    from _util import oracle_step_jvp
    S, gm, om, prm, torch, dt = env["S"], env["gm"], env["om"], env["prm"], env["torch"], env["dt"]
    st = env["st1"]
    rng = np.random.default_rng(41)
    rnd = lambda a: rng.standard_normal(a.shape) * np.abs(a).mean()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    v = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    # stage RHS
    _, dR = oracle.rhs_jvp(om, prm, st, *v)
    w = np.stack([rnd(st.rho) for _ in range(5)])
    g = gm.rhs_vjp(dev(st.rho), dev(st.q.T), dev(st.E), dev(st.mu_e.T), dev(st.mu_factor), dev(w[0]), dev(w[1:4]),
                   dev(w[4]))
    lhs = float((w * dR).sum())
    rhs = sum(float((gi.cpu().numpy() * vi).sum()) for gi, vi in zip(g, (v[0], v[1].T, v[2])))
    assert abs(lhs - rhs) <= 1e-11 * float(np.abs(w * dR).sum()), (lhs, rhs)
    # one RK4 step
    y1, dy1 = oracle_step_jvp(oracle, om, prm, st, dt, v)
    wb = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    dtd = torch.full((1,), dt, dtype=torch.float64, device="cuda")
    out = gm.rk4_step_vjp(dev(st.rho), dev(st.q.T), dev(st.E), dev(st.mu_e.T), dev(st.mu_factor), dtd,
                          dev(wb[0]), dev(wb[1].T), dev(wb[2]))
    gs = [o.cpu().numpy() for o in out]
    gs[1] = gs[1].T
    terms = [wb[f] * dy1[f] for f in range(3)]
    lhs = sum(t.sum() for t in terms)
    rhs = sum((gs[f] * v[f]).sum() for f in range(3))
    assert abs(lhs - rhs) <= 1e-11 * sum(np.abs(t).sum() for t in terms), (lhs, rhs)


def test_set_params_drops_captured_graphs(env):
    """A step graph captured before sod_mesh_set_params must not be replayed with the old
    parameters: the same state tensors (the same graph key) stepped again after the change."""
    S, gm, torch, prm, dt = env["S"], env["gm"], env["torch"], env["prm"], env["dt"]
    a = S.Sod2dState.from_host(env["st0"], gm.nelem); a.dt.fill_(dt)
    gm.set_params(dataclasses.replace(prm, flag_total_enthalpy=0))
    gm.rk4_steps(a, 2, precision=S.FP64)  # captures a graph with the enthalpy form
    e_h = a.E.clone()
    fresh = S.Sod2dState.from_host(env["st0"], gm.nelem)
    for f in S.Sod2dState.FIELDS:
        getattr(a, f).copy_(getattr(fresh, f))
    a.dt.fill_(dt)
    gm.set_params(prm)
    gm.rk4_steps(a, 2, precision=S.FP64)
    b = S.Sod2dState.from_host(env["st0"], gm.nelem); b.dt.fill_(dt)
    for _ in range(2):
        gm.rk_4_main(b, precision=S.FP64, update_dt=True)
    torch.cuda.synchronize()
    for k in ("rho", "E", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    assert not torch.equal(a.E, e_h)
