"""Wall models of rk_4_main (isWallModelOn; evalWallModelReichardt / evalWallModelABL,
mod_wall_model.f90) on the device against the oracle's restatement: the routine as an entry
point (1e-12) and three RK4 steps on a channel with slip-wall-model walls (code 7; FP64 1e-12 per
field), Reichardt with the stage velocity and ABL with a time-averaged velocity and roughness;
graph == eager bitwise, mixed vs FP64 1e-7; the RHS and step adjoints through the wall model
(dot products against the oracle's dual-number JVPs of its own law, 1e-11)."""
import numpy as np
import pytest

from _util import rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
FIELDS = ("rho", "q", "E", "u", "pr", "Tem", "e_int", "eta", "mu_fluid", "mu_e")


@pytest.fixture(scope="module")
def torch_mod():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build
    build.build()
    return torch


def dev(torch, a):
    a = np.asarray(a)
    return torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).cuda()


def host(t):
    a = t.cpu().numpy()
    return np.asfortranarray(a.T) if a.ndim == 2 else a


def case(seed=5, wtype=1):
    from sod2d_refmap_b200 import mesh as M
    m = M.channel_box(3, jitter=0.05, seed=seed, codes=(7, 7))
    prm = M.TGVParams(Re=800.0)
    st = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=seed)
    rng = np.random.default_rng(seed)
    ub = np.asfortranarray(np.column_stack([np.full(m.npoin, 1.0), rng.uniform(-0.1, 0.1, (m.npoin, 2))]))
    bound, codes, bounorm, wgp_b = M.wall_faces(m)
    lw = np.flatnonzero(codes == 7).astype(np.int32)
    zo = np.full(m.npoin, 0.05) if wtype == 2 else None
    walave = np.asfortranarray(st.u * 0.9) if wtype == 2 else None
    return M, m, prm, st, ub, (bound, bounorm, wgp_b, lw, m.extra["point2elem"], m.coord, m.extra["normals"], zo,
                               walave)


def test_wall_model_entry(torch_mod, oracle):
    from sod2d_refmap_b200 import solver as S
    torch = torch_mod
    M, m, prm, st, ub, w = case(seed=6)
    om = oracle.OracleMesh(m)
    owm = oracle.WallModel(1, *w)
    R = np.zeros((m.npoin, 3), order="F")
    oracle.wall_model(om, owm, st.rho, st.u, st.mu_fluid, R)
    assert np.abs(R).max() > 0
    gm = S.Sod2dMesh(m, prm)
    gm.set_wall_model(1, *w[:7])
    Rd = torch.zeros(3, m.npoin, dtype=torch.float64, device="cuda")
    tw = torch.zeros(3, m.npoin, dtype=torch.float64, device="cuda")
    gm.wall_model(dev(torch, st.rho), dev(torch, st.u), dev(torch, st.mu_fluid), Rd, tw)
    assert rel_l2(host(Rd), R) < TOL64
    assert rel_l2(host(tw), owm.tauw) < TOL64
    gm.close()


@pytest.mark.parametrize("wtype", [1, 2])
def test_steps_with_wall_model(torch_mod, oracle, wtype):
    from sod2d_refmap_b200 import _lib, solver as S
    torch = torch_mod
    M, m, prm, st0, ub, w = case(seed=7, wtype=wtype)
    bc = M.bc_params(prm)
    om = oracle.OracleMesh(m)
    bnd = oracle.Boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    owm = oracle.WallModel(wtype, *w)
    dt = oracle.adapt_dt(om, st0, prm)
    ref = st0.copy()
    oracle.rk4(om, prm, ref, dt, nsteps=3, bnd=bnd, wall=owm)
    plain = st0.copy()
    oracle.rk4(om, prm, plain, dt, nsteps=3, bnd=bnd)
    assert rel_l2(plain.q, ref.q) > 1e-10  # the model acts
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    walave = None if w[8] is None else dev(torch, w[8])
    gm.set_wall_model(wtype, *w[:8], walave_u=walave)
    s = S.Sod2dState.from_host(st0, gm.nelem)
    s.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    h = s.to_host()
    for k in FIELDS:
        err = rel_l2(h[k], getattr(ref, k))
        assert err < TOL64, f"{wtype} {k}: rel L2 {err:.3e}"
    assert rel_l2(host(gm.wall_model_tauw()), owm.tauw) < TOL64
    # graph == eager, mixed close to FP64, adjoint refused, removal
    a = S.Sod2dState.from_host(st0, gm.nelem); a.dt.fill_(dt)
    b = S.Sod2dState.from_host(st0, gm.nelem); b.dt.fill_(dt)
    c = S.Sod2dState.from_host(st0, gm.nelem); c.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(a, precision=S.FP64, update_dt=True)
        gm.rk_4_main(c, precision=S.MIXED, update_dt=True)
    gm.rk4_steps(b, 3, precision=S.FP64)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    for k in ("rho", "q", "E"):
        assert float((getattr(c, k) - getattr(a, k)).norm() / getattr(a, k).norm()) < 1e-7, k
    # without the model the step is the boundary-only step
    gm.set_wall_model(wtype, None, None, None, None, None, None, None)
    one = st0.copy()
    oracle.rk4(om, prm, one, dt, nsteps=1, bnd=bnd)
    d = S.Sod2dState.from_host(st0, gm.nelem); d.dt.fill_(dt)
    gm.rk_4_main(d, precision=S.FP64, update_dt=False)
    hd = d.to_host()
    for k in ("rho", "q", "E"):
        assert rel_l2(hd[k], getattr(one, k)) < TOL64, k
    gm.close()


@pytest.mark.parametrize("wtype", [1, 2])
def test_adjoint_through_wall_model(torch_mod, oracle, wtype):
    """<w, J v> == <J^T w, v> for the stage RHS and for one step on the code-7 channel with the
    wall model (Reichardt on the stage velocity; ABL on a time-averaged velocity, which then
    carries no state dependence): J v from the oracle's dual numbers through its law, its
    boundary routine and the read velocity of the slip branch; bound 1e-11 relative to
    sum |w_i (J v)_i|; recorded and recomputed stage states."""
    from _util import oracle_bc_jvp_map, oracle_step_jvp
    from sod2d_refmap_b200 import solver as S
    torch = torch_mod
    M, m, prm, st0, ub, w = case(seed=9, wtype=wtype)
    bc = M.bc_params(prm)
    om = oracle.OracleMesh(m)
    bnd = oracle.Boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    owm = oracle.WallModel(wtype, *w)
    dt = oracle.adapt_dt(om, st0, prm)
    st = st0.copy()
    oracle.rk4(om, prm, st, dt, nsteps=1, bnd=bnd, wall=owm)
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    walave = None if w[8] is None else dev(torch, w[8])
    gm.set_wall_model(wtype, *w[:8], walave_u=walave)
    rng = np.random.default_rng(47)
    rnd = lambda a: rng.standard_normal(a.shape) * np.abs(a).mean()
    v = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    # the stage RHS (no boundary routine inside it)
    _, dR = oracle.rhs_jvp(om, prm, st, *v, wall=owm)
    wr = np.stack([rnd(st.rho) for _ in range(5)])
    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    g = gm.rhs_vjp(dv(st.rho), dv(st.q.T), dv(st.E), dv(st.mu_e.T), dv(st.mu_factor), dv(wr[0]), dv(wr[1:4]),
                   dv(wr[4]))
    lhs = float((wr * dR).sum())
    rhs = sum(float((gi.cpu().numpy() * vi).sum()) for gi, vi in zip(g, (v[0], v[1].T, v[2])))
    assert abs(lhs - rhs) <= 1e-11 * float(np.abs(wr * dR).sum()), (lhs, rhs)
    # one step
    y1, dy1 = oracle_step_jvp(oracle, om, prm, st, dt, v, bc_jvp=oracle_bc_jvp_map(oracle, bnd), wall=owm)
    s = S.Sod2dState.from_host(st, gm.nelem)
    s.dt.fill_(dt)
    stages = torch.zeros(15 * m.npoin, dtype=torch.float64, device="cuda")
    y0 = (s.rho.clone(), s.q.clone(), s.E.clone(), s.mu_e.clone())
    gm.rk_4_main_record(s, stages, update_dt=False)
    h = s.to_host()
    for got, ref in ((h["rho"], y1[0]), (h["q"], y1[1]), (h["E"], y1[2])):
        assert rel_l2(got, ref) < TOL64
    wb = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    terms = [wb[f] * dy1[f] for f in range(3)]
    lhs = sum(t.sum() for t in terms)
    scale = sum(np.abs(t).sum() for t in terms)
    for stg in (stages, None):
        out = gm.rk4_step_vjp(*y0, s.mu_factor, s.dt, *(dev(torch, a) for a in wb), stages=stg)
        gs = [host(o) for o in out]
        rhs = sum((gs[f] * v[f]).sum() for f in range(3))
        assert abs(lhs - rhs) <= 1e-11 * scale, (stg is None, lhs, rhs)
    gm.close()
