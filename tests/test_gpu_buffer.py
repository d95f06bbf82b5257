"""Buffer zone (flag_buffer_on: updateBuffer, time_integ.f90:510-589, on every stage state and on
the updated state) on the device against the oracle: the routine as an entry point (1e-14),
three RK4 steps on a periodic box and on a wall channel with boundaries (FP64 1e-12 per field,
mixed vs FP64 1e-7, graph == eager bitwise), and the step adjoint through the zone (dot products
against the oracle's dual-number stage JVPs composed through its own routines, 1e-11)."""
import numpy as np
import pytest

from _util import rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
FIELDS = ("rho", "q", "E", "u", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid", "mu_e")


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


def zones(M, m, prm, channel=False):
    """East and top zones (and, on the channel, a north zone reaching the upper wall) whose far
    ends lie just beyond the outermost nodes."""
    L = 2.0 * np.pi
    lo, hi = m.coord.min(axis=0), m.coord.max(axis=0)
    z = dict(east=(0.6 * L, (hi[0] - 0.6 * L) / 0.995), top=(0.7 * L, (hi[2] - 0.7 * L) / 0.995))
    if channel:
        z["north"] = (0.75 * L, (hi[1] - 0.75 * L) / 0.995)
    return M.buffer_params(prm, u_inf=0.5, **z)


def case(seed=4, channel_codes=None, n=3):
    from sod2d_refmap_b200 import mesh as M
    if channel_codes is None:
        m = M.periodic_box(n, jitter=0.05, seed=seed)
    else:
        m = M.channel_box(n, jitter=0.05, seed=seed, codes=channel_codes)
    prm = M.TGVParams(Re=800.0)
    st = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=seed)
    rng = np.random.default_rng(seed)
    ub = np.asfortranarray(np.column_stack([np.full(m.npoin, 0.5), rng.uniform(-0.05, 0.05, (m.npoin, 2))]))
    return M, m, prm, st, ub, zones(M, m, prm, channel_codes is not None)


def setup(M, S, oracle, m, prm, ub, bp, with_bc):
    gm = S.Sod2dMesh(m, prm)
    gm.set_buffer(bp, m.coord, ub)
    buf = oracle.BufferZone(m.coord, ub, bp)
    bnd = None
    if with_bc:
        bc = M.bc_params(prm)
        gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
        bnd = oracle.Boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    return gm, buf, bnd


def test_update_buffer_entry(torch_mod, oracle):
    from sod2d_refmap_b200 import solver as S
    torch = torch_mod
    M, m, prm, st, ub, bp = case(seed=5)
    gm, buf, _ = setup(M, S, oracle, m, prm, ub, bp, False)
    ref = [np.array(a, order="F", copy=True) for a in (st.rho, st.q, st.E)]
    oracle.update_buffer(buf, *ref)
    t = [dev(torch, a) for a in (st.rho, st.q, st.E)]
    gm.update_buffer(*t)
    torch.cuda.synchronize()
    assert rel_l2(host(t[0]), st.rho) > 1e-6  # the zone changed the state
    for name, a, r in zip(("rho", "q", "E"), t, ref):
        assert rel_l2(host(a), r) < 1e-14, name
    gm.close()


@pytest.mark.parametrize("codes", [None, (3, 4)])
def test_steps_fp64_vs_oracle(torch_mod, oracle, codes):
    from sod2d_refmap_b200 import solver as S
    M, m, prm, st0, ub, bp = case(seed=6, channel_codes=codes)
    gm, buf, bnd = setup(M, S, oracle, m, prm, ub, bp, codes is not None)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    ref = st0.copy()
    oracle.rk4(om, prm, ref, dt, nsteps=3, bnd=bnd, buf=buf)
    plain = st0.copy()
    oracle.rk4(om, prm, plain, dt, nsteps=3, bnd=bnd)
    assert rel_l2(plain.rho, ref.rho) > 1e-8  # the zone acts
    s = S.Sod2dState.from_host(st0, gm.nelem)
    s.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    h = s.to_host()
    for k in FIELDS:
        err = rel_l2(h[k], getattr(ref, k))
        assert err < TOL64, f"{codes} {k}: rel L2 {err:.3e}"
    gm.close()


def test_graph_mixed_and_removal(torch_mod, oracle):
    from sod2d_refmap_b200 import solver as S
    torch = torch_mod
    M, m, prm, st0, ub, bp = case(seed=7, channel_codes=(5, 3))
    gm, buf, bnd = setup(M, S, oracle, m, prm, ub, bp, True)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    a = S.Sod2dState.from_host(st0, gm.nelem); a.dt.fill_(dt)
    b = S.Sod2dState.from_host(st0, gm.nelem); b.dt.fill_(dt)
    c = S.Sod2dState.from_host(st0, gm.nelem); c.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    gm.rk4_steps(b, 3, precision=S.FP64)
    for _ in range(3):
        gm.rk_4_main(c, precision=S.MIXED, update_dt=True)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "u", "mu_e", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    for k in ("rho", "q", "E"):
        assert float((getattr(c, k) - getattr(a, k)).norm() / getattr(a, k).norm()) < 1e-7, k
    # without the zone the step is the boundary-only step
    gm.set_buffer(None)
    ref = st0.copy()
    oracle.rk4(om, prm, ref, dt, nsteps=1, bnd=bnd)
    d = S.Sod2dState.from_host(st0, gm.nelem); d.dt.fill_(dt)
    gm.rk_4_main(d, precision=S.FP64, update_dt=False)
    h = d.to_host()
    for k in ("rho", "q", "E", "mu_e"):
        assert rel_l2(h[k], getattr(ref, k)) < TOL64, k
    gm.close()


@pytest.mark.parametrize("codes", [None, (3, 4)])
def test_step_vjp_through_buffer(torch_mod, oracle, codes):
    """<w, J v> == <J^T w, v> for one step with the zone (and wall boundaries), J v from the
    oracle's dual-number stage JVPs composed through its own updateBuffer and boundary routine
    (B(Z(y + v)) - B(Z(y)), exact up to rounding for these affine maps); bound 1e-11 relative
    to sum |w_i (J v)_i|; recorded and recomputed stage states."""
    from _util import oracle_bc_map, oracle_step_jvp
    from sod2d_refmap_b200 import solver as S
    torch = torch_mod
    M, m, prm, st0, ub, bp = case(seed=8, channel_codes=codes)
    gm, buf, bnd = setup(M, S, oracle, m, prm, ub, bp, codes is not None)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    st = st0.copy()
    oracle.rk4(om, prm, st, dt, nsteps=1, bnd=bnd, buf=buf)  # mu_e > 0
    B = oracle_bc_map(oracle, bnd) if bnd is not None else (lambda r, q, E: (r, q, E))

    def ZB(rho, q, E):
        r = np.array(rho, copy=True); qq = np.array(q, order="F", copy=True); e = np.array(E, copy=True)
        oracle.update_buffer(buf, r, qq, e)
        return B(r, qq, e)
    rng = np.random.default_rng(19)
    rnd = lambda a: rng.standard_normal(a.shape) * np.abs(a).mean()
    v = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    y1, dy1 = oracle_step_jvp(oracle, om, prm, st, dt, v, bc=ZB)
    s = S.Sod2dState.from_host(st, gm.nelem)
    s.dt.fill_(dt)
    stages = torch.zeros(15 * m.npoin, dtype=torch.float64, device="cuda")
    y0 = (s.rho.clone(), s.q.clone(), s.E.clone(), s.mu_e.clone())
    gm.rk_4_main_record(s, stages, update_dt=False)
    h = s.to_host()
    for got, ref in ((h["rho"], y1[0]), (h["q"], y1[1]), (h["E"], y1[2])):
        assert rel_l2(got, ref) < TOL64
    wb = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    bars = (dev(torch, wb[0]), dev(torch, wb[1]), dev(torch, wb[2]))
    terms = [wb[f] * dy1[f] for f in range(3)]
    lhs = sum(t.sum() for t in terms)
    scale = sum(np.abs(t).sum() for t in terms)
    for stg in (stages, None):
        out = gm.rk4_step_vjp(*y0, s.mu_factor, s.dt, *bars, stages=stg)
        g = [host(o) for o in out]
        rhs = sum((g[f] * v[f]).sum() for f in range(3))
        assert abs(lhs - rhs) <= 1e-11 * scale, (stg is None, lhs, rhs)
    gm.close()
