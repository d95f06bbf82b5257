"""Boundary conditions on the device (non-periodic path of rk_4_main, mod_bc_routines.f90)
against the oracle: the per-routine entry points on random states with every code, and
three RK4 steps on channel meshes.  FP64 bound 1e-12 relative per field (the rest of the
FP64 path's bound; the routines themselves agree to rounding); mixed vs FP64 1e-7 after 3
steps of the 3^3 channel (as the LES steps)."""
import numpy as np
import pytest

from _util import rel_l2
from test_oracle_bc import random_case

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


def test_bc_dirichlet_prim_parity(torch_mod, oracle):
    from sod2d_refmap_b200 import mesh as M, solver as S
    torch = torch_mod
    m, prm, st, codes, lnbn, nrm, ub, u_old = random_case(seed=11, n=3)
    bc = M.bc_params(prm)
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(codes, lnbn, nrm, ub, bc)
    ref = [np.array(a, order="F", copy=True) for a in (st.rho, st.q, u_old, st.pr, st.E)]
    oracle.bc_dirichlet_prim(oracle.Boundaries(codes, lnbn, nrm, ub, bc), *ref)
    t = [dev(torch, a) for a in (st.rho, st.q, u_old, st.pr, st.E)]
    gm.bc_dirichlet_prim(*t)
    torch.cuda.synchronize()
    for name, a, r in zip(("rho", "q", "u", "pr", "E"), t, ref):
        assert rel_l2(host(a), r) < 1e-14, name
    gm.close()


def test_bc_fix_parity(torch_mod, oracle):
    from sod2d_refmap_b200 import mesh as M, solver as S
    torch = torch_mod
    m, prm, st, codes, lnbn, nrm, ub, _ = random_case(seed=13, n=3)
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(codes, lnbn, nrm, ub, M.bc_params(prm))
    rng = np.random.default_rng(2)
    Rm, Re, R = (rng.standard_normal(m.npoin) for _ in range(3))
    Rmo = np.asfortranarray(rng.standard_normal((m.npoin, 3)))
    t = [dev(torch, a) for a in (Rm, Rmo, Re, R)]
    bnd = oracle.Boundaries(codes, lnbn, nrm, ub, M.bc_params(prm))
    oracle.bc_fix_residual(bnd, Rm, Rmo, Re)
    oracle.bc_fix_residual_entropy(bnd, R)
    gm.bc_fix_residual(t[0], t[1], t[2])
    gm.bc_fix_residual_entropy(t[3])
    for a, r in zip(t, (Rm, Rmo, Re, R)):
        assert np.array_equal(host(a), r)
    gm.close()


def channel(codes, seed=4, n=3):
    from sod2d_refmap_b200 import mesh as M
    m = M.channel_box(n, jitter=0.05, seed=seed, codes=codes)
    prm = M.TGVParams(Re=800.0)
    st = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=seed)
    rng = np.random.default_rng(seed)
    ub = np.asfortranarray(np.column_stack([np.full(m.npoin, 1.0), rng.uniform(-0.1, 0.1, (m.npoin, 2))]))
    return m, prm, st, ub


@pytest.mark.parametrize("codes", [(3, 6), (4, 1), (5, 7)])
def test_channel_steps_fp64_vs_oracle(torch_mod, oracle, codes):
    from sod2d_refmap_b200 import mesh as M, solver as S
    m, prm, st0, ub = channel(codes)
    bc = M.bc_params(prm)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    ref = st0.copy()
    oracle.rk4(om, prm, ref, dt, nsteps=3,
               bnd=oracle.Boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc))
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    s = S.Sod2dState.from_host(st0, gm.nelem)
    s.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    h = s.to_host()
    for k in FIELDS:
        err = rel_l2(h[k], getattr(ref, k))
        assert err < TOL64, f"{codes} {k}: rel L2 {err:.3e}"
    gm.close()


def test_channel_dt_graph_mixed(torch_mod, oracle):
    from sod2d_refmap_b200 import mesh as M, solver as S
    torch = torch_mod
    m, prm, st0, ub = channel((3, 6), seed=8)
    bc = M.bc_params(prm)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    ref = st0.copy()
    oracle.rk4(om, prm, ref, dt, nsteps=1,
               bnd=oracle.Boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc))
    dt_ref = oracle.adapt_dt(om, ref, prm)
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    a = S.Sod2dState.from_host(st0, gm.nelem); a.dt.fill_(dt)
    b = S.Sod2dState.from_host(st0, gm.nelem); b.dt.fill_(dt)
    c = S.Sod2dState.from_host(st0, gm.nelem); c.dt.fill_(dt)
    gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    assert abs(float(a.dt.item()) - dt_ref) <= 1e-13 * dt_ref
    for _ in range(2):
        gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    gm.rk4_steps(b, 3, precision=S.FP64)
    for _ in range(3):
        gm.rk_4_main(c, precision=S.MIXED, update_dt=True)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "u", "mu_e", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    for k in ("rho", "q", "E"):
        assert float((getattr(c, k) - getattr(a, k)).norm() / getattr(a, k).norm()) < 1e-7, k
    gm.close()


def test_boundaries_removed(torch_mod, oracle):
    """The recording step runs with a slip wall (code 6) and a buffer zone; removing the
    boundaries and the zone gives the periodic step."""
    from sod2d_refmap_b200 import _lib, mesh as M, solver as S
    torch = torch_mod
    m, prm, st0, ub = channel((3, 6), seed=9, n=2)
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub)
    s = S.Sod2dState.from_host(st0, gm.nelem)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    s.dt.fill_(dt)
    stages = torch.zeros(15 * m.npoin, dtype=torch.float64, device="cuda")
    y0 = (s.rho.clone(), s.q.clone(), s.E.clone(), s.mu_e.clone())
    L = 2.0 * np.pi
    gm.set_buffer(M.buffer_params(prm, east=(0.8 * L, 0.3 * L)), m.coord, ub)
    gm.rk_4_main_record(s, stages, update_dt=False)
    gm.set_buffer(None)
    fresh = S.Sod2dState.from_host(st0, gm.nelem)
    for f in S.Sod2dState.FIELDS:
        getattr(s, f).copy_(getattr(fresh, f))
    # without boundaries the step is the periodic-path step of the same mesh
    gm.set_boundaries(None, None, None)
    ref = st0.copy()
    oracle.rk4(om, prm, ref, dt, nsteps=1)
    gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    h = s.to_host()
    for k in ("rho", "q", "E", "mu_e"):
        assert rel_l2(h[k], getattr(ref, k)) < TOL64, k
    gm.close()


@pytest.mark.parametrize("codes", [(3, 4), (5, 3), (4, 2)])
def test_channel_step_vjp_walls(torch_mod, oracle, codes):
    """Step adjoint on wall channels (no-slip adiabatic / isothermal, outlet): the routine is
    affine there, so its adjoint is a constant mask after every stage VJP and on the seed.
    <w, J v> with J v from the oracle's dual-number stage JVPs through its own boundary routine
    equals <J^T w, v>, bound 1e-11 relative to sum |w_i (J v)_i|, with recorded and with
    recomputed stage states; the device step matches the oracle step (1e-12)."""
    from _util import oracle_bc_map, oracle_step_jvp
    from sod2d_refmap_b200 import mesh as M, solver as S
    torch = torch_mod
    m, prm, st0, ub = channel(codes, seed=21)
    bc = M.bc_params(prm)
    om = oracle.OracleMesh(m)
    bnd = oracle.Boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    dt = oracle.adapt_dt(om, st0, prm)
    st = st0.copy()
    oracle.rk4(om, prm, st, dt, nsteps=1, bnd=bnd)  # mu_e > 0, wall nodes at their wall values
    rng = np.random.default_rng(17)
    rnd = lambda a: rng.standard_normal(a.shape) * np.abs(a).mean()
    v = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    y1, dy1 = oracle_step_jvp(oracle, om, prm, st, dt, v, bc=oracle_bc_map(oracle, bnd))
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
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
    outs = []
    for stg in (stages, None):
        out = gm.rk4_step_vjp(*y0, s.mu_factor, s.dt, *bars, stages=stg)
        g = [host(o) for o in out]
        rhs = sum((g[f] * v[f]).sum() for f in range(3))
        assert abs(lhs - rhs) <= 1e-11 * scale, (stg is None, lhs, rhs)
        outs.append(out)
    for a, b in zip(*outs):
        assert float((a - b).norm() / b.norm()) < 1e-13
    # the seed's wall rows are masked: a cotangent only on the wall nodes' rho and q gives none
    nodes = np.flatnonzero(np.isin(m.extra["bou_codes_nodes"], codes[:1]))
    wr = np.zeros(m.npoin); wr[nodes] = 1.0
    wq = np.zeros((m.npoin, 3), order="F"); wq[nodes, :] = 1.0
    z = gm.rk4_step_vjp(*y0, s.mu_factor, s.dt, dev(torch, wr), dev(torch, wq), dev(torch, np.zeros(m.npoin)),
                        stages=stages)
    assert all(float(t.abs().max()) == 0.0 for t in z)
    gm.close()


def test_channel_rollout_gradient_fd(torch_mod, oracle):
    """Loss 1/2 sum |q_K|^2 after K = 4 steps of a no-slip channel (codes 3 and 5), checkpoints
    every 2, against central differences of the frozen-coefficient map (mu_e, dt frozen),
    h = 1e-4 and 1e-6, bound 1e-6 relative."""
    from sod2d_refmap_b200 import mesh as M, solver as S
    from sod2d_refmap_b200.adjoint import Sod2dRollout, replay, trajectory_coefficients, _clone_state
    torch = torch_mod
    m, prm, st0, ub = channel((3, 5), seed=23)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, M.bc_params(prm))
    s = S.Sod2dState.from_host(st0, gm.nelem)
    s.dt.fill_(dt)
    gm.rk_4_main(s, precision=S.FP64, update_dt=True)
    K = 4
    rho = s.rho.clone().requires_grad_(True)
    q = s.q.clone().requires_grad_(True)
    E = s.E.clone().requires_grad_(True)
    rK, qK, EK = Sod2dRollout.apply(gm, s, rho, q, E, K, 2)
    (0.5 * (qK * qK).sum()).backward()
    rng = np.random.default_rng(29)
    v = [torch.from_numpy(rng.standard_normal(t.shape)).cuda() * t.abs().mean() for t in (s.rho, s.q, s.E)]
    dL = float(sum((g * d).sum() for g, d in zip((rho.grad, q.grad, E.grad), v)).item())
    mus, dts = trajectory_coefficients(gm, s, K)

    def L_at(h):
        t = _clone_state(s)
        t.rho.add_(h * v[0]); t.q.add_(h * v[1]); t.E.add_(h * v[2])
        replay(gm, t, mus, dts)
        return 0.5 * float((t.q * t.q).sum().item())
    for h in (1e-4, 1e-6):
        fd = (L_at(h) - L_at(-h)) / (2 * h)
        assert abs(fd - dL) <= 1e-6 * abs(dL), (h, fd, dL)
    gm.close()


@pytest.mark.parametrize("codes", [(1, 3), (3, 1), (1, 1), (1, 6), (6, 3), (7, 1)])
def test_channel_step_vjp_far_field(torch_mod, oracle, codes):
    """Step adjoint through far-field nodes (the HLL state of the lnbn node) and slip walls (which
    read the velocity of the previous post-routine stage state, and for the update q/rho of the
    step's own input): <w, J v> with J v from the oracle's dual-number stage JVPs composed with
    its boundary routine in dual numbers (the read velocity's tangent carried along) equals
    <J^T w, v>, bound 1e-11 relative to sum |w_i (J v)_i|, recorded and recomputed stage states;
    without slip walls, the routine's own adjoint (sod_bc_dirichlet_prim_vjp) against the
    oracle's JVP of it (1e-12)."""
    from _util import oracle_bc_jvp_map, oracle_step_jvp
    from sod2d_refmap_b200 import mesh as M, solver as S
    torch = torch_mod
    m, prm, st0, ub = channel(codes, seed=31)
    bc = M.bc_params(prm)
    om = oracle.OracleMesh(m)
    bnd = oracle.Boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    dt = oracle.adapt_dt(om, st0, prm)
    st = st0.copy()
    oracle.rk4(om, prm, st, dt, nsteps=1, bnd=bnd)
    rng = np.random.default_rng(23)
    rnd = lambda a: rng.standard_normal(a.shape) * np.abs(a).mean()
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    v = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    w = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    if not {6, 7} & set(codes):
        # the routine alone
        _, Jv = oracle.bc_jvp(bnd, st.rho, st.q, st.E, *v)
        bars = [dev(torch, a) for a in w]
        gm.bc_dirichlet_prim_vjp(dev(torch, st.rho), dev(torch, st.q), dev(torch, st.E), *bars)
        g = [host(t) for t in bars]
        terms = [w[f] * Jv[f] for f in range(3)]
        lhs = sum(t.sum() for t in terms)
        rhs = sum((g[f] * v[f]).sum() for f in range(3))
        assert abs(lhs - rhs) <= 1e-12 * sum(np.abs(t).sum() for t in terms), (lhs, rhs)
    # one step
    y1, dy1 = oracle_step_jvp(oracle, om, prm, st, dt, v, bc_jvp=oracle_bc_jvp_map(oracle, bnd))
    s = S.Sod2dState.from_host(st, gm.nelem)
    s.dt.fill_(dt)
    stages = torch.zeros(15 * m.npoin, dtype=torch.float64, device="cuda")
    y0 = (s.rho.clone(), s.q.clone(), s.E.clone(), s.mu_e.clone())
    gm.rk_4_main_record(s, stages, update_dt=False)
    h = s.to_host()
    for got, ref in ((h["rho"], y1[0]), (h["q"], y1[1]), (h["E"], y1[2])):
        assert rel_l2(got, ref) < TOL64
    terms = [w[f] * dy1[f] for f in range(3)]
    lhs = sum(t.sum() for t in terms)
    scale = sum(np.abs(t).sum() for t in terms)
    outs = []
    for stg in (stages, None):
        out = gm.rk4_step_vjp(*y0, s.mu_factor, s.dt, *(dev(torch, a) for a in w), stages=stg)
        g = [host(o) for o in out]
        rhs = sum((g[f] * v[f]).sum() for f in range(3))
        assert abs(lhs - rhs) <= 1e-11 * scale, (stg is None, lhs, rhs)
        outs.append(out)
    for a, b in zip(*outs):
        assert float((a - b).norm() / b.norm()) < 1e-13
    gm.close()


@pytest.mark.parametrize("codes", [(1, 3), (6, 1)])
def test_far_field_rollout_fd_and_refusals(torch_mod, oracle, codes):
    """4-step rollouts with a far-field side (codes 1 and 3) and with a slip wall and a far-field
    side (6 and 1) against central differences of the frozen-coefficient map with u = q/rho in
    the perturbed initial state (h = 1e-5, 1e-6; 1e-6 relative); the standalone routine adjoint
    with slip walls is refused."""
    from sod2d_refmap_b200 import _lib, mesh as M, solver as S
    from sod2d_refmap_b200.adjoint import Sod2dRollout, replay, trajectory_coefficients, _clone_state
    torch = torch_mod
    m, prm, st0, ub = channel(codes, seed=33)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, M.bc_params(prm))
    s = S.Sod2dState.from_host(st0, gm.nelem)
    s.dt.fill_(dt)
    gm.rk_4_main(s, precision=S.FP64, update_dt=True)
    K = 4
    rho = s.rho.clone().requires_grad_(True)
    q = s.q.clone().requires_grad_(True)
    E = s.E.clone().requires_grad_(True)
    rK, qK, EK = Sod2dRollout.apply(gm, s, rho, q, E, K, 2)
    (0.5 * (qK * qK).sum()).backward()
    rng = np.random.default_rng(37)
    v = [torch.from_numpy(rng.standard_normal(t.shape)).cuda() * t.abs().mean() for t in (s.rho, s.q, s.E)]
    dL = float(sum((g * d).sum() for g, d in zip((rho.grad, q.grad, E.grad), v)).item())
    mus, dts = trajectory_coefficients(gm, s, K)

    def L_at(h):
        t = _clone_state(s)
        t.rho.add_(h * v[0]); t.q.add_(h * v[1]); t.E.add_(h * v[2])
        t.u.copy_(t.q / t.rho)
        replay(gm, t, mus, dts)
        return 0.5 * float((t.q * t.q).sum().item())
    for h in (1e-5, 1e-6):
        fd = (L_at(h) - L_at(-h)) / (2 * h)
        assert abs(fd - dL) <= 1e-6 * abs(dL), (h, fd, dL)
    # refusal: the standalone routine adjoint does not get the velocity slip walls read
    bars = (s.rho.clone(), s.q.clone(), s.E.clone())
    m6, prm6, _, ub6 = channel((1, 6), seed=33)
    gm6 = S.Sod2dMesh(m6, prm6)
    gm6.set_boundaries(m6.extra["bou_codes_nodes"], m6.extra["lnbn_nodes"], m6.extra["normals"], ub6)
    with pytest.raises(_lib.SodError, match="SOD_ERR_UNSUPPORTED"):
        gm6.bc_dirichlet_prim_vjp(s.rho, s.q, s.E, *bars)
    gm6.close()
    gm.close()


@pytest.mark.parametrize("codes", [(1, 3), (6, 1)])
def test_step_vjp_far_field_slip_with_buffer_zone(torch_mod, oracle, codes):
    """Far-field and slip boundaries together with a buffer zone reaching both walls: the step
    adjoint against the oracle's dual-number JVP of B(Z(.)) per stage (1e-11), recorded and
    recomputed stage states."""
    from _util import oracle_bc_jvp_map, oracle_step_jvp
    from sod2d_refmap_b200 import mesh as M, solver as S
    torch = torch_mod
    m, prm, st0, ub = channel(codes, seed=41)
    bc = M.bc_params(prm)
    L = 2.0 * np.pi
    lo, hi = m.coord.min(axis=0), m.coord.max(axis=0)
    bp = M.buffer_params(prm, u_inf=0.5, south=(0.3 * L, (0.3 * L - lo[1]) / 0.995),
                         north=(0.7 * L, (hi[1] - 0.7 * L) / 0.995))
    om = oracle.OracleMesh(m)
    bnd = oracle.Boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    buf = oracle.BufferZone(m.coord, ub, bp)
    dt = oracle.adapt_dt(om, st0, prm)
    st = st0.copy()
    oracle.rk4(om, prm, st, dt, nsteps=1, bnd=bnd, buf=buf)
    J = oracle_bc_jvp_map(oracle, bnd)

    def ZJ(y, v, u=None, du=None):
        def Z(r, q, E):
            r = np.array(r, copy=True); q = np.array(q, order="F", copy=True); E = np.array(E, copy=True)
            oracle.update_buffer(buf, r, q, E)
            return r, q, E
        zy = Z(*y)
        zyv = Z(*(y[f] + v[f] for f in range(3)))
        return J(zy, tuple(zyv[f] - zy[f] for f in range(3)), u, du)
    rng = np.random.default_rng(43)
    rnd = lambda a: rng.standard_normal(a.shape) * np.abs(a).mean()
    v = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    w = (rnd(st.rho), np.asfortranarray(rnd(st.q)), rnd(st.E))
    y1, dy1 = oracle_step_jvp(oracle, om, prm, st, dt, v, bc_jvp=ZJ)
    gm = S.Sod2dMesh(m, prm)
    gm.set_boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"], ub, bc)
    gm.set_buffer(bp, m.coord, ub)
    s = S.Sod2dState.from_host(st, gm.nelem)
    s.dt.fill_(dt)
    stages = torch.zeros(15 * m.npoin, dtype=torch.float64, device="cuda")
    y0 = (s.rho.clone(), s.q.clone(), s.E.clone(), s.mu_e.clone())
    gm.rk_4_main_record(s, stages, update_dt=False)
    h = s.to_host()
    for got, ref in ((h["rho"], y1[0]), (h["q"], y1[1]), (h["E"], y1[2])):
        assert rel_l2(got, ref) < TOL64
    terms = [w[f] * dy1[f] for f in range(3)]
    lhs = sum(t.sum() for t in terms)
    scale = sum(np.abs(t).sum() for t in terms)
    for stg in (stages, None):
        out = gm.rk4_step_vjp(*y0, s.mu_factor, s.dt, *(dev(torch, a) for a in w), stages=stg)
        g = [host(o) for o in out]
        rhs = sum((g[f] * v[f]).sum() for f in range(3))
        assert abs(lhs - rhs) <= 1e-11 * scale, (stg is None, lhs, rhs)
    gm.close()
