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


def test_boundaries_removed_and_adjoint_rejected(torch_mod, oracle):
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
    with pytest.raises(_lib.SodError, match="SOD_ERR_UNSUPPORTED"):
        gm.rk_4_main_record(s, stages, update_dt=False)
    # without boundaries the step is the periodic-path step of the same mesh
    gm.set_boundaries(None, None, None)
    ref = st0.copy()
    oracle.rk4(om, prm, ref, dt, nsteps=1)
    gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    h = s.to_host()
    for k in ("rho", "q", "E", "mu_e"):
        assert rel_l2(h[k], getattr(ref, k)) < TOL64, k
    gm.close()
