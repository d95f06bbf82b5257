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


def test_les_step_adjoint_rejected(env):
    """The step adjoint does not differentiate the SGS viscosity: it refuses LES steps."""
    from sod2d_refmap_b200 import _lib
    S, gm, torch = env["S"], env["gm"], env["torch"]
    s = S.Sod2dState.from_host(env["st0"], gm.nelem)
    s.dt.fill_(env["dt"])
    stages = torch.zeros(15 * env["m"].npoin, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.SodError, match="SOD_ERR_UNSUPPORTED"):
        gm.rk_4_main_record(s, stages, update_dt=False)
    with pytest.raises(_lib.SodError, match="SOD_ERR_UNSUPPORTED"):
        gm.rk4_step_vjp(s.rho, s.q, s.E, s.mu_e, s.mu_factor, s.dt, s.rho.clone(), s.q.clone(), s.E.clone(),
                        stages=stages)
