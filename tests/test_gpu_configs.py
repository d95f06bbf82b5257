"""Parity on the benchmark's named configurations, CUDA path (through the C ABI) against the
CPU oracle.

* c0: the 8x8x8 undistorted periodic TGV on [0, 2 pi]^3 (13,824 unique nodes), FP64: the full
  stage-1 residual of rk_4_main (time_integ.f90:266-393) at the initial state and at a state with
  mu_e > 0, and the post-step state of one and of two steps with dt from adapt_dt_cfl, all
  <= 1e-12 relative L2 per field.  The mixed path is held to 2e-5 per field here: on this
  coarse mesh (an element spans 0.79 rad of the vortex) the second-order remainder that the
  mixed kernel rounds to FP32 is about 60 times larger relative to the fields than on the 64^3
  mesh, and the mass residual is a small difference of large terms; its 1e-6 bound is checked
  on c1, the configuration the mixed-precision figure is quoted on.
* c1: the 64^3 jittered benchmark mesh (7,077,888 nodes).  The oracle evaluates the stage
  residual on a slab of the first four element layers in z (16,384 elements); a node whose
  elements all lie in the slab (lattice planes k = 1..11) has its complete residual there.  At
  those 405,504 nodes the GPU residual of the whole mesh is compared, at the initial state and
  after one GPU step (the slab's mu_e taken from the GPU).  FP64: <= 1e-12 against the oracle
  wherever the FP64 rounding floor of the field allows it.  The momentum residual is not such
  a field at this resolution: grad p is formed from p ~ p0 = 1/(gamma M^2) = 71 around
  variations of 0.06, so FP64 rounding alone moves it by ~6e-12 relative (the oracle's own
  FP64 evaluation against the same formulas in x87 extended precision, rhs_stage_ld; the floor
  grows linearly with the elements per side: 7e-13 at 8^3, 1.4e-12 at 16^3).  Each field is
  therefore measured against the extended-precision value, and the GPU's FP64 error must be
  <= max(1e-12, 2 x the oracle's own FP64 error).  Mixed: <= 1e-6 against the same value.
* c2: the gradient of L = 1/2 sum_a |q_a|^2 after 50 RK4 steps (checkpoint every 10) on the
  32^3 jittered mesh, along a seeded Gaussian direction, against the oracle's forward-mode
  derivative through the same 50 FP64 steps (dual numbers, mu_e and dt frozen at the values of
  the forward run): <= 1e-10 relative.
"""
import numpy as np
import pytest

from _util import oracle_step_jvp, rel_l2, slab_oracle, slab_state, t2n

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_MIXED = 1e-6
TOL_MIXED_C0 = 2e-5


def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build
    build.build()
    return torch


# ---------------------------------------------------------------------------------------------
# c0: 8^3 undistorted TGV
# ---------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c0(oracle):
    torch = _cuda()
    from sod2d_refmap_b200 import mesh as M, solver as S
    m = M.periodic_box(8, jitter=0.0)
    prm = M.TGVParams()
    st0 = M.taylor_green_state(m, prm, pert_amp=1e-3, seed=0)
    om = oracle.OracleMesh(m)
    gm = S.Sod2dMesh(m, prm)
    dt0 = oracle.adapt_dt(om, st0, prm)
    st1 = st0.copy()
    oracle.rk4(om, prm, st1, dt0, nsteps=1)
    yield dict(torch=torch, M=M, S=S, m=m, prm=prm, om=om, gm=gm, st0=st0, st1=st1, dt0=dt0)
    gm.close()


def test_c0_mesh_size(c0):
    assert c0["m"].nelem == 512 and c0["m"].npoin == 13824


@pytest.mark.parametrize("which", ["st0", "st1"])
def test_c0_stage_rhs(c0, oracle, which):
    """Full stage-1 residual (R/Ml for mass, momentum, energy; entropy residual) at the initial
    state (mu_e = 0) and after one step (mu_e > 0): FP64 <= 1e-12, mixed <= 2e-5."""
    S, gm, om, prm = c0["S"], c0["gm"], c0["om"], c0["prm"]
    st = c0[which]
    ref = oracle.rk4(om, prm, st.copy(), c0["dt0"], nsteps=1, capture_stage=1)
    s = S.Sod2dState.from_host(st, gm.nelem)
    out = {k: t2n(v) for k, v in gm.rhs(s, precision=S.FP64).items()}
    mix = {k: t2n(v) for k, v in gm.rhs(s, precision=S.MIXED).items()}
    e64 = {k: rel_l2(out[k], ref[k]) for k in ("Rmass", "Rmom", "Rener", "Reta")}
    e32 = {k: rel_l2(mix[k], ref[k]) for k in e64}
    print(f"c0 {which} fp64 {e64} mixed {e32}")
    for k in e64:
        assert e64[k] < TOL64, (k, e64[k])
        assert e32[k] < TOL_MIXED_C0, (k, e32[k])


@pytest.mark.parametrize("nsteps", [1, 2])
def test_c0_post_step_state(c0, oracle, nsteps):
    """rk_4_main steps with dt from the CFL condition after each step (CFDSolverBase.f90:1592):
    every output field and the next dt <= 1e-12."""
    S, gm, om, prm = c0["S"], c0["gm"], c0["om"], c0["prm"]
    ref = c0["st0"].copy()
    dt = c0["dt0"]
    for _ in range(nsteps):
        oracle.rk4(om, prm, ref, dt, nsteps=1)
        dt = oracle.adapt_dt(om, ref, prm)
    s = S.Sod2dState.from_host(c0["st0"], gm.nelem)
    s.dt.fill_(c0["dt0"])
    for _ in range(nsteps):
        gm.rk_4_main(s, precision=S.FP64, update_dt=True)
    h = s.to_host()
    for k in ("rho", "q", "E", "u", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid", "mu_e"):
        err = rel_l2(h[k], getattr(ref, k))
        assert err < TOL64, f"{k}: rel L2 {err:.3e}"
    assert abs(float(s.dt.item()) - dt) <= 1e-13 * dt


def test_c0_mixed_post_step_state(c0, oracle):
    """One mixed-precision step against the FP64 oracle: <= 1e-6 on every conserved field."""
    S, gm, om, prm = c0["S"], c0["gm"], c0["om"], c0["prm"]
    ref = c0["st0"].copy()
    oracle.rk4(om, prm, ref, c0["dt0"], nsteps=1)
    s = S.Sod2dState.from_host(c0["st0"], gm.nelem)
    s.dt.fill_(c0["dt0"])
    gm.rk_4_main(s, precision=S.MIXED, update_dt=False)
    h = s.to_host()
    for k in ("rho", "q", "E"):
        err = rel_l2(h[k], getattr(ref, k))
        print(f"c0 mixed step {k}: {err:.2e}")
        assert err < TOL_MIXED, (k, err)


# ---------------------------------------------------------------------------------------------
# c1: 64^3 jittered benchmark mesh, compared on the interior of a 4-layer slab
# ---------------------------------------------------------------------------------------------
SLAB_LAYERS = 4


@pytest.fixture(scope="module")
def c1(oracle):
    torch = _cuda()
    from sod2d_refmap_b200 import mesh as M, solver as S
    m = M.periodic_box(64, jitter=0.05, seed=1)
    prm = M.TGVParams()
    st0 = M.taylor_green_state(m, prm, pert_amp=1e-3, seed=0)
    gm = S.Sod2dMesh(m, prm)
    om, nodes, E, interior = slab_oracle(oracle, M, m, SLAB_LAYERS)
    yield dict(torch=torch, M=M, S=S, m=m, prm=prm, gm=gm, st0=st0, om=om, nodes=nodes, E=E, interior=interior)
    gm.close()


def test_c1_slab_interior(c1):
    assert c1["m"].npoin == 7077888 and c1["E"] == 16384
    assert len(c1["interior"]) == 11 * 192 * 192


@pytest.mark.parametrize("which", ["initial", "after_step"])
def test_c1_slab_stage_rhs(c1, oracle, which):
    """Stage residual of the whole 64^3 mesh on the GPU vs the oracle's at the slab-interior
    nodes: FP64 <= 1e-12, mixed <= 1e-6 per field (Rmass, Rmom x3, Rener)."""
    S, gm, prm, M = c1["S"], c1["gm"], c1["prm"], c1["M"]
    s = S.Sod2dState.from_host(c1["st0"], gm.nelem)
    host = c1["st0"]
    mu_e = None
    if which == "after_step":
        gm.adapt_dt(s)
        gm.rk_4_main(s, precision=S.FP64, update_dt=True)
        h = s.to_host()
        host = c1["st0"].copy()
        for k in ("rho", "q", "E", "u", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid"):
            setattr(host, k, h[k])
        mu_e = h["mu_e"]
        assert float(np.abs(mu_e).max()) > 0.0
    nodes, E, idx = c1["nodes"], c1["E"], c1["interior"]
    ss = slab_state(host, nodes, E, mu_e)
    ref = oracle.rhs_stage(c1["om"], prm, ss)            # (5, npoin_slab): mass, mom x3, energy
    ext = oracle.rhs_stage_ld(c1["om"], prm, ss)         # the same formulas in extended precision
    g = nodes[idx]
    floor = [rel_l2(ref[f, idx], ext[f, idx]) for f in range(5)]
    for prec in (S.FP64, S.MIXED):
        out = gm.rhs(s, precision=prec)
        got = np.stack([t2n(out["Rmass"])[g], *(t2n(out["Rmom"])[g, c] for c in range(3)), t2n(out["Rener"])[g]])
        for f in range(5):
            e_ext = rel_l2(got[f], ext[f, idx])
            e_ora = rel_l2(got[f], ref[f, idx])
            print(f"c1 {which} prec={prec} field {f}: vs extended {e_ext:.2e}, vs oracle {e_ora:.2e}, "
                  f"oracle's own FP64 error {floor[f]:.2e}")
            if prec == S.FP64:
                bound = max(TOL64, 2.0 * floor[f])
                assert e_ext <= bound and e_ora <= bound, (which, f, e_ext, e_ora, floor[f])
            else:
                assert e_ext < TOL_MIXED, (which, f, e_ext)


# ---------------------------------------------------------------------------------------------
# c2: gradient of 50 RK4 steps against the oracle's forward-mode derivative
# ---------------------------------------------------------------------------------------------
def test_c2_gradient_vs_oracle_forward_mode(oracle):
    """dL/dy0 . v by the checkpointed adjoint (Sod2dRollout, 50 steps, checkpoint every 10, FP64
    trajectory) against sum_a q_a . dq_a from the oracle's dual-number stage JVPs composed over
    the same 50 steps (rk_4_main's stage sequence, time_integ.f90:288-426) with mu_e_n and dt_n
    frozen at the forward run's values: <= 1e-10 relative."""
    torch = _cuda()
    from sod2d_refmap_b200 import mesh as M, solver as S
    from sod2d_refmap_b200.adjoint import Sod2dRollout, trajectory_coefficients
    K, every = 50, 10
    m = M.periodic_box(32, jitter=0.05, seed=2)
    prm = M.TGVParams()
    st0 = M.taylor_green_state(m, prm, pert_amp=1e-3, seed=0)
    gm = S.Sod2dMesh(m, prm)
    s = S.Sod2dState.from_host(st0, gm.nelem)
    gm.adapt_dt(s)
    rng = np.random.default_rng(3)
    v = (rng.standard_normal(m.npoin) * np.abs(st0.rho).mean(),
         np.asfortranarray(rng.standard_normal((m.npoin, 3)) * np.abs(st0.q).mean()),
         rng.standard_normal(m.npoin) * np.abs(st0.E).mean())
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    rho = s.rho.clone().requires_grad_(True)
    q = s.q.clone().requires_grad_(True)
    E = s.E.clone().requires_grad_(True)
    _, qK, _ = Sod2dRollout.apply(gm, s, rho, q, E, K, every, True, S.FP64)
    loss = 0.5 * (qK * qK).sum()
    loss.backward()
    dL_gpu = float((rho.grad * dev(v[0])).sum() + (q.grad * dev(v[1].T)).sum() + (E.grad * dev(v[2])).sum())
    mus, dts = trajectory_coefficients(gm, s, K, S.FP64)
    gm.close()
    # the oracle: the frozen-coefficient map in dual numbers
    om = oracle.OracleMesh(m)
    st = st0.copy()
    y = (st.rho.copy(), np.asfortranarray(st.q.copy()), st.E.copy())
    w = v
    for n in range(K):
        st.mu_e = np.asfortranarray(mus[n].cpu().numpy().T)
        st.rho, st.q, st.E = y[0], y[1], y[2]
        acc_y, acc_v = oracle_step_jvp(oracle, om, prm, st, float(dts[n].item()), w)
        y = (np.ascontiguousarray(acc_y[0]), np.asfortranarray(acc_y[1]), np.ascontiguousarray(acc_y[2]))
        w = (np.ascontiguousarray(acc_v[0]), np.asfortranarray(acc_v[1]), np.ascontiguousarray(acc_v[2]))
    dL_ref = float((y[1] * w[1]).sum())
    L_ref = 0.5 * float((y[1] * y[1]).sum())
    print(f"c2: L gpu {float(loss.item()):.15e} oracle {L_ref:.15e}; dL gpu {dL_gpu:.15e} oracle {dL_ref:.15e}")
    assert abs(float(loss.item()) - L_ref) <= 1e-12 * abs(L_ref)
    assert abs(dL_gpu - dL_ref) <= 1e-10 * abs(dL_ref), (dL_gpu, dL_ref)
