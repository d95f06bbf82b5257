"""Size-independent properties at the benchmark's full size (TGV on 64^3 periodic HEX64 meshes:
262,144 elements, 7,077,888 nodes), where the oracle would take minutes per step.  Discrete
conservation on the undistorted mesh (on a jittered one the pointwise metric breaks it at
truncation level): the split-form convection and the weak-form stress sum to zero over a
periodic mesh, so total momentum sum_a Ml_a q_a changes by rounding only over 10 steps; total
mass as well while mu_e = 0 (the first step from the initial state: the artificial mass
diffusion nu_e div grad rho, elem_diffu.f90:144,184, multiplies the divergence by a nodal
coefficient and is not conservative by construction, nor is the nodal-conductivity energy
flux); bounds 1e-12 (FP64) and 1e-9 (mixed) relative to sum_a Ml_a rho_a for mass and to
sum_a Ml_a |q_a|_1 (all three components) for each momentum component.  On the jittered
benchmark mesh: the mixed path against FP64 (stage residuals and the state after 10 steps,
1e-6 per field: the precision bound), and bitwise determinism of graph replays."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    prm = M.TGVParams()
    out = dict(torch=torch, S=S)
    for name, jit in (("affine", 0.0), ("jittered", 0.05)):
        m = M.periodic_box(64, jitter=jit, seed=1)
        st = M.taylor_green_state(m, prm, pert_amp=1e-3, seed=0)
        gm = S.Sod2dMesh(m, prm)
        ic = S.Sod2dState.from_host(st, gm.nelem)
        gm.adapt_dt(ic)
        s0 = S.Sod2dState.from_host(st, gm.nelem)
        s0.dt.copy_(ic.dt)
        gm.rk_4_main(s0, S.FP64, update_dt=True)  # a state with mu_e > 0
        Ml = 1.0 / gm.lumped_solver(torch.ones(m.npoin, dtype=torch.float64, device="cuda"))
        out[name] = dict(gm=gm, ic=ic, s0=s0, Ml=Ml)
    yield out
    for name in ("affine", "jittered"):
        out[name]["gm"].close()


def clone(env, mesh="jittered", which="s0"):
    from sod2d_refmap_b200.adjoint import _clone_state
    return _clone_state(env[mesh][which])


def totals(Ml, s, fields):
    cols = {"rho": s.rho, "q0": s.q[0], "q1": s.q[1], "q2": s.q[2]}
    return {f: (float((Ml * cols[f]).sum().item()), float((Ml * cols[f].abs()).sum().item())) for f in fields}


@pytest.mark.parametrize("prec,bound", [("FP64", 1e-12), ("MIXED", 1e-9)])
def test_conservation_full_size(env, prec, bound):
    S = env["S"]
    p = getattr(S, prec)
    A = env["affine"]
    # momentum over 10 steps with mu_e > 0
    s = clone(env, "affine")
    before = totals(A["Ml"], s, ("q0", "q1", "q2"))
    A["gm"].rk4_steps(s, 10, precision=p)
    after = totals(A["Ml"], s, ("q0", "q1", "q2"))
    scale = sum(before[f][1] for f in before)  # sum_a Ml_a |q_a|_1: the momentum's magnitude
    for f in before:
        (b, _), (a, _) = before[f], after[f]
        assert abs(a - b) <= bound * scale, (prec, f, a, b, scale)
    # mass over the first step from the initial state (mu_e = 0)
    s = clone(env, "affine", "ic")
    (b, scale) = totals(A["Ml"], s, ("rho",))["rho"]
    A["gm"].rk_4_main(s, p, update_dt=False)
    (a, _) = totals(A["Ml"], s, ("rho",))["rho"]
    assert abs(a - b) <= bound * scale, (prec, "rho", a, b, scale)


def test_mixed_vs_fp64_full_size(env):
    torch, S, gm = env["torch"], env["S"], env["jittered"]["gm"]
    s = clone(env)
    r64 = {k: v.clone() for k, v in gm.rhs(s, precision=S.FP64).items()}
    r32 = gm.rhs(s, precision=S.MIXED)
    for k in r64:
        err = float((r32[k] - r64[k]).norm() / r64[k].norm())
        assert err < 1e-6, (k, err)
    a, b = clone(env), clone(env)
    gm.rk4_steps(a, 10, precision=S.FP64)
    gm.rk4_steps(b, 10, precision=S.MIXED)
    for k in ("rho", "q", "E"):
        err = float((getattr(b, k) - getattr(a, k)).norm() / getattr(a, k).norm())
        assert err < 1e-6, (k, err)


def test_graph_replay_deterministic_full_size(env):
    torch, S, gm = env["torch"], env["S"], env["jittered"]["gm"]
    for p in (S.FP64, S.MIXED):
        a, b = clone(env), clone(env)
        gm.rk4_steps(a, 3, precision=p)
        gm.rk4_steps(b, 3, precision=p)
        torch.cuda.synchronize()
        for k in ("rho", "q", "E", "mu_e", "dt"):
            assert torch.equal(getattr(a, k), getattr(b, k)), (p, k)
