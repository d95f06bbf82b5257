"""Hand-written adjoint (sod_rhs_vjp, sod_rk4_step_vjp, Sod2dRollout) against the oracle.

The oracle differentiates the same FP64 stage RHS in forward mode with dual numbers
(oracle_rhs_jvp), so <w, J v> from the oracle against <J^T w, v> from the CUDA adjoint is a
dot-product test whose only error is rounding: bound 1e-11 relative to sum |w_i (J v)_i|.
Entry-wise gradient checks use the oracle JVP along unit vectors (bound 1e-10 of max |g|).
The K-step adjoint is also checked against central finite differences of the frozen-coefficient
forward map (h = 1e-4 and 1e-6, bound 1e-6 relative).
"""
import numpy as np
import pytest

from _util import t2n

pytestmark = pytest.mark.gpu

DOT_TOL = 1e-11
FD_TOL = 1e-6


@pytest.fixture(scope="module")
def env(oracle):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    m = M.periodic_box(3, jitter=0.05, seed=7)
    prm = M.TGVParams()
    om = oracle.OracleMesh(m)
    gm = S.Sod2dMesh(m, prm)
    st0 = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=3)
    dt = oracle.adapt_dt(om, st0, prm)
    st1 = st0.copy()
    oracle.rk4(om, prm, st1, dt, nsteps=1)  # mu_e > 0 from the entropy residual
    # a viscous state with a large entropy viscosity so that every diffusion term matters
    st2 = M.taylor_green_state(m, prm, pert_amp=5e-2, seed=4, re=20.0)
    rng = np.random.default_rng(11)
    st2.mu_e = np.asfortranarray(rng.uniform(0.0, 0.05, size=st2.mu_e.shape))
    return dict(M=M, S=S, m=m, prm=prm, om=om, gm=gm, st={"st1": st1, "st2": st2}, dt=dt, torch=torch)


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _with(st, rho, q, E):
    s = st.copy()
    s.rho = np.ascontiguousarray(rho)
    s.q = np.asfortranarray(q)
    s.E = np.ascontiguousarray(E)
    return s


def _rand_dir(rng, st, scale=1.0):
    """A direction with each field scaled like the field itself."""
    drho = rng.standard_normal(st.rho.shape) * np.abs(st.rho).mean() * scale
    dq = rng.standard_normal(st.q.shape) * np.abs(st.q).mean() * scale
    dE = rng.standard_normal(st.E.shape) * np.abs(st.E).mean() * scale
    return drho, np.asfortranarray(dq), dE


def _gpu_vjp(env, st, w):
    """w: (5, N) seeds in (mass, mom x3, energy) order -> (g_rho, g_q (N,3), g_E) on host."""
    torch, gm = env["torch"], env["gm"]
    g = gm.rhs_vjp(_dev(torch, st.rho), _dev(torch, st.q.T), _dev(torch, st.E), _dev(torch, st.mu_e.T),
                   _dev(torch, st.mu_factor), _dev(torch, w[0]), _dev(torch, w[1:4]), _dev(torch, w[4]))
    torch.cuda.synchronize()
    return t2n(g[0]), t2n(g[1]), t2n(g[2])


@pytest.mark.parametrize("which", ["st1", "st2"])
@pytest.mark.parametrize("field", [None, 0, 1, 2, 3, 4])
def test_rhs_vjp_dot_product(env, oracle, which, field):
    """<w, J v> (oracle dual numbers) == <J^T w, v> (CUDA adjoint); field seeds one output only."""
    st = env["st"][which]
    rng = np.random.default_rng(100 + (field if field is not None else 9))
    drho, dq, dE = _rand_dir(rng, st)
    _, dR = oracle.rhs_jvp(env["om"], env["prm"], st, drho, dq, dE)
    w = rng.standard_normal(dR.shape)
    if field is not None:
        keep = np.zeros(5, bool); keep[field] = True
        w[~keep] = 0.0
    g_rho, g_q, g_E = _gpu_vjp(env, st, w)
    lhs_terms = w * dR
    lhs = lhs_terms.sum()
    rhs = (g_rho * drho).sum() + (g_q * dq).sum() + (g_E * dE).sum()
    scale = np.abs(lhs_terms).sum()
    assert abs(lhs - rhs) <= DOT_TOL * scale, f"<w,Jv>={lhs:.15e} <JTw,v>={rhs:.15e} scale={scale:.3e}"


@pytest.mark.parametrize("which", ["st1", "st2"])
def test_rhs_vjp_entries(env, oracle, which):
    """Gradient entries d<w,R>/dU_i against the oracle JVP along unit vectors."""
    st = env["st"][which]
    rng = np.random.default_rng(5)
    N = len(st.rho)
    w = rng.standard_normal((5, N))
    g_rho, g_q, g_E = _gpu_vjp(env, st, w)
    gmax = max(np.abs(g_rho).max(), np.abs(g_q).max(), np.abs(g_E).max())
    for trial in range(12):
        f = trial % 5
        i = int(rng.integers(N))
        drho = np.zeros(N); dq = np.zeros((N, 3), order="F"); dE = np.zeros(N)
        if f == 0:
            drho[i] = 1.0; got = g_rho[i]
        elif f == 4:
            dE[i] = 1.0; got = g_E[i]
        else:
            dq[i, f - 1] = 1.0; got = g_q[i, f - 1]
        _, dR = oracle.rhs_jvp(env["om"], env["prm"], st, drho, dq, dE)
        ref = (w * dR).sum()
        assert abs(got - ref) <= 1e-10 * gmax, f"field {f} node {i}: {got:.15e} vs {ref:.15e}"


def _oracle_step_jvp(oracle, env, st, dt, v):
    """One rk_4_main step (time_integ.f90:288-426) and its JVP by composing oracle_rhs_jvp."""
    om, prm = env["om"], env["prm"]
    y0 = (st.rho, st.q, st.E)
    acc_y = [a.copy() for a in y0]
    acc_v = [a.copy() for a in v]
    ys, vs = y0, v
    a_next = [0.5, 0.5, 1.0, None]
    b = [1 / 6, 1 / 3, 1 / 3, 1 / 6]
    for s in range(4):
        R, dR = oracle.rhs_jvp(om, prm, _with(st, *ys), vs[0], vs[1], vs[2])
        Rc = (R[0], np.asfortranarray(R[1:4].T), R[4])
        dRc = (dR[0], np.asfortranarray(dR[1:4].T), dR[4])
        for f in range(3):
            acc_y[f] = acc_y[f] - dt * b[s] * Rc[f]
            acc_v[f] = acc_v[f] - dt * b[s] * dRc[f]
        if a_next[s] is not None:
            ys = tuple(y0[f] - dt * a_next[s] * Rc[f] for f in range(3))
            vs = tuple(v[f] - dt * a_next[s] * dRc[f] for f in range(3))
    return acc_y, acc_v


@pytest.mark.parametrize("which", ["st1", "st2"])
def test_rk4_step_vjp_dot_product(env, oracle, which):
    torch, gm, S = env["torch"], env["gm"], env["S"]
    st = env["st"][which]
    dt = env["dt"] * (0.2 if which == "st2" else 1.0)
    rng = np.random.default_rng(21)
    v = _rand_dir(rng, st)
    y1, dy1 = _oracle_step_jvp(oracle, env, st, dt, v)
    # the composed oracle step is the solver's step: compare the state with the CUDA step
    s = S.Sod2dState.from_host(st, gm.nelem)
    s.dt.fill_(dt)
    gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    h = s.to_host()
    for got, ref in ((h["rho"], y1[0]), (h["q"], y1[1]), (h["E"], y1[2])):
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
    wb = _rand_dir(rng, st)
    dtd = torch.full((1,), dt, dtype=torch.float64, device="cuda")
    out = gm.rk4_step_vjp(_dev(torch, st.rho), _dev(torch, st.q.T), _dev(torch, st.E), _dev(torch, st.mu_e.T),
                          _dev(torch, st.mu_factor), dtd, _dev(torch, wb[0]), _dev(torch, wb[1].T), _dev(torch, wb[2]))
    torch.cuda.synchronize()
    g = (t2n(out[0]), t2n(out[1]), t2n(out[2]))
    terms = [wb[f] * dy1[f] for f in range(3)]
    lhs = sum(t.sum() for t in terms)
    rhs = sum((g[f] * v[f]).sum() for f in range(3))
    scale = sum(np.abs(t).sum() for t in terms)
    assert abs(lhs - rhs) <= DOT_TOL * scale, f"{lhs:.15e} vs {rhs:.15e}"


def test_rk4_step_vjp_aliasing(env):
    """out may alias bar: the in-place result equals the out-of-place one bit for bit."""
    torch, gm = env["torch"], env["gm"]
    st = env["st"]["st1"]
    rng = np.random.default_rng(3)
    wb = _rand_dir(rng, st)
    dtd = torch.full((1,), env["dt"], dtype=torch.float64, device="cuda")
    args = (_dev(torch, st.rho), _dev(torch, st.q.T), _dev(torch, st.E), _dev(torch, st.mu_e.T),
            _dev(torch, st.mu_factor), dtd)
    bars = [_dev(torch, wb[0]), _dev(torch, wb[1].T), _dev(torch, wb[2])]
    ref = gm.rk4_step_vjp(*args, *bars)
    gm.rk4_step_vjp(*args, *bars, out=tuple(bars))
    torch.cuda.synchronize()
    for a, b in zip(ref, bars):
        assert torch.equal(a, b)


def _rollout_env(env, nsteps):
    torch, S, gm = env["torch"], env["S"], env["gm"]
    st = env["st"]["st1"]
    s = S.Sod2dState.from_host(st, gm.nelem)
    s.dt.fill_(env["dt"])
    return s


def test_rollout_gradient_dot_product_and_fd(env, oracle):
    """Loss 1/2 sum |q_K|^2 after K = 7 steps (checkpoints every 3: segments 3,3,1).
    Directional derivative from the adjoint against (a) the oracle forward-mode derivative of
    the same frozen-coefficient map, (b) central differences with h = 1e-4 and 1e-6."""
    from sod2d_refmap_b200.adjoint import Sod2dRollout, replay, trajectory_coefficients, _clone_state
    torch, gm, S = env["torch"], env["gm"], env["S"]
    K = 7
    s = _rollout_env(env, K)
    rho = s.rho.clone().requires_grad_(True)
    q = s.q.clone().requires_grad_(True)
    E = s.E.clone().requires_grad_(True)
    rK, qK, EK = Sod2dRollout.apply(gm, s, rho, q, E, K, 3)
    loss = 0.5 * (qK * qK).sum()
    loss.backward()
    g = (t2n(rho.grad), t2n(q.grad), t2n(E.grad))
    mus, dts = trajectory_coefficients(gm, s, K)
    # (a) oracle forward mode through the same K frozen steps
    st = env["st"]["st1"].copy()
    rng = np.random.default_rng(8)
    v = _rand_dir(rng, st)
    cur, dv = st, (v[0], v[1], v[2])
    for n in range(K):
        cur = cur.copy()
        cur.mu_e = t2n(mus[n])
        y1, dy1 = _oracle_step_jvp(oracle, env, cur, float(dts[n].item()), dv)
        cur = _with(cur, *y1)
        dv = tuple(dy1)
    dL_oracle = (cur.q * dv[1]).sum()
    vq = v[1].T  # (3, N): the torch layout of q
    dL_adj = (g[0] * v[0]).sum() + (g[1] * v[1]).sum() + (g[2] * v[2]).sum()
    assert abs(dL_adj - dL_oracle) <= 1e-10 * abs(dL_oracle), f"{dL_adj:.15e} vs {dL_oracle:.15e}"

    # (b) central differences of the frozen-coefficient forward map on the GPU
    def L_at(h):
        t = _clone_state(s)
        t.rho.add_(h * _dev(torch, v[0]))
        t.q.add_(h * _dev(torch, vq))
        t.E.add_(h * _dev(torch, v[2]))
        replay(gm, t, mus, dts)
        return 0.5 * float((t.q * t.q).sum().item())
    for h in (1e-4, 1e-6):
        fd = (L_at(h) - L_at(-h)) / (2 * h)
        assert abs(fd - dL_adj) <= FD_TOL * abs(dL_adj), f"h={h}: fd {fd:.12e} adjoint {dL_adj:.12e}"


def test_stored_stages_match_recompute(env):
    """sod_rk4_main_record + stored stages gives the same step and VJP, bit for bit."""
    torch, gm, S = env["torch"], env["gm"], env["S"]
    st = env["st"]["st1"]
    a = S.Sod2dState.from_host(st, gm.nelem); a.dt.fill_(env["dt"])
    b = S.Sod2dState.from_host(st, gm.nelem); b.dt.fill_(env["dt"])
    stages = torch.empty(15 * gm.npoin, dtype=torch.float64, device="cuda")
    x0 = (a.rho.clone(), a.q.clone(), a.E.clone(), a.mu_e.clone(), a.dt.clone())
    gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    gm.rk_4_main_record(b, stages, update_dt=True)  # FP64
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "dt", "u", "pr", "eta"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    rng = np.random.default_rng(6)
    wb = _rand_dir(rng, st)
    bars = (_dev(torch, wb[0]), _dev(torch, wb[1].T), _dev(torch, wb[2]))
    r1 = gm.rk4_step_vjp(x0[0], x0[1], x0[2], x0[3], b.mu_factor, x0[4], *bars)
    r2 = gm.rk4_step_vjp(x0[0], x0[1], x0[2], x0[3], b.mu_factor, x0[4], *bars, stages=stages)
    torch.cuda.synchronize()
    for u, v in zip(r1, r2):
        assert torch.equal(u, v)


def test_rollout_checkpoint_spacing_invariant(env):
    """The gradient does not depend on the checkpoint spacing, on stored vs recomputed stage
    states, nor on keeping the forward's trajectory (bitwise: the re-forward is
    deterministic)."""
    from sod2d_refmap_b200.adjoint import Sod2dRollout
    torch, gm, S = env["torch"], env["gm"], env["S"]
    grads = []
    for every, store, keep in ((1, True, False), (2, True, False), (5, True, False), (2, False, False),
                               (2, True, True)):
        s = _rollout_env(env, 5)
        rho = s.rho.clone().requires_grad_(True)
        q = s.q.clone().requires_grad_(True)
        E = s.E.clone().requires_grad_(True)
        _, qK, _ = Sod2dRollout.apply(gm, s, rho, q, E, 5, every, store, S.FP64, keep)
        (0.5 * (qK * qK).sum()).backward()
        grads.append((rho.grad.clone(), q.grad.clone(), E.grad.clone()))
    for other in grads[1:]:
        for a, b in zip(grads[0], other):
            assert torch.equal(a, b)


def test_mixed_trajectory_adjoint_close_to_fp64(env):
    """Adjoint along the mixed-precision trajectory (FP64 step VJPs at the mixed stage states):
    the recorded mixed step equals sod_rk4_main(SOD_MIXED) bit for bit, and the directional
    derivative stays within 1e-5 of the FP64 one (the mixed state differs by ~1e-9)."""
    from sod2d_refmap_b200.adjoint import Sod2dRollout
    torch, gm, S = env["torch"], env["gm"], env["S"]
    st = env["st"]["st1"]
    a = S.Sod2dState.from_host(st, gm.nelem); a.dt.fill_(env["dt"])
    b = S.Sod2dState.from_host(st, gm.nelem); b.dt.fill_(env["dt"])
    stages = torch.empty(15 * gm.npoin, dtype=torch.float64, device="cuda")
    gm.rk_4_main(a, precision=S.MIXED, update_dt=True)
    gm.rk_4_main_record(b, stages, update_dt=True, precision=S.MIXED)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    rng = np.random.default_rng(12)
    v = [_dev(torch, x) for x in (lambda d: (d[0], d[1].T, d[2]))(_rand_dir(rng, st))]
    dl = {}
    for prec in (S.FP64, S.MIXED):
        s = _rollout_env(env, 4)
        rho = s.rho.clone().requires_grad_(True)
        q = s.q.clone().requires_grad_(True)
        E = s.E.clone().requires_grad_(True)
        _, qK, _ = Sod2dRollout.apply(gm, s, rho, q, E, 4, 2, True, prec)
        (0.5 * (qK * qK).sum()).backward()
        dl[prec] = float(sum((g * w).sum() for g, w in zip((rho.grad, q.grad, E.grad), v)).item())
    assert abs(dl[S.MIXED] - dl[S.FP64]) <= 1e-5 * abs(dl[S.FP64]), dl
