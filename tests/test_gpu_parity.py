"""CUDA path (through the C ABI) against the CPU oracle on seeded inputs.

Tolerances: FP64 path <= 1e-12 relative L2 per field (the reference's FP64 path, written in
each assertion); mixed path bounds are stated per test.
"""
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
    m = M.periodic_box(4, jitter=0.05, seed=2)
    prm = M.TGVParams()
    om = oracle.OracleMesh(m)
    gm = S.Sod2dMesh(m, prm)
    st0 = M.taylor_green_state(m, prm)
    dt = oracle.adapt_dt(om, st0, prm)
    st1 = st0.copy()
    oracle.rk4(om, prm, st1, dt, nsteps=1)   # a state with mu_e > 0
    return dict(M=M, S=S, m=m, prm=prm, om=om, gm=gm, st0=st0, st1=st1, dt=dt, torch=torch)


def test_geometry_parity(env):
    om, gm = env["om"], env["gm"]
    g = gm.geometry()
    assert rel_l2(g["He"], om.He) < 1e-13
    assert rel_l2(g["gpvol"], om.gpvol) < 1e-13
    assert rel_l2(g["Ml"], om.Ml) < 1e-13
    assert np.array_equal(g["helem"], om.helem) or rel_l2(g["helem"], om.helem) < 1e-15
    assert rel_l2(g["helem_l"], om.helem_l) < 1e-15


def test_adapt_dt_parity(env):
    S, gm, st0, dt = env["S"], env["gm"], env["st0"], env["dt"]
    s = S.Sod2dState.from_host(st0, gm.nelem)
    got = float(gm.adapt_dt(s).item())
    assert abs(got - dt) <= 1e-14 * dt


@pytest.mark.parametrize("which", ["st0", "st1"])
def test_rhs_fp64_parity(env, oracle, which):
    """Stage-1 residual R/Ml of rk_4_main (time_integ.f90:266-393) at a given state."""
    S, gm, om, prm = env["S"], env["gm"], env["om"], env["prm"]
    st = env[which]
    ref = oracle.rk4(om, prm, st.copy(), env["dt"], nsteps=1, capture_stage=1)
    s = S.Sod2dState.from_host(st, gm.nelem)
    out = gm.rhs(s, precision=S.FP64)
    env["torch"].cuda.synchronize()
    for k in ("Rmass", "Rmom", "Rener", "Reta"):
        err = rel_l2(t2n(out[k]), ref[k])
        assert err < TOL64, f"{k}: rel L2 {err:.3e}"


def test_rk4_fp64_parity(env, oracle):
    """Three rk_4_main steps at fixed dt (time_integ.f90:137-508) incl. EOS, mu_fluid and mu_e."""
    S, gm, om, prm, dt = env["S"], env["gm"], env["om"], env["prm"], env["dt"]
    ref = env["st0"].copy()
    oracle.rk4(om, prm, ref, dt, nsteps=3)
    s = S.Sod2dState.from_host(env["st0"], gm.nelem)
    s.dt.fill_(dt)
    for _ in range(3):
        gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    h = s.to_host()
    for k in ("rho", "q", "E", "u", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid", "mu_e"):
        err = rel_l2(h[k], getattr(ref, k))
        assert err < TOL64, f"{k}: rel L2 {err:.3e}"


def test_graph_steps_bitwise_match_eager(env):
    """sod_rk4_steps (captured graph, dt on device) == repeated sod_rk4_main, bit for bit."""
    S, gm, st0, dt = env["S"], env["gm"], env["st0"], env["dt"]
    a = S.Sod2dState.from_host(st0, gm.nelem); a.dt.fill_(dt)
    b = S.Sod2dState.from_host(st0, gm.nelem); b.dt.fill_(dt)
    for _ in range(4):
        gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    gm.rk4_steps(b, 4, precision=S.FP64)
    env["torch"].cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "dt"):
        assert env["torch"].equal(getattr(a, k), getattr(b, k)), k


def test_rhs_configs_bitwise_equal(env):
    """Every elements-per-CTA configuration of the fused RHS computes each element with the same
    operations: outputs bit for bit equal; unknown configurations are refused."""
    from sod2d_refmap_b200 import _lib
    S, gm, st1, torch = env["S"], env["gm"], env["st1"], env["torch"]
    for prec, cfgs in ((S.FP64, (1, 2, 4, 8)), (S.MIXED, (1, 2, 4, 8))):
        outs = []
        for c in cfgs:
            gm.set_rhs_config(prec, c)
            s = S.Sod2dState.from_host(st1, gm.nelem)
            outs.append({k: v.clone() for k, v in gm.rhs(s, precision=prec).items()})
        for o in outs[1:]:
            for k in o:
                assert torch.equal(o[k], outs[0][k]), (prec, k)
        with pytest.raises(_lib.SodError, match="SOD_ERR_ARG"):
            gm.set_rhs_config(prec, 3)
        gm.set_rhs_config(prec, 0)


def test_deterministic(env):
    S, gm, st1 = env["S"], env["gm"], env["st1"]
    outs = []
    for _ in range(2):
        s = S.Sod2dState.from_host(st1, gm.nelem)
        outs.append(gm.rhs(s, precision=S.FP64))
    for k in outs[0]:
        assert env["torch"].equal(outs[0][k], outs[1][k])


def test_per_routine_parity(env, oracle):
    """full_convec_ijk / generic_scalar_convec_ijk / full_diffusion_ijk / smart_visc_spectral
    through their reference argument lists, on independent (non-EOS-consistent) inputs."""
    torch, S, gm, om, prm, m = env["torch"], env["S"], env["gm"], env["om"], env["prm"], env["m"]
    rng = np.random.default_rng(11)
    N, E = m.npoin, m.nelem
    st = env["st1"]
    u = np.asfortranarray(st.u + 0.01 * rng.standard_normal((N, 3)))
    q = np.asfortranarray(st.q + 0.01 * rng.standard_normal((N, 3)))
    rho = st.rho + 0.01 * rng.standard_normal(N)
    pr = st.pr + 0.01 * rng.standard_normal(N)
    h = 250.0 + rng.standard_normal(N)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).cuda()
    Rm, Rmo, Re = gm.full_convec_ijk(dev(u), dev(q), dev(rho), dev(pr), dev(h))
    rm, rmo, re = oracle.convec(om, u, q, rho, pr, h)
    assert rel_l2(t2n(Rm), rm) < TOL64 and rel_l2(t2n(Rmo), rmo) < TOL64 and rel_l2(t2n(Re), re) < TOL64
    eta = st.eta + 0.01 * rng.standard_normal(N)
    f = np.asfortranarray(rng.standard_normal((N, 3)))
    Rt = gm.generic_scalar_convec_ijk(dev(f), dev(eta), dev(u))
    assert rel_l2(t2n(Rt), oracle.scalar_convec(om, f, eta, u)) < TOL64
    mue = np.asfortranarray(1e-3 * rng.random((E, 64)))
    musgs = np.asfortranarray(1e-4 * rng.random((E, 64)))
    Dm, Dmo, De = gm.full_diffusion_ijk(dev(rho), dev(rho), dev(u), dev(st.Tem), dev(st.mu_fluid), dev(mue), dev(musgs))
    dm, dmo, de = oracle.diffusion(om, prm, rho, rho, u, st.Tem, st.mu_fluid, mue, musgs)
    assert rel_l2(t2n(Dm), dm) < TOL64 and rel_l2(t2n(Dmo), dmo) < TOL64 and rel_l2(t2n(De), de) < TOL64
    Reta = rng.standard_normal(N) * 0.1
    mu_gpu = gm.smart_visc_spectral(dev(Reta), dev(st.rho), dev(st.u), dev(st.csound), dev(st.Tem), dev(st.eta))
    mu_ref = oracle.smart_visc(om, prm, Reta, st.rho, st.u, st.csound, st.Tem, st.eta, st.mu_e)
    assert rel_l2(t2n(mu_gpu), mu_ref) < TOL64
    R = dev(rm.copy())
    gm.lumped_solver(R)
    assert rel_l2(t2n(R), rm / om.Ml) < 1e-14   # Ml assembled in a different order
    mu = S.sutherland_viscosity(dev(st.Tem), dev(st.mu_factor))
    ref_mu = st.mu_factor * 0.000001458 * st.Tem ** 1.5 / (st.Tem + 110.4)
    assert rel_l2(t2n(mu), ref_mu) < 1e-15


def test_csr_spmv_kat_gpu(env, kats):
    torch, S = env["torch"], env["S"]
    k = kats["csr_spmv"]
    t = lambda v, dt: torch.tensor(v, dtype=dt, device="cuda")
    u = S.csr_spmv_scal(t(k["rdom"], torch.int32), t(k["cdom"], torch.int32), t(k["Mc"], torch.float64),
                        t(k["v"], torch.float64))
    assert u.cpu().tolist() == [25.0, 54.0, 29.0, 34.0, 72.0, 38.0]


def test_mixed_precision_error(env, oracle):
    """Mixed path: stage RHS per-field rel L2 vs FP64 and the state after 10 RK4 steps."""
    S, gm, st1 = env["S"], env["gm"], env["st1"]
    s = S.Sod2dState.from_host(st1, gm.nelem)
    r64 = gm.rhs(s, precision=S.FP64)
    r32 = gm.rhs(s, precision=S.MIXED)
    errs = {k: rel_l2(t2n(r32[k]), t2n(r64[k])) for k in r64}
    print("mixed RHS rel L2:", errs)
    # 5e-6 on this 4^3 box (measured <= 2.2e-6): an element spans 1.6 rad of the vortex, so the
    # second-order remainder the mixed kernel rounds to FP32 is far larger relative to the fields
    # than on the 64^3 benchmark mesh, where the 1e-6 bound is checked (test_gpu_configs.py)
    for k, e in errs.items():
        assert e < 5e-6, (k, e)
    a = S.Sod2dState.from_host(env["st0"], gm.nelem); a.dt.fill_(env["dt"])
    b = S.Sod2dState.from_host(env["st0"], gm.nelem); b.dt.fill_(env["dt"])
    gm.rk4_steps(a, 10, precision=S.FP64)
    gm.rk4_steps(b, 10, precision=S.MIXED)
    serr = {k: rel_l2(t2n(getattr(b, k)), t2n(getattr(a, k))) for k in ("rho", "q", "E")}
    print("mixed state rel L2 after 10 steps:", serr)
    for k, e in serr.items():
        assert e < 1e-6, (k, e)


def test_step_capturable_in_caller_graph(env):
    """sod_rk4_main allocates and synchronizes nothing after its first call, so a caller can
    capture it in its own CUDA graph; replays equal eager steps bit for bit (mixed, dt updated)."""
    S, gm, torch = env["S"], env["gm"], env["torch"]
    a = S.Sod2dState.from_host(env["st0"], gm.nelem); a.dt.fill_(env["dt"])
    b = S.Sod2dState.from_host(env["st0"], gm.nelem); b.dt.fill_(env["dt"])
    warm = S.Sod2dState.from_host(env["st0"], gm.nelem); warm.dt.fill_(env["dt"])
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        gm.rk_4_main(warm, precision=S.MIXED, update_dt=True)  # first call: buffers allocated here
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        gm.rk_4_main(a, precision=S.MIXED, update_dt=True)
    for _ in range(3):
        g.replay()
        gm.rk_4_main(b, precision=S.MIXED, update_dt=True)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
