"""Failure detection without a GPU fault: a NaN planted in the host input state (data, not a
bad access) raises the step's non-finite flag, and a host-side wait limit expires while a CG
solve is still queued (the device work completes on its own)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(oracle):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    m = M.periodic_box(4, jitter=0.05, seed=3)
    prm = M.TGVParams()
    gm = S.Sod2dMesh(m, prm)
    st = M.taylor_green_state(m, prm)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st, prm)
    return dict(M=M, S=S, m=m, prm=prm, gm=gm, st=st, dt=dt, torch=torch)


def test_nonfinite_flag(env):
    from sod2d_refmap_b200 import _lib
    S, gm, st, dt = env["S"], env["gm"], env["st"], env["dt"]
    s = S.Sod2dState.from_host(st, gm.nelem)
    s.dt.fill_(dt)
    gm.rk_4_main(s, precision=S.FP64, update_dt=False)
    gm.check_finite()                     # clean step: no error
    bad = st.copy()
    bad.rho[17] = np.nan
    t = S.Sod2dState.from_host(bad, gm.nelem)
    t.dt.fill_(dt)
    gm.rk4_steps(t, 2, precision=S.MIXED)
    with pytest.raises(_lib.SodError, match="SOD_ERR_NONFINITE"):
        gm.check_finite()
    gm.check_finite()                     # the flag was cleared by the check


def test_nonfinite_host_step(env):
    from sod2d_refmap_b200 import _lib
    S, gm, st, dt = env["S"], env["gm"], env["st"], env["dt"]
    bad = st.copy()
    bad.E[5] = np.inf
    host = {f: np.asfortranarray(getattr(bad, f)) if hasattr(bad, f) else None for f in S.Sod2dState.FIELDS}
    host["Reta"] = np.zeros(env["m"].npoin)
    host["mu_sgs"] = None
    with pytest.raises(_lib.SodError, match="SOD_ERR_NONFINITE"):
        gm.rk4_main_host(host, dt, precision=S.FP64)
    gm.check_finite()


def test_wait_timeout(env):
    from sod2d_refmap_b200 import _lib, mesh as M, solver as S
    torch = env["torch"]
    m = M.periodic_box(16, jitter=0.05, seed=6)
    gm = S.Sod2dMesh(m, M.TGVParams())
    P = S.Sod2dPoisson(gm)
    rhs = np.random.default_rng(7).standard_normal(m.npoin)
    rhs -= rhs.mean()
    b = torch.from_numpy(rhs).cuda()
    P.solve(b, tol=1e-6)  # graphs built, device warm
    S.set_wait_timeout(0.01)
    try:
        # a fixed-length busy kernel (about 0.1 s) ahead of the solve on the same stream
        torch.cuda._sleep(int(2e8))
        with pytest.raises(_lib.SodError, match="SOD_ERR_TIMEOUT"):
            P.solve(b, tol=1e-10)
    finally:
        S.set_wait_timeout(0.0)
    torch.cuda.synchronize()              # the abandoned work ends by itself
    x, it, rel = P.solve(b, tol=1e-10)    # the handle is usable again
    assert rel < 1e-10 and it > 0
    P.close()
    gm.close()
