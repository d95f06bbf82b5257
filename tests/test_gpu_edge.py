"""Edge cases of the mesh handling against the oracle: a single periodic element (its 64 local
nodes map to 27 unique nodes, every one shared with the element's own periodic images) and a
27-element mesh, whose element count is not a multiple of the elements per CTA of any kernel
(partial CTAs everywhere).  FP64 bound 1e-12 relative per field; the mixed path 1e-3 on these
coarse meshes (the mixed tests' bound for 4^3)."""
import numpy as np
import pytest

from _util import rel_l2, t2n

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


@pytest.fixture(scope="module")
def mods():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    return torch, M, S


@pytest.mark.parametrize("n", [1, 3])
def test_rhs_and_step_parity_small(mods, oracle, n):
    torch, M, S = mods
    m = M.periodic_box(n, jitter=0.05 if n > 1 else 0.0, seed=12)
    prm = M.TGVParams()
    st0 = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=12)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    st1 = st0.copy()
    oracle.rk4(om, prm, st1, dt, nsteps=1)
    ref = oracle.rk4(om, prm, st1.copy(), dt, nsteps=1, capture_stage=1)
    gm = S.Sod2dMesh(m, prm)
    s = S.Sod2dState.from_host(st1, gm.nelem)
    out = gm.rhs(s, precision=S.FP64)
    for k in ("Rmass", "Rener", "Reta"):
        assert rel_l2(out[k].cpu().numpy(), ref[k]) < TOL64, (n, k)
    assert rel_l2(t2n(out["Rmom"]), ref["Rmom"]) < TOL64
    out32 = gm.rhs(s, precision=S.MIXED)
    for k in ("Rmass", "Rmom", "Rener"):
        assert rel_l2(t2n(out32[k]), t2n(out[k])) < 1e-3, (n, k)
    a = S.Sod2dState.from_host(st0, gm.nelem)
    a.dt.fill_(dt)
    gm.rk_4_main(a, precision=S.FP64, update_dt=True)
    h = a.to_host()
    for k in ("rho", "q", "E", "mu_e", "eta"):
        assert rel_l2(h[k], getattr(st1, k)) < TOL64, (n, k)
    assert abs(float(a.dt.item()) - oracle.adapt_dt(om, st1, prm)) <= 1e-13 * dt
    gm.close()


@pytest.mark.parametrize("n", [1, 3])
def test_poisson_small(mods, oracle, n):
    torch, M, S = mods
    m = M.periodic_box(n, jitter=0.05 if n > 1 else 0.0, seed=13)
    om = oracle.OracleMesh(m)
    gm = S.Sod2dMesh(m, M.TGVParams())
    P = S.Sod2dPoisson(gm)
    x = np.random.default_rng(5).standard_normal(m.npoin)
    y = P.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel_l2(y, oracle.laplacian_mult(om, x)) < TOL64
    rhs = np.random.default_rng(6).standard_normal(m.npoin)
    rhs -= rhs.mean()
    sol, it, rel = P.solve(torch.from_numpy(rhs).cuda(), tol=1e-10)
    ref, itr, relr = oracle.conjgrad_pressure(om, rhs, tol=1e-10)
    assert rel < 1e-10 and abs(it - itr) <= 2
    assert rel_l2(sol.cpu().numpy(), ref) < 1e-8
    P.close()
    gm.close()
