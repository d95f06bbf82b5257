"""Pressure Poisson operator and PCG (lib_sod2d_incomp) against the oracle."""
import numpy as np
import pytest

from _util import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def penv(oracle):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    m = M.periodic_box(4, jitter=0.05, seed=6)
    om = oracle.OracleMesh(m)
    gm = S.Sod2dMesh(m, M.TGVParams())
    P = S.Sod2dPoisson(gm)
    rng = np.random.default_rng(7)
    rhs = rng.standard_normal(m.npoin)
    rhs -= rhs.mean()
    return dict(torch=torch, m=m, om=om, gm=gm, P=P, rhs=rhs)


def test_laplacian_mult_parity(penv, oracle):
    """eval_laplacian_mult (mod_operators.f90:20-128) via the assembled CSR, incl. the pinned node."""
    torch, P, om, m = penv["torch"], penv["P"], penv["om"], penv["m"]
    x = np.random.default_rng(3).standard_normal(m.npoin)
    y = P.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = oracle.laplacian_mult(om, x)
    assert rel_l2(y, ref) < 1e-12
    assert y[0] == 0.0


def test_laplacian_diag_parity(penv, oracle):
    d = penv["P"].diag().cpu().numpy()
    assert rel_l2(d, oracle.laplacian_diag(penv["om"])) < 1e-12


def test_cg_fp64_matches_oracle(penv, oracle):
    """conjGrad_pressure_incomp (mod_solver_incomp.f90:247-434) to ||r|| < 1e-10 ||r0||."""
    torch, P, om, rhs = penv["torch"], penv["P"], penv["om"], penv["rhs"]
    x, it, rel = P.solve(torch.from_numpy(rhs).cuda(), tol=1e-10)
    xr, itr, relr = oracle.conjgrad_pressure(om, rhs, tol=1e-10)
    assert rel < 1e-10 and relr < 1e-10
    assert abs(it - itr) <= 2, (it, itr)
    assert rel_l2(x.cpu().numpy(), xr) < 1e-8


def test_cg_mixed_refinement(penv):
    """FP32 inner PCG + FP64 residual refinement reaches the same FP64 tolerance."""
    torch, P, rhs = penv["torch"], penv["P"], penv["rhs"]
    b = torch.from_numpy(rhs).cuda()
    x64, it64, _ = P.solve(b, tol=1e-10)
    x32, it32, rel32 = P.solve(b, tol=1e-10, mixed=True)
    assert rel32 < 1e-10
    assert rel_l2(x32.cpu().numpy(), x64.cpu().numpy()) < 1e-8
    # the true FP64 residual of the mixed solution
    r = b.clone(); r[0] = 0.0
    res = (r - P.apply(x32)).norm().item() / r.norm().item()
    assert res < 1e-9, res


def test_cg_iteration_limit(penv):
    """The device-side iteration limit ends the batched replays at exactly max_iter (not a
    multiple of the 16-iteration batch) and the call reports non-convergence."""
    torch, P, rhs = penv["torch"], penv["P"], penv["rhs"]
    b = torch.from_numpy(rhs).cuda()
    with pytest.raises(RuntimeError, match="after 21 iterations"):
        P.solve(b, tol=1e-10, max_iter=21)
    # the handle stays usable: the next solve converges as before
    _, it, rel = P.solve(b, tol=1e-10)
    assert rel < 1e-10 and it > 21


def test_cg_zero_rhs(penv):
    torch, P = penv["torch"], penv["P"]
    x, it, rel = P.solve(torch.zeros(P.n, dtype=torch.float64, device="cuda"), tol=1e-10)
    assert it == 0 and rel == 0.0 and float(x.abs().max()) == 0.0
