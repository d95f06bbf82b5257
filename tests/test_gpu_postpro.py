"""compute_fieldDerivs (mod_postpro.f90:12-139) on the device against the oracle: a jittered TGV
state (1e-12 relative per output) and the closed forms on an undistorted channel (1e-10)."""
import numpy as np
import pytest

from _util import rel_l2
from test_oracle_postpro import linear_case

pytestmark = pytest.mark.gpu


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


def test_field_derivs_vs_oracle(torch_mod, oracle):
    from sod2d_refmap_b200 import mesh as M, solver as S
    torch = torch_mod
    m = M.periodic_box(4, jitter=0.05, seed=9)
    prm = M.TGVParams()
    st = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=9)
    ref = oracle.compute_field_derivs(oracle.OracleMesh(m), st.rho, st.u)
    gm = S.Sod2dMesh(m, prm)
    out = gm.compute_field_derivs(dev(torch, st.rho), dev(torch, st.u))
    got = [out[0].cpu().numpy().T, out[1].cpu().numpy().T, out[2].cpu().numpy(), out[3].cpu().numpy()]
    for name, a, r in zip(("gradRho", "curlU", "divU", "Qcrit"), got, ref):
        assert rel_l2(a, r) < 1e-12, name
    # an explicit symbol gives the same as the default one, its negative flips the curl
    lv = oracle.levi_civita()
    o2 = gm.compute_field_derivs(dev(torch, st.rho), dev(torch, st.u), leviCivi=lv)
    o3 = gm.compute_field_derivs(dev(torch, st.rho), dev(torch, st.u), leviCivi=-lv)
    assert torch.equal(o2[1], out[1]) and torch.equal(o3[1], -out[1]) and torch.equal(o3[3], out[3])
    gm.close()


def test_field_derivs_exact_fields(torch_mod):
    from sod2d_refmap_b200 import mesh as M, solver as S
    torch = torch_mod
    m, rho, u, exact = linear_case(M)
    gm = S.Sod2dMesh(m, M.TGVParams())
    g, c, dv, qc = gm.compute_field_derivs(dev(torch, rho), dev(torch, u))
    for got, ref in ((g.cpu().numpy().T, exact["gradRho"]), (c.cpu().numpy().T, exact["curlU"]),
                     (dv.cpu().numpy(), exact["divU"]), (qc.cpu().numpy(), exact["Qcrit"])):
        assert np.abs(got - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())
    gm.close()
