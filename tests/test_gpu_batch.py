"""Ensemble batching: every member of a batch advances exactly as it does alone."""
import numpy as np
import pytest

from _util import rel_l2

pytestmark = pytest.mark.gpu


def test_batch_members_match_individual_runs():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    prm = M.TGVParams()
    sizes, res = [2, 3, 4], [400.0, 1600.0, 3200.0]
    meshes = [M.periodic_box(n, jitter=0.05, seed=10 + i) for i, n in enumerate(sizes)]
    states = [M.taylor_green_state(m, prm, seed=20 + i, re=re) for i, (m, re) in enumerate(zip(meshes, res))]
    B = S.Sod2dBatch(meshes, states, prm)
    B.adapt_dt()
    dts = B.dt()
    B.rk4_steps(3, precision=S.FP64)
    torch.cuda.synchronize()
    for i, (m, st) in enumerate(zip(meshes, states)):
        gm = S.Sod2dMesh(m, prm)
        s = S.Sod2dState.from_host(st, gm.nelem)
        gm.adapt_dt(s)
        assert abs(float(s.dt.item()) - dts[i]) <= 1e-14 * dts[i]
        gm.rk4_steps(s, 3, precision=S.FP64)
        h = s.to_host()
        got = B.get_member(i)
        for k in ("rho", "q", "E", "mu_e", "pr"):
            err = rel_l2(got[k], h[k])
            assert err < 1e-13, (i, k, err)
    assert np.all(B.dt() > 0)
    B.close()
