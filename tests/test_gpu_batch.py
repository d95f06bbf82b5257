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


def test_batch_mixed_ragged_with_autotune_and_set_dt():
    """Ragged members (1, 3 and 5 elements per side: a single periodic element among them), the
    mixed precision path, a tuned CTA shape and per-member time steps set by the caller: each
    member still advances as it does alone (the tuned shapes give bitwise the same residuals)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    prm = M.TGVParams()
    sizes = [1, 3, 5]
    meshes = [M.periodic_box(n, jitter=0.05 if n > 1 else 0.0, seed=30 + i) for i, n in enumerate(sizes)]
    states = [M.taylor_green_state(m, prm, pert_amp=1e-2, seed=40 + i) for i, m in enumerate(meshes)]
    B = S.Sod2dBatch(meshes, states, prm)
    B.adapt_dt()
    dts = 0.5 * B.dt()
    B.set_dt(dts)
    assert np.array_equal(B.dt(), dts)
    best, ms = B.autotune(S.MIXED)
    assert best in (1, 2, 4, 8) and ms > 0
    B.set_dt(dts)
    B.rk4_steps(2, precision=S.MIXED)
    torch.cuda.synchronize()
    for i, (m, st) in enumerate(zip(meshes, states)):
        gm = S.Sod2dMesh(m, prm)
        s = S.Sod2dState.from_host(st, gm.nelem)
        s.dt.fill_(float(dts[i]))
        gm.rk4_steps(s, 2, precision=S.MIXED)
        h = s.to_host()
        got = B.get_member(i)
        for k in ("rho", "q", "E", "mu_e", "eta"):
            err = rel_l2(got[k], h[k])
            assert err < 1e-12, (i, k, err)
        gm.close()
    B.close()
