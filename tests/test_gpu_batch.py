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


def _batch(M, S, prm, sizes, res, seed0=50):
    meshes = [M.periodic_box(n, jitter=0.05, seed=seed0 + i) for i, n in enumerate(sizes)]
    states = [M.taylor_green_state(m, prm, seed=seed0 + 10 + i, re=re) for i, (m, re) in enumerate(zip(meshes, res))]
    return meshes, states


@pytest.mark.parametrize("shape", ["two_launches", "one_launch"])
def test_batch_members_match_oracle(oracle, shape):
    """Every member of an FP64 ensemble against the oracle's rk_4_main on that member alone, with
    the member's own Re and dt (3 steps, dt from each member's CFL condition): <= 1e-12, with the
    stage run as two launches and as one cooperative launch per stage."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    prm = M.TGVParams()
    meshes, states = _batch(M, S, prm, [2, 3, 4], [400.0, 1600.0, 3200.0])
    B = S.Sod2dBatch(meshes, states, prm)
    B.set_stage_launch(S.FP64, 0 if shape == "two_launches" else 32)
    B.adapt_dt()
    B.rk4_steps(3, precision=S.FP64)
    torch.cuda.synchronize()
    for i, (m, st) in enumerate(zip(meshes, states)):
        om = oracle.OracleMesh(m)
        ref = st.copy()
        dt = oracle.adapt_dt(om, ref, prm)
        for _ in range(3):
            oracle.rk4(om, prm, ref, dt, nsteps=1)
            dt = oracle.adapt_dt(om, ref, prm)
        got = B.get_member(i)
        for k in ("rho", "q", "E", "u", "pr", "Tem", "eta", "mu_fluid", "mu_e"):
            err = rel_l2(got[k], getattr(ref, k))
            assert err < 1e-12, (shape, i, k, err)
        assert abs(B.dt()[i] - dt) <= 1e-13 * dt
    B.close()


@pytest.mark.parametrize("prec", ["FP64", "MIXED"])
def test_one_launch_stage_matches_two_launches(prec):
    """The cooperative one-launch-per-stage step computes every element and node as the
    two-launch step does; only the blocking of the entropy sums differs (the state to 1e-13,
    mu_e, which divides by the spread of eta, to 1e-12).  Its captured graph replays equal its
    eager steps bit for bit, and a step is four of the library's launches."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S, _lib
    build.build()
    p = getattr(S, prec)
    prm = M.TGVParams()
    meshes, states = _batch(M, S, prm, [3, 5, 2], [800.0, 1600.0, 2400.0], seed0=70)
    runs = {}
    for shape, ctas in (("two", 0), ("one", 32)):
        B = S.Sod2dBatch(meshes, states, prm)
        B.set_stage_launch(p, ctas)
        B.adapt_dt()
        B.rk4_steps(3, precision=p)
        torch.cuda.synchronize()
        runs[shape] = [B.get_member(i) for i in range(len(meshes))]
        B.close()
    for i in range(len(meshes)):
        a, b = runs["two"][i], runs["one"][i]
        for k in ("rho", "q", "E"):
            assert rel_l2(b[k], a[k]) < 1e-13, (prec, i, k)
        assert rel_l2(b["mu_e"], a["mu_e"]) < 1e-12, (prec, i)
    # one mesh: graph replays == eager steps, and the launch count of a step
    m = M.periodic_box(4, jitter=0.05, seed=5)
    st = M.taylor_green_state(m, prm)
    gm = S.Sod2dMesh(m, prm)
    gm.set_stage_launch(p, 32)
    x = S.Sod2dState.from_host(st, gm.nelem); gm.adapt_dt(x)
    y = S.Sod2dState.from_host(st, gm.nelem); y.dt.copy_(x.dt)
    gm.rk_4_main(x, precision=p, update_dt=True)   # first call: buffers allocated
    torch.cuda.synchronize()
    n0 = _lib.launch_count()
    gm.rk_4_main(x, precision=p, update_dt=True)
    n1 = _lib.launch_count()
    extra = 2 if prec == "MIXED" else 1              # the mu_e layout copies (and its FP32 copy)
    assert n1 - n0 == 4 + 1 + extra, n1 - n0
    gm.rk_4_main(y, precision=p, update_dt=True)
    gm.rk4_steps(y, 1, precision=p)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "dt"):
        assert torch.equal(getattr(x, k), getattr(y, k)), k
    gm.close()


def test_autotune_sweeps_two_dimensions():
    """The tuner's table covers elements per CTA {1,2,4,8} and, for each, the two-launch stage and
    at least one cooperative shape; its choice is one of the rows, and the step it configures
    matches the FP64 oracle-checked two-launch step."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S
    build.build()
    prm = M.TGVParams()
    m = M.periodic_box(6, jitter=0.05, seed=8)
    gm = S.Sod2dMesh(m, prm)
    s = S.Sod2dState.from_host(M.taylor_green_state(m, prm), gm.nelem)
    for p in (S.FP64, S.MIXED):
        best, _ = gm.autotune(s, p)
        table = gm.autotune_table(p)
        print("autotune", p, table)
        assert {r[0] for r in table} == {1, 2, 4, 8}
        for epb in (1, 2, 4, 8):
            shapes = [r[1] for r in table if r[0] == epb]
            assert 0 in shapes and any(c > 0 for c in shapes), (p, epb, shapes)
        assert best in (1, 2, 4, 8) and all(r[2] > 0 for r in table)
    gm.close()
