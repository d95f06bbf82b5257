"""A mesh in SOD2D's own array form through the C ABI: every lattice point a row (coordPar),
connecParWork with periodic images replaced by their masters, and workingNodesPar as lpoin_w
(time_integ.f90:147,267-285,445-471; mod_solver.f90:23-58; mod_entropy_viscosity.f90:43-62).

The periodic slave rows must be left as they are by every step (rk_4_main's node loops run over
lpoin_w; the stage and update formulas give them a zero residual), except mu_fluid, which
sutherland_viscosity re-evaluates over all npoin from the row's own Tem.  On the working rows
the result must equal the unique-node mesh's result to rounding (same elements and gather order;
only the blocking of the entropy sums over the rows differs: 1e-14 on the state; mu_e divides by
the spread max|eta - mean(eta)|, about 1e-3 of eta, which amplifies the mean's rounding, so
1e-12 there) and the oracle's on the same arrays <= 1e-12.
"""
import ctypes as C

import numpy as np
import pytest

from _util import rel_l2, t2n

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
FIELDS = ("rho", "q", "E", "u", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid", "mu_e")


@pytest.fixture(scope="module")
def env(oracle):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S, _lib
    build.build()
    b = M.periodic_box(4, jitter=0.05, seed=2)
    f = M.sod2d_form(b)
    prm = M.TGVParams()
    st = M.taylor_green_state(b, prm)
    ob = oracle.OracleMesh(b)
    dt = oracle.adapt_dt(ob, st, prm)
    oracle.rk4(ob, prm, st, dt, nsteps=1)          # a state with mu_e > 0
    sf = M.expand_state(st, f)
    gb, gf = S.Sod2dMesh(b, prm), S.Sod2dMesh(f, prm)
    slave = np.setdiff1d(np.arange(f.npoin), f.extra["lpoin_w"])
    yield dict(torch=torch, M=M, S=S, L=_lib, b=b, f=f, prm=prm, st=st, sf=sf, dt=dt, gb=gb, gf=gf,
               of=oracle.OracleMesh(f), ru=f.extra["row_of_unique"], slave=slave)
    gb.close()
    gf.close()


def test_form_sizes(env):
    f, b = env["f"], env["b"]
    assert f.npoin == 13 ** 3 and len(f.extra["lpoin_w"]) == b.npoin == 12 ** 3
    assert f.extra["mas_sla"].shape == (13 ** 3 - 12 ** 3, 2)
    assert set(np.unique(f.connec)) == set(f.extra["lpoin_w"])


@pytest.mark.parametrize("prec", ["FP64", "MIXED"])
def test_steps_on_sod2d_arrays(env, oracle, prec):
    S, torch = env["S"], env["torch"]
    p = getattr(S, prec)
    a = S.Sod2dState.from_host(env["st"], env["gb"].nelem); a.dt.fill_(env["dt"])
    w = S.Sod2dState.from_host(env["sf"], env["gf"].nelem); w.dt.fill_(env["dt"])
    for _ in range(3):
        env["gb"].rk_4_main(a, precision=p, update_dt=True)
        env["gf"].rk_4_main(w, precision=p, update_dt=True)
    ha, hw = a.to_host(), w.to_host()
    ru, sl, sf = env["ru"], env["slave"], env["sf"]
    for k in FIELDS:
        if k == "mu_e":
            assert rel_l2(hw[k], ha[k]) < TOL64, k
            continue
        assert rel_l2(hw[k][ru], ha[k]) < 1e-14, k                     # working rows
        if k != "mu_fluid":
            assert np.array_equal(hw[k][sl], getattr(sf, k)[sl]), k     # slave rows untouched
    muf = env["M"].sutherland(sf.Tem[sl], sf.mu_factor[sl])
    assert rel_l2(hw["mu_fluid"][sl], muf) < 1e-15
    assert abs(float(w.dt.item()) - float(a.dt.item())) <= 1e-14 * float(a.dt.item())
    if prec == "FP64":  # and the oracle on the same arrays
        ref = sf.copy()
        d = env["dt"]
        for _ in range(3):
            oracle.rk4(env["of"], env["prm"], ref, d, nsteps=1)
            d = oracle.adapt_dt(env["of"], ref, env["prm"])
        for k in FIELDS:
            assert rel_l2(hw[k], getattr(ref, k)) < TOL64, k


def test_graph_steps_and_host_step(env):
    S, torch = env["S"], env["torch"]
    a = S.Sod2dState.from_host(env["sf"], env["gf"].nelem); a.dt.fill_(env["dt"])
    b = S.Sod2dState.from_host(env["sf"], env["gf"].nelem); b.dt.fill_(env["dt"])
    for _ in range(2):
        env["gf"].rk_4_main(a, precision=S.MIXED, update_dt=True)
    env["gf"].rk4_steps(b, 2, precision=S.MIXED)
    torch.cuda.synchronize()
    for k in ("rho", "q", "E", "mu_e", "mu_fluid", "dt"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    # the host-array step on the same rows
    c = S.Sod2dState.from_host(env["sf"], env["gf"].nelem); c.dt.fill_(env["dt"])
    env["gf"].rk_4_main(c, precision=S.FP64, update_dt=True)
    host = {}
    for k in S.Sod2dState.FIELDS:
        v = getattr(env["sf"], k, None)
        host[k] = None if v is None else np.array(v, order="F", copy=True)
    host["Reta"] = None
    dtn = env["gf"].rk4_main_host(host, env["dt"], precision=S.FP64)
    hc = c.to_host()
    for k in ("rho", "q", "E", "pr", "mu_fluid", "mu_e"):
        assert np.array_equal(host[k], hc[k]), k
    assert dtn == float(c.dt.item())


def test_rhs_and_routines_on_sod2d_arrays(env, oracle):
    """sod_rhs: slave rows 0, working rows == the unique mesh; the per-routine entries (slave
    rows 0, as the reference zeroes 1:npoin before the element scatter); the lumped solver
    leaves slave rows alone; smart_visc_spectral normalises over lpoin_w."""
    S, torch, ru, sl = env["S"], env["torch"], env["ru"], env["slave"]
    sb = S.Sod2dState.from_host(env["st"], env["gb"].nelem)
    sw = S.Sod2dState.from_host(env["sf"], env["gf"].nelem)
    rb = {k: t2n(v) for k, v in env["gb"].rhs(sb, precision=S.FP64).items()}
    rw = {k: t2n(v) for k, v in env["gf"].rhs(sw, precision=S.FP64).items()}
    for k in rb:
        assert np.array_equal(rw[k][ru], rb[k]), k
        assert not np.any(rw[k][sl]), k
    ref = oracle.rhs_stage(env["of"], env["prm"], env["sf"])
    assert rel_l2(rw["Rmass"], ref[0]) < TOL64 and rel_l2(rw["Rener"], ref[4]) < TOL64
    sf = env["sf"]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).cuda()
    Rm, Rmo, Re = env["gf"].full_convec_ijk(dev(sf.u), dev(sf.q), dev(sf.rho), dev(sf.pr), dev(sf.E))
    rm, rmo, re = oracle.convec(env["of"], sf.u, sf.q, sf.rho, sf.pr, sf.E)
    assert rel_l2(t2n(Rm), rm) < TOL64 and rel_l2(t2n(Rmo), rmo) < TOL64 and rel_l2(t2n(Re), re) < TOL64
    assert not np.any(t2n(Rm)[sl])
    R = dev(np.where(np.isin(np.arange(len(rm)), sl), 7.0, rm))
    env["gf"].lumped_solver(R)
    out = t2n(R)
    assert np.all(out[sl] == 7.0)
    lw = env["f"].extra["lpoin_w"]
    assert rel_l2(out[lw], rm[lw] / env["of"].Ml[lw]) < 1e-14
    rng = np.random.default_rng(4)
    Reta = rng.standard_normal(len(sf.rho)) * 0.1
    eta = sf.eta.copy()
    eta[sl] = 1e6                      # a slave row outside lpoin_w must not enter the mean/spread
    mu_w = env["gf"].smart_visc_spectral(dev(Reta), dev(sf.rho), dev(sf.u), dev(sf.csound), dev(sf.Tem), dev(eta))
    mu_r = oracle.smart_visc(env["of"], env["prm"], Reta, sf.rho, sf.u, sf.csound, sf.Tem, eta, sf.mu_e)
    assert rel_l2(t2n(mu_w), mu_r) < TOL64


def test_unsupported_with_slave_rows(env):
    S, L, torch = env["S"], env["L"], env["torch"]
    lib = L.load()
    P = C.c_void_p(0)
    assert lib.sod_poisson_create(env["gf"].handle, C.byref(P)) == -7
    assert b"slave" in lib.sod_last_error()
    sw = S.Sod2dState.from_host(env["sf"], env["gf"].nelem)
    with pytest.raises(L.SodError, match="SOD_ERR_UNSUPPORTED"):
        env["gf"].rhs_vjp(sw.rho, sw.q, sw.E, sw.mu_e, sw.mu_factor, sw.rho, sw.q, sw.E)


def test_lpoin_w_must_match_connec(env):
    """connec must reference exactly the working rows: a list that misses a referenced row, or
    that names a row no element holds, is refused."""
    S, L, M = env["S"], env["L"], env["M"]
    f = env["f"]
    lw = f.extra["lpoin_w"]
    for bad in (lw[1:], np.concatenate([lw, env["slave"][:1]])):
        g = M.BoxMesh(**{**f.__dict__, "extra": dict(f.extra, lpoin_w=np.sort(bad))})
        with pytest.raises(L.SodError, match="SOD_ERR_ARG"):
            S.Sod2dMesh(g, env["prm"])
