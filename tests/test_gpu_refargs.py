"""The reference subroutines through entry points that carry their complete argument lists
(full_convec_ijk, full_convec_ijk_H, generic_scalar_convec_ijk, full_diffusion_ijk,
smart_visc_spectral), called as SOD2D's time loop calls them: 1-based ids, Fortran layouts,
the mesh's own arrays on every call.  Checked against the oracle's restatement of each routine
(<= 1e-12) and against the handle-based entry points on the same geometry (bit for bit), on a
mesh in SOD2D's array form with periodic slave rows (their residuals stay zero, as the
reference zeroes 1:npoin before its element scatter), plus the argument checks."""
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
    from sod2d_refmap_b200 import build, mesh as M, solver as S, _lib
    build.build()
    b = M.periodic_box(3, jitter=0.05, seed=7)
    f = M.sod2d_form(b)
    prm = M.TGVParams()
    of = oracle.OracleMesh(f)
    st = M.expand_state(M.taylor_green_state(b, prm), f)
    ob = oracle.OracleMesh(b)
    sb = M.taylor_green_state(b, prm)
    oracle.rk4(ob, prm, sb, oracle.adapt_dt(ob, sb, prm), nsteps=1)
    st = M.expand_state(sb, f)                       # a state with mu_e > 0 on the SOD2D rows
    rng = np.random.default_rng(21)
    N, E = f.npoin, f.nelem
    fin = dict(u=np.asfortranarray(st.u + 0.01 * rng.standard_normal((N, 3))),
               q=np.asfortranarray(st.q + 0.01 * rng.standard_normal((N, 3))),
               rho=st.rho + 0.01 * rng.standard_normal(N), pr=st.pr + 0.01 * rng.standard_normal(N),
               h=250.0 + rng.standard_normal(N), eta=st.eta + 0.01 * rng.standard_normal(N),
               fe=np.asfortranarray(rng.standard_normal((N, 3))), Tem=st.Tem, muf=st.mu_fluid,
               mue=np.asfortranarray(1e-3 * rng.random((E, 64))), musgs=np.asfortranarray(1e-4 * rng.random((E, 64))),
               Reta=rng.standard_normal(N) * 0.1)
    d64 = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float64).ravel(order="F"))).cuda()
    d32 = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.int32).ravel(order="F"))).cuda()
    # the shape tables the handle-based mesh is built from (mesh.py), so that both paths see the
    # same D; the geometry is the oracle's
    tb = f.tables
    T = dict(connec=d32(of.connec + 1), Ngp=d64(tb.Ngp), dNgp=d64(tb.dNgp), He=d64(of.He), gpvol=d64(of.gpvol),
             dl=d64(tb.dlxigp_ip), xgp=d64(tb.xgp), inv=d32(tb.invAtoIJK + 1), gI=d32(tb.gmshAtoI + 1),
             gJ=d32(tb.gmshAtoJ + 1), gK=d32(tb.gmshAtoK + 1), wgp=d64(tb.wgp), Ml=d64(of.Ml), helem=d64(of.helem),
             helem_l=d64(of.helem_l), lw=d32(f.extra["lpoin_w"] + 1), coord=d64(f.coord))
    D = {k: d64(v) for k, v in fin.items()}
    gm = S.Sod2dMesh(f, prm, geometry=dict(He=of.He, gpvol=of.gpvol, Ml=of.Ml, helem=of.helem, helem_l=of.helem_l))
    slave = np.setdiff1d(np.arange(N), f.extra["lpoin_w"])
    yield dict(torch=torch, S=S, L=_lib, f=f, prm=prm, of=of, st=st, fin=fin, T=T, D=D, gm=gm, slave=slave, d32=d32)
    gm.close()


def _conv(env, total_enthalpy=False, T=None):
    S, f, D = env["S"], env["f"], env["D"]
    T = T or env["T"]
    return S.full_convec_ijk_ref(f.nelem, f.npoin, T["connec"], T["Ngp"], T["dNgp"], T["He"], T["gpvol"], T["dl"],
                                 T["xgp"], T["inv"], T["gI"], T["gJ"], T["gK"], D["u"], D["q"], D["rho"], D["pr"],
                                 D["h"], total_enthalpy=total_enthalpy)


@pytest.mark.parametrize("toth", [False, True])
def test_full_convec_ijk_ref(env, oracle, toth):
    fin, of, N = env["fin"], env["of"], env["f"].npoin
    Rm, Rmo, Re = (t.cpu().numpy() for t in _conv(env, toth))
    fn = oracle.convec_H if toth else oracle.convec
    rm, rmo, re = fn(of, fin["u"], fin["q"], fin["rho"], fin["pr"], fin["h"])
    assert rel_l2(Rm, rm) < TOL64 and rel_l2(Rmo, rmo.ravel(order="F")) < TOL64 and rel_l2(Re, re) < TOL64
    assert not np.any(Rm[env["slave"]]) and not np.any(Re[env["slave"]])
    # the handle-based entry point on the same geometry: the same kernels, bit for bit
    dv = lambda a: env["torch"].from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).cuda()
    g = env["gm"].full_convec_ijk_H if toth else env["gm"].full_convec_ijk
    hm, hmo, he = g(dv(fin["u"]), dv(fin["q"]), dv(fin["rho"]), dv(fin["pr"]), dv(fin["h"]))
    assert np.array_equal(hm.cpu().numpy(), Rm) and np.array_equal(he.cpu().numpy(), Re)
    assert np.array_equal(hmo.cpu().numpy().ravel(), Rmo)


def test_generic_scalar_and_diffusion_ref(env, oracle):
    S, f, T, D, fin, of, prm = env["S"], env["f"], env["T"], env["D"], env["fin"], env["of"], env["prm"]
    R = S.generic_scalar_convec_ijk_ref(f.nelem, f.npoin, T["connec"], T["Ngp"], T["dNgp"], T["He"], T["gpvol"],
                                        T["dl"], T["xgp"], T["inv"], T["gI"], T["gJ"], T["gK"], D["fe"], D["eta"],
                                        D["u"]).cpu().numpy()
    assert rel_l2(R, oracle.scalar_convec(of, fin["fe"], fin["eta"], fin["u"])) < TOL64
    Dm, Dmo, De = (t.cpu().numpy() for t in S.full_diffusion_ijk_ref(
        f.nelem, f.npoin, T["connec"], T["Ngp"], T["He"], T["gpvol"], T["dl"], T["inv"], T["gI"], T["gJ"], T["gK"],
        prm.Cp, prm.Prt, D["rho"], D["rho"], D["u"], D["Tem"], D["muf"], D["mue"], D["musgs"], T["Ml"]))
    dm, dmo, de = oracle.diffusion(of, prm, fin["rho"], fin["rho"], fin["u"], fin["Tem"], fin["muf"], fin["mue"],
                                   fin["musgs"])
    assert rel_l2(Dm, dm) < TOL64 and rel_l2(Dmo, dmo.ravel(order="F")) < TOL64 and rel_l2(De, de) < TOL64
    assert not np.any(Dm[env["slave"]])


def test_smart_visc_spectral_ref(env, oracle):
    S, f, T, D, fin, of, prm, st = env["S"], env["f"], env["T"], env["D"], env["fin"], env["of"], env["prm"], env["st"]
    dv = lambda a: env["torch"].from_numpy(np.ascontiguousarray(np.asarray(a).ravel(order="F"))).cuda()
    mu = S.smart_visc_spectral_ref(f.nelem, f.npoin, len(f.extra["lpoin_w"]), T["connec"], T["lw"], D["Reta"],
                                   T["Ngp"], T["coord"], T["dNgp"], T["gpvol"], T["wgp"], prm.gamma_gas, dv(st.rho),
                                   dv(st.u), dv(st.csound), dv(st.Tem), dv(st.eta), T["helem_l"], T["helem"], T["Ml"],
                                   T["inv"], T["gI"], T["gJ"], T["gK"], prm=prm).cpu().numpy()
    ref = oracle.smart_visc(of, prm, fin["Reta"], st.rho, st.u, st.csound, st.Tem, st.eta, st.mu_e)
    assert rel_l2(mu, ref.ravel(order="F")) < TOL64


def test_ref_entry_argument_checks(env):
    L, T, d32, f = env["L"], env["T"], env["d32"], env["f"]
    bad = T["connec"].clone()
    bad[3] = f.npoin + 1                              # one past the last 1-based id
    with pytest.raises(L.SodError, match="SOD_ERR_ARG"):
        _conv(env, T=dict(T, connec=bad))
    assert b"connec holds node ids" in L.load().sod_last_error()
    inv = T["inv"].clone()
    inv[[0, 1]] = inv[[1, 0]]                        # no longer the inverse of the gmshAto maps
    with pytest.raises(L.SodError, match="SOD_ERR_ARG"):
        _conv(env, T=dict(T, inv=inv))
    assert b"invAtoIJK" in L.load().sod_last_error()
    _conv(env)                                        # and a valid call afterwards
