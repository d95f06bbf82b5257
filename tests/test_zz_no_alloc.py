"""The allocation-free full_convec_ijk entry point against the regular one and the oracle.

sod_full_convec_ijk_noalloc serves callers that cannot allocate device memory (their device
memory belongs to the OpenACC runtime or to a fixed pool of the host code), so it keeps its
scratch in a static device array instead of a SodMesh.  It must give the same residuals as
sod_full_convec_ijk on the same reference-layout inputs, call after call (the shared scratch
keeps the previous call's contents), with 1-based and 0-based ids, and must report bad node
ids and bad gmshAto tables (both kernels clamp such indices, so these cases read only valid
memory) and then work again.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from _util import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same FP64 arithmetic; only the element loop's data layout differs


def _setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S, _lib
    build.build()
    m = M.periodic_box(3, jitter=0.05, seed=4)
    prm = M.TGVParams()
    gm = S.Sod2dMesh(m, prm)
    geo = gm.geometry()
    st = M.taylor_green_state(m, prm)
    rng = np.random.default_rng(5)
    N = m.npoin
    f64 = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))).cuda()
    u = np.asfortranarray(st.u + 0.01 * rng.standard_normal((N, 3)))
    host = dict(u=u, q=st.q, rho=st.rho, pr=st.pr, E=3.5 * st.pr / st.rho)
    inp = {k: f64(v) for k, v in host.items()}
    return torch, S, _lib, m, gm, geo, inp, host, f64


def _mesh(torch, m, geo, base):
    i32 = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel(order="F"))).cuda()
    f64 = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))).cuda()
    T = m.tables
    return dict(connec=i32(np.asarray(m.connec) + base), He=f64(geo["He"]), gpvol=f64(geo["gpvol"]),
                dl=f64(T.dlxigp_ip), gI=i32(T.gmshAtoI + base), gJ=i32(T.gmshAtoJ + base), gK=i32(T.gmshAtoK + base))


def _noalloc(torch, _lib, m, mesh, inp, nelem=None, base=1):
    N = m.npoin
    out = [torch.full((N,), np.nan, dtype=torch.float64, device="cuda"),
           torch.full((3 * N,), np.nan, dtype=torch.float64, device="cuda"),
           torch.full((N,), np.nan, dtype=torch.float64, device="cuda")]
    p = lambda t: C.c_void_p(int(t.data_ptr()))
    rc = _lib.load().sod_full_convec_ijk_noalloc(
        m.nelem if nelem is None else nelem, N, base, p(mesh["connec"]), p(mesh["He"]), p(mesh["gpvol"]),
        p(mesh["dl"]), p(mesh["gI"]), p(mesh["gJ"]), p(mesh["gK"]), p(inp["u"]), p(inp["q"]), p(inp["rho"]),
        p(inp["pr"]), p(inp["E"]), p(out[0]), p(out[1]), p(out[2]),
        C.c_void_p(int(torch.cuda.current_stream().cuda_stream)))
    return rc, out


def _regular(gm, inp, N):
    Rm, Rmo, Re = gm.full_convec_ijk(inp["u"].view(3, N), inp["q"].view(3, N), inp["rho"], inp["pr"], inp["E"])
    return [Rm, Rmo.reshape(-1), Re]


def _close(torch, out, ref, what):
    torch.cuda.synchronize()
    for got, want in zip(out, ref):
        err = float((got - want).norm() / want.norm())
        assert err <= TOL, (what, err)


def test_noalloc_matches_regular_entry_point_twice(oracle):
    torch, S, _lib, m, gm, geo, inp, host, _ = _setup()
    N = m.npoin
    ref = _regular(gm, inp, N)
    mesh = _mesh(torch, m, geo, 1)
    for call in range(2):
        rc, out = _noalloc(torch, _lib, m, mesh, inp)
        assert rc == 0, _lib.load().sod_last_error()
        _close(torch, out, ref, call)
    # and against the oracle's full_convec_ijk directly
    om = oracle.OracleMesh(m)
    rm, rmo, re = oracle.convec(om, host["u"], host["q"], host["rho"], host["pr"], host["E"])
    got = [t.cpu().numpy() for t in out]
    assert rel_l2(got[0], rm) < TOL and rel_l2(got[1], rmo.ravel(order="F")) < TOL and rel_l2(got[2], re) < TOL


def test_noalloc_zero_based_ids():
    torch, S, _lib, m, gm, geo, inp, host, _ = _setup()
    ref = _regular(gm, inp, m.npoin)
    mesh = _mesh(torch, m, geo, 0)
    for call in range(2):
        rc, out = _noalloc(torch, _lib, m, mesh, inp, base=0)
        assert rc == 0, _lib.load().sod_last_error()
        _close(torch, out, ref, call)


@pytest.mark.parametrize("which", ["connec", "gI"])
def test_noalloc_reports_bad_ids_then_recovers(which):
    torch, S, _lib, m, gm, geo, inp, host, _ = _setup()
    ref = _regular(gm, inp, m.npoin)
    mesh = _mesh(torch, m, geo, 1)
    bad = mesh[which].clone()
    bad[5] = (m.npoin + 1) if which == "connec" else (4 + 1)   # one past the last valid 1-based id
    rc, _ = _noalloc(torch, _lib, m, dict(mesh, **{which: bad}), inp)
    assert rc == -1
    msg = _lib.load().sod_last_error()
    assert (b"connec holds node ids" in msg) if which == "connec" else (b"gmshAtoI/J/K" in msg), msg
    rc, out = _noalloc(torch, _lib, m, mesh, inp)
    assert rc == 0, _lib.load().sod_last_error()
    _close(torch, out, ref, "after error")


def test_noalloc_refuses_capturing_stream():
    torch, S, _lib, m, gm, geo, inp, host, _ = _setup()
    mesh = _mesh(torch, m, geo, 1)
    rc, _ = _noalloc(torch, _lib, m, mesh, inp)          # the device's first call happens outside capture
    assert rc == 0
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    rcs = []
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            rcs.append(_noalloc(torch, _lib, m, mesh, inp)[0])
    assert rcs == [-7], rcs
    assert b"capturing" in _lib.load().sod_last_error()


def test_noalloc_rejects_oversized_mesh():
    torch, S, _lib, m, gm, geo, inp, host, _ = _setup()
    mesh = _mesh(torch, m, geo, 1)
    rc, _ = _noalloc(torch, _lib, m, mesh, inp, nelem=4097)
    assert rc == -1
    assert b"4096 elements" in _lib.load().sod_last_error()
